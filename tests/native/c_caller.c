/* A plain C caller of libedp_b200 (no C++ and no Python): it checks the ABI
 * version and the status strings, which need no GPU. */
#include <stdio.h>
#include <string.h>

#include "edp.h"

int main(void) {
  if (edp_abi_version() != EDP_ABI_VERSION) {
    fprintf(stderr, "ABI version %d, header %d\n", edp_abi_version(), EDP_ABI_VERSION);
    return 1;
  }
  if (strcmp(edp_status_string(EDP_OK), "ok") != 0) return 2;
  if (strcmp(edp_status_string(EDP_ERR_ARGUMENT), "invalid argument") != 0) return 3;
  printf("abi %d metrics %d status %d\n", edp_abi_version(), EDP_METRICS, EDP_STATUS_SLOTS);
  return 0;
}
