// Exact-position vertex welding for callers that cannot allocate device memory.
//
// The workspace path (edp_event_create / edp_device_create) allocates its pools
// with cudaMalloc when it is created.  Some callers cannot do that at the
// point where they need welded ids: a plugin whose host framework owns every
// byte of device memory through its own arena or caching allocator (a raw
// cudaMalloc there fails or fragments the arena), and real-time or serving
// loops that forbid any allocation after start-up because an allocation can
// block on the driver and break their latency budget.  edp_weld_noalloc gives
// them the welding step on its own: the caller passes the vertex buffer and
// the output buffer, and the hash-table scratch lives in a fixed array below
// that every GPU loading this library holds until the process exits.
#include <climits>
#include <mutex>

#include "../../include/edp.h"
#include "edp_internal.h"

namespace {

constexpr int64_t kMaxVertices = EDP_WELD_NOALLOC_MAX_VERTICES;
constexpr int64_t kTableSlots = 2 * kMaxVertices;  // open addressing at <= 50% load
constexpr int kMaxDevices = 64;

struct WeldScratch {
  int table[kTableSlots];    // vertex index owning each slot, -1 when empty
  int minimum[kTableSlots];  // smallest vertex index with the slot's position
  int slot[kMaxVertices];    // slot of each vertex
};

// 5 MiB per device; shared by every call on that device.
static __device__ __align__(256) WeldScratch g_weld_scratch;

// Device address of g_weld_scratch per device, resolved on the first call made
// with that device current.  Only a successful lookup is cached, so a failed
// one (for example, a first call made inside a stream capture) is retried by
// the next call.
std::mutex g_scratch_mutex;
WeldScratch *g_scratch_ptr[kMaxDevices] = {};

__device__ inline uint64_t position_hash(const double *v) {
  uint64_t h = edp::mix64(edp::key_bits(v[0]));
  h = edp::mix64(h ^ edp::key_bits(v[1]));
  return edp::mix64(h ^ edp::key_bits(v[2]));
}

__global__ void k_noalloc_clear(WeldScratch *s, int mask) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i <= mask;
       i += int64_t(gridDim.x) * blockDim.x) {
    s->table[i] = -1;
    s->minimum[i] = INT_MAX;
  }
}

__global__ void k_noalloc_insert(const double *vertices, int nv, WeldScratch *s, int mask) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nv;
       i += int64_t(gridDim.x) * blockDim.x) {
    const double *v = vertices + 3 * i;
    uint32_t slot = uint32_t(position_hash(v)) & uint32_t(mask);
    for (int probe = 0; probe <= mask; ++probe) {
      int cur = atomicCAS(&s->table[slot], -1, int(i));
      if (cur == -1) break;
      const double *w = vertices + 3 * int64_t(cur);
      if (w[0] == v[0] && w[1] == v[1] && w[2] == v[2]) break;
      slot = (slot + 1) & uint32_t(mask);
    }
    atomicMin(&s->minimum[slot], int(i));
    s->slot[i] = int(slot);
  }
}

__global__ void k_noalloc_resolve(int nv, const WeldScratch *s, int *canonical) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nv;
       i += int64_t(gridDim.x) * blockDim.x)
    canonical[i] = s->minimum[s->slot[i]];
}

}  // namespace

#define EDP_NOALLOC_STR2(x) #x
#define EDP_NOALLOC_STR(x) EDP_NOALLOC_STR2(x)
#define EDP_NOALLOC_SITE __FILE__ ":" EDP_NOALLOC_STR(__LINE__)

extern "C" int edp_weld_noalloc(const double *vertices, int64_t nv, int32_t *canonical,
                                void *stream) {
  if (nv < 0 || nv > kMaxVertices) return EDP_ERR_ARGUMENT;
  if (nv == 0) return EDP_OK;
  if (!vertices || !canonical) return EDP_ERR_ARGUMENT;
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return edp::record_cuda_failure(e, EDP_NOALLOC_SITE);
  if (device < 0 || device >= kMaxDevices) return EDP_ERR_ARGUMENT;
  // Set-up, once per device with that device current: the symbol's name is a
  // host-side stand-in, so the kernels receive its device address instead.
  WeldScratch *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[device]) {
      void *ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_weld_scratch);
      if (e != cudaSuccess || !ptr)
        return edp::record_cuda_failure(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                                        EDP_NOALLOC_SITE);
      g_scratch_ptr[device] = static_cast<WeldScratch *>(ptr);
    }
    scratch = g_scratch_ptr[device];
  }
  const int mask = int(edp::pow2_at_least(2 * nv) - 1);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned clear_blocks = unsigned(edp::ceil_div(int64_t(mask) + 1, 256) < 1184
                                             ? edp::ceil_div(int64_t(mask) + 1, 256)
                                             : 1184);
  const unsigned blocks = unsigned(edp::ceil_div(nv, 256) < 1184 ? edp::ceil_div(nv, 256) : 1184);
  // Launch errors are read without clearing the thread's error state: an
  // error left pending by the caller's own earlier work stays pending for the
  // caller (this call reports it too, as EDP_ERR_CUDA).
  k_noalloc_clear<<<clear_blocks, 256, 0, st>>>(scratch, mask);
  if ((e = cudaPeekAtLastError()) != cudaSuccess)
    return edp::record_cuda_failure(e, EDP_NOALLOC_SITE);
  k_noalloc_insert<<<blocks, 256, 0, st>>>(vertices, int(nv), scratch, mask);
  if ((e = cudaPeekAtLastError()) != cudaSuccess)
    return edp::record_cuda_failure(e, EDP_NOALLOC_SITE);
  k_noalloc_resolve<<<blocks, 256, 0, st>>>(int(nv), scratch, canonical);
  if ((e = cudaPeekAtLastError()) != cudaSuccess)
    return edp::record_cuda_failure(e, EDP_NOALLOC_SITE);
  return EDP_OK;
}
