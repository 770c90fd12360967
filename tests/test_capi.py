"""The C ABI library loads on the CPU and exports every entry point that
include/edp.h declares (no compute calls: there may be no GPU)."""

import re

from conftest import ROOT


def declared():
    text = (ROOT / "include/edp.h").read_text()
    return sorted(set(re.findall(r"\b(edp_[a-z_]+)\s*\(", text)))


def test_header_declares_the_reference_surface():
    names = declared()
    for required in ("edp_event_create", "edp_device_create", "edp_warmup", "edp_enqueue",
                     "edp_capture", "edp_run", "edp_read_status", "edp_get_outputs",
                     "edp_destroy"):
        assert required in names


def test_library_exports_every_declared_symbol():
    import ctypes

    from peel_b200 import _lib

    lib = _lib.load()
    for name in declared():
        assert hasattr(lib, name), name
    assert set(declared()) <= set(_lib.EXPORTS)
    assert lib.edp_abi_version() >= 1
    assert lib.edp_status_string(1) == b"invalid argument"



def header_constant(name):
    text = (ROOT / "include/edp.h").read_text()
    return int(re.search(rf"\b{name}\s*=\s*(\d+)", text).group(1))


def test_header_constants_match_the_host():
    """The counter array and ABI version the header states are the ones the
    Python host reads and the library reports."""
    from peel_b200 import _lib
    from peel_b200.events import METRIC_NAMES
    from peel_b200.solver import METRIC_COUNT

    assert header_constant("EDP_METRICS") == METRIC_COUNT == len(METRIC_NAMES)
    assert header_constant("EDP_STATUS_SLOTS") == 16
    assert header_constant("EDP_ABI_VERSION") == _lib.ABI_VERSION == _lib.load().edp_abi_version()


def test_default_capacities_match_reference():
    import ctypes

    from peel_b200 import Capacities, EventCapacities, _lib

    lib = _lib.load()
    c = _lib.EventCapacitiesC()
    lib.edp_event_default_capacities(1000, ctypes.byref(c))
    ref = EventCapacities.for_mesh(1000)
    assert [getattr(c, f) for f, _ in c._fields_] == [getattr(ref, f) for f, _ in c._fields_]
    d = _lib.DeviceCapacitiesC()
    lib.edp_device_default_capacities(20000, ctypes.byref(d))
    ref = Capacities.for_mesh(20000)
    assert [getattr(d, f) for f, _ in d._fields_] == [getattr(ref, f) for f, _ in d._fields_]


def test_create_rejects_bad_arguments_without_touching_the_device():
    import ctypes

    from peel_b200 import _lib

    lib = _lib.load()
    out = ctypes.c_void_p()
    # Null output pointer, negative sizes: argument errors before any CUDA call.
    assert lib.edp_event_create(None, -1, None, 0, None, None, None, None, None,
                                ctypes.byref(out)) == 1
    assert not out.value


def test_host_inputs_are_validated():
    import pytest
    import torch

    from peel_b200 import EventPeeler

    with pytest.raises(ValueError):
        EventPeeler(torch.zeros((3, 3), dtype=torch.float64), torch.zeros((1, 3), dtype=torch.int32),
                    torch.eye(4, dtype=torch.float64), torch.zeros(6, dtype=torch.float64))


def test_stage_names_match_the_header():
    """The Python stage names follow enum edp_stage, one per value."""
    from peel_b200 import _lib

    text = (ROOT / "include/edp.h").read_text()
    body = text[text.index("enum edp_stage {"):text.index("EDP_STAGE_COUNT\n")]
    names = re.findall(r"EDP_STAGE_([A-Z_]+)", body)
    assert [n.lower() for n in names] == list(_lib.STAGE_NAMES)
