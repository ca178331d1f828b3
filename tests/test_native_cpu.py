"""The C-ABI library builds for sm_100a, loads without a GPU, exports every
entry point its header declares, and rejects bad arguments with status codes
(host-side checks only; no kernel is launched here)."""
import ctypes as C
import os
import re

import pytest

import demso_b200 as D
from demso_b200 import _lib, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
           if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(dem_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_binding_covers_header():
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_abi_version_and_struct_sizes():
    lib = _lib.load()
    assert lib.dem_abi_version() == 2
    # DemSystem: 4 + 8 + 8 + 4 + 8 + 4 + 4 + 4 bytes + DEM_MAX_MATERIALS * 24
    assert C.sizeof(_lib.DemSystem) == 44 + _lib.DEM_MAX_MATERIALS * 24
    assert C.sizeof(_lib.DemMaterial) == 24
    assert C.sizeof(_lib.DemStateSet) == 8 * 8  # eight pointers
    assert _lib.STATE_PAD == 8


def _sys(**kw):
    s = scenes.settling_pile(side=8, box=0.02).sys
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def test_validate_system():
    lib = _lib.load()
    assert lib.dem_validate_system(_sys().to_c()) == 0
    assert lib.dem_validate_system(_sys(gx=24).to_c()) == 1
    assert b"power" in lib.dem_last_error_string()
    assert lib.dem_validate_system(_sys(gy=0).to_c()) == 1
    s = _sys().to_c()
    s.numMaterials = 0
    assert lib.dem_validate_system(s) == 1
    s.numMaterials = _lib.DEM_MAX_MATERIALS + 1
    assert lib.dem_validate_system(s) == 1
    s = _sys().to_c()
    s.cubeDimension[0] = 0.0
    assert lib.dem_validate_system(s) == 1


def test_sort_scratch_sizes():
    lib = _lib.load()
    for n in (1, 1000, 4096, 1 << 20):
        for bits in (0, 1, 10, 20, 32):
            b = lib.dem_sort_scratch_bytes(n, bits)
            assert b >= 8 * n
    assert lib.dem_sort_scratch_bytes(1 << 22, 20) > lib.dem_sort_scratch_bytes(1 << 20, 20)


def test_bad_arguments_are_status_codes_not_crashes():
    lib = _lib.load()
    s = _sys().to_c()
    # NULL buffers with n > 0 are rejected before any CUDA call
    assert lib.dem_calc_hash(s, None, None, None, 10, None) == 1
    assert lib.dem_sort_particles(None, None, 10, 20, None, 0, None) == 1
    assert lib.dem_sort_particles(None, None, 10, 33, None, 0, None) == 1
    assert lib.dem_collide(s, None, None, None, None, None, None, None, None, None, None, 10,
                           64, None, None) == 1
    assert lib.dem_collide(s, None, None, None, None, None, None, None, None, None, None, 10,
                           63, None, None) == 1  # numCells mismatch
    assert lib.dem_integrate_system(s, None, None, None, None, None, None, None, None, None,
                                    None, 10, None) == 1
    h = C.c_void_p()
    assert lib.dem_create(None, 10, 0, C.byref(h)) == 1
    assert lib.dem_create(s, 0, 0, C.byref(h)) == 1
    assert lib.dem_step(None, 1, None) == 1
    ids = (C.c_uint32 * 2)(0, 1)
    rows = (C.c_float * 24)()
    assert lib.dem_step_followed(None, 1, ids, 2, rows, None) == 1
    assert lib.dem_get_followed(None, ids, 2, rows, None) == 1
    assert lib.dem_get_followed_async(None, ids, 2, rows, None) == 1
    assert lib.dem_adj_forward(None, 10, 5, None) == 1
    assert lib.dem_adj_backward(None, None, None, None, None, None) == 1
    assert lib.dem_adopt_state(None, 10, None, None, None) == 1
    assert lib.dem_state_view(None, None, None) == 1
    assert lib.dem_destroy(None) == 0
    # n = 0 is a no-op
    assert lib.dem_calc_hash(s, None, None, None, 0, None) == 0


def test_row_windows_check_their_rows():
    """dem_create_rows refuses a bad block of rows before any CUDA call."""
    lib = _lib.load()
    sys_ = _sys()
    s = sys_.to_c()
    gy = sys_.gy
    h = C.c_void_p()
    assert gy >= 4 and gy & (gy - 1) == 0
    assert lib.dem_create_rows(s, 10, 0, 0, 3, C.byref(h)) == 1       # not a power of two
    assert lib.dem_create_rows(s, 10, 0, 0, 0, C.byref(h)) == 1
    assert lib.dem_create_rows(s, 10, 0, 0, 2 * gy, C.byref(h)) == 1  # more rows than the grid
    assert lib.dem_create_rows(s, 10, 0, gy, 2, C.byref(h)) == 1      # first row outside it
    assert lib.dem_create_rows(s, 0, 0, 0, 2, C.byref(h)) == 1        # no capacity
    assert lib.dem_create_rows(None, 10, 0, 0, 2, C.byref(h)) == 1
    assert lib.dem_create_rows(s, 10, 0, 0, 2, None) == 1
    assert lib.dem_row_slots(None, 0, 1, None, None, None) == 1
    assert not h.value


def test_python_errors_raise():
    with pytest.raises(D.DemError):
        _lib.check(1)


def test_batch_create_rejects_bad_specimens():
    import ctypes as C
    lib = _lib.load()
    arr = (_lib.DemSystem * 2)()
    arr[0] = _sys().to_c(10)
    arr[1] = _sys(gx=12).to_c(10)
    h = C.c_void_p()
    assert lib.dem_batch_create(arr, 2, 0, C.byref(h)) == 1
    assert lib.dem_batch_create(None, 0, 0, C.byref(h)) == 1
    assert lib.dem_batch_specimen(None, 0, None, None) == 1


def test_test_hooks_check_their_arguments():
    lib = _lib.load()
    assert lib.dem_debug_fail_allocation(-1) == 1
    assert lib.dem_debug_fail_allocation(0) == 0
    assert lib.dem_debug_live_allocations() == 0
    assert lib.dem_debug_sort_hold(None, 0, 10) == 1
