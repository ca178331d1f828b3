"""dem_sort_particles_static: the sort for callers that cannot allocate.

Callers whose step loop must not stall on the device-wide synchronisation of
an allocation, or whose own memory manager owns all device memory, cannot
hand the sort scratch memory; this entry point uses a fixed array inside the
library instead.  The
test calls it through the C ABI and checks that it gives exactly the result
of dem_sort_particles (caller scratch) -- the sort is integer work, so the
tolerance is zero -- on two calls in a row that share the fixed array, and
that oversized calls are refused before anything runs on the GPU.

Kept in a file of its own that pytest collects last.
"""
import numpy as np
import pytest

from helpers import dev, host

pytestmark = pytest.mark.gpu

MAX_PAIRS = 262144


def _sort_with_scratch(keys, vals, bits):
    import torch
    import demso_b200 as D
    k, v = dev(keys), dev(vals)
    need = D.sort_scratch_bytes(keys.size, bits)
    scratch = torch.empty(max(need, 1), dtype=torch.uint8, device="cuda")
    D.check(D.load().dem_sort_particles(k.data_ptr(), v.data_ptr(), keys.size, bits,
                                        scratch.data_ptr(), scratch.numel(), D._stream()))
    torch.cuda.synchronize()
    return host(k), host(v)


def _sort_static(keys, vals, bits):
    import torch
    import demso_b200 as D
    k, v = dev(keys), dev(vals)
    D.check(D.load().dem_sort_particles_static(k.data_ptr(), v.data_ptr(), keys.size, bits,
                                               D._stream()))
    torch.cuda.synchronize()
    return host(k), host(v)


def test_static_sort_matches_scratch_sort_on_two_calls_in_a_row():
    rng = np.random.default_rng(2024)
    cases = [(MAX_PAIRS, 20), (100003, 32)]
    for n, bits in cases:
        hi = (1 << bits) if bits < 32 else (1 << 32)
        keys = rng.integers(0, hi, size=n, dtype=np.uint64).astype(np.uint32)
        vals = rng.permutation(n).astype(np.uint32)
        k_ref, v_ref = _sort_with_scratch(keys, vals, bits)
        k_st, v_st = _sort_static(keys, vals, bits)
        assert np.array_equal(k_st, k_ref)
        assert np.array_equal(v_st, v_ref)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(k_st, keys[order]) and np.array_equal(v_st, vals[order])


def test_static_sort_rejects_sizes_beyond_its_scratch():
    import demso_b200 as D
    lib = D.load()
    # refused on the host before any launch: the pointers are never touched
    assert lib.dem_sort_particles_static(None, None, MAX_PAIRS + 1, 20, None) == 6
    assert b"exceed" in lib.dem_last_error_string()
    assert lib.dem_sort_particles_static(None, None, 10, 33, None) == 1
