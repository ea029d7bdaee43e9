"""The allocation-free self-test entry point (its file name makes pytest collect it last).

Hosts that cannot allocate device memory when they want to check the sweep's division
(a fixed device-memory budget, or an application that owns every device allocation
through its own pool) call piks_selftest_division_noalloc, which uses a static device
buffer compiled into the library instead of allocating. Its result must equal the
allocating piks_selftest_division's on the same samples, call after call.

Positive control: besides the mismatches, the kernels count the samples they tested, and
the entry point returns PIKS_ERR_CUDA unless that count equals the request (it clears the
total first). A kernel that never ran, or ran on part of the samples, therefore fails the
status assertions below instead of reading as zero mismatches; the ragged sample counts
check that the count is exact for partly filled blocks.
"""
import ctypes

import pytest

import piks3d_b200 as pk

pytestmark = pytest.mark.gpu

MAX_SAMPLES = 16_777_216
PER_BLOCK = 256 * 64


def _bind():
    lib = pk.load_library()
    for name in ("piks_selftest_division", "piks_selftest_division_noalloc"):
        fn = getattr(lib, name)
        fn.argtypes = [ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int64)]
        fn.restype = ctypes.c_int
    return lib


def _run(fn, samples, seed):
    out = ctypes.c_int64(-1)
    status = fn(0, samples, seed, ctypes.byref(out))
    return status, out.value


def test_noalloc_matches_allocating_entry_point_twice():
    lib = _bind()
    for seed in (2024, 99991):  # two calls in a row on the shared static scratch
        st_a, bad_a = _run(lib.piks_selftest_division, MAX_SAMPLES, seed)
        st_b, bad_b = _run(lib.piks_selftest_division_noalloc, MAX_SAMPLES, seed)
        assert st_a == 0 and st_b == 0, lib.piks_last_error()
        assert bad_b == bad_a == 0


def test_noalloc_counts_every_sample_of_ragged_requests():
    lib = _bind()
    # one sample, one past a block, a partial last block: the completion count must equal
    # the request exactly or the call fails
    for samples in (1, PER_BLOCK + 1, 3 * PER_BLOCK - 5):
        st_a, bad_a = _run(lib.piks_selftest_division, samples, 11)
        st_b, bad_b = _run(lib.piks_selftest_division_noalloc, samples, 11)
        assert st_b == 0, lib.piks_last_error()
        assert st_a == 0 and bad_b == bad_a


def test_noalloc_rejects_more_samples_than_its_scratch_holds():
    lib = _bind()
    st, _ = _run(lib.piks_selftest_division_noalloc, MAX_SAMPLES + 1, 7)
    assert st == 1  # PIKS_ERR_ARG
    assert b"16777216" in lib.piks_last_error()
