"""harm_utoprim_2d_batch_noalloc against harm_utoprim_2d_batch, through the C ABI.

The no-alloc entry point serves hosts that cannot allocate device memory in
mid-run: their GPU memory is already committed to a resident simulation
state or to another allocator, or they must not trigger cudaFree's
device-wide synchronisation while other streams work.  It keeps its device
copies in one fixed array inside the library instead.  Because that array is
shared by every call and keeps the previous call's contents, the GPU test
makes two calls in a row with different batches and checks each against the
allocating entry point on the same inputs.

This file is named to be collected last, so that a run stopping at the first
failure has run every other test before it."""
import ctypes
import os

import numpy as np
import pytest

from helpers import GOLDEN, load_fixture, problem_from_fixture

TOL = 1e-13   # relative, as for the other inversion tests
IP = ctypes.POINTER(ctypes.c_int)
DP = ctypes.POINTER(ctypes.c_double)


def _inputs():
    kat = dict(np.load(os.path.join(GOLDEN, "kat_u2p.npz")))
    pr = problem_from_fixture(load_fixture("t2d"))
    g = pr.geometry
    ij = kat["ij"]
    gcov = np.ascontiguousarray(np.stack([g["gcov"][i, j, 3].ravel() for i, j in ij]))
    gcon = np.ascontiguousarray(np.stack([g["gcon"][i, j, 3].ravel() for i, j in ij]))
    gdet = np.ascontiguousarray(np.array([g["gdet"][i, j, 3] for i, j in ij]))
    return (np.ascontiguousarray(kat["U"]), gcov, gcon, gdet, np.ascontiguousarray(kat["guess"]),
            float(kat["gam"]))


def _call(fn, U, gcov, gcon, gdet, guess, gam):
    prim = guess.copy()
    ret = np.full(U.shape[0], -12345, dtype=np.int32)
    rc = fn(U.ctypes.data_as(DP), gcov.ctypes.data_as(DP), gcon.ctypes.data_as(DP), gdet.ctypes.data_as(DP),
            prim.ctypes.data_as(DP), ret.ctypes.data_as(IP), U.shape[0], gam)
    return rc, prim, ret


def _agree(a, b):
    rc_a, prim_a, ret_a = a
    rc_b, prim_b, ret_b = b
    assert rc_a == 0 and rc_b == 0
    np.testing.assert_array_equal(ret_a, ret_b)
    ok = ret_b == 0
    assert ok.sum() > 0
    err = np.max(np.abs(prim_a[ok] - prim_b[ok]) / np.maximum(np.abs(prim_b[ok]), 1e-300))
    assert err <= TOL, err


@pytest.mark.gpu
def test_noalloc_batch_matches_allocating_batch_twice(harm_lib):
    U, gcov, gcon, gdet, guess, gam = _inputs()
    lib = harm_lib
    # first call: the whole known-answer set
    _agree(_call(lib.harm_utoprim_2d_batch_noalloc, U, gcov, gcon, gdet, guess, gam),
           _call(lib.harm_utoprim_2d_batch, U, gcov, gcon, gdet, guess, gam))
    # second call right after: a smaller batch in another order, so anything
    # left over from the first call in the shared array would show
    sel = np.ascontiguousarray(np.arange(U.shape[0])[::-3])
    args = tuple(np.ascontiguousarray(x[sel]) for x in (U, gcov, gcon, gdet, guess)) + (gam,)
    _agree(_call(lib.harm_utoprim_2d_batch_noalloc, *args), _call(lib.harm_utoprim_2d_batch, *args))


def test_noalloc_batch_rejects_oversized_batch(harm_lib):
    """Checked before any device work, so it runs without a GPU too."""
    n = 16384 + 1
    z = np.zeros(1, dtype=np.float64)
    r = np.zeros(1, dtype=np.int32)
    rc = harm_lib.harm_utoprim_2d_batch_noalloc(z.ctypes.data_as(DP), z.ctypes.data_as(DP), z.ctypes.data_as(DP),
                                                z.ctypes.data_as(DP), z.ctypes.data_as(DP), r.ctypes.data_as(IP),
                                                n, 4. / 3.)
    assert rc == -1
    assert b"HARM_U2P_NOALLOC_MAX" in harm_lib.harm_last_error()
