"""The allocation-free inversion entry point.

negf_zinv_batched_noalloc serves callers that cannot let the library call
cudaMalloc / cudaFree (all device memory owned by the caller's own pool, or
loops that cannot take cudaFree's device-wide synchronisation).  Its scratch is
a fixed 64 MiB __device__ array shared by every call.  This test checks it
through the C ABI against the allocating negf_zinv_batched, on two calls in a
row (so the second call starts from the first call's leftover scratch), and
that an oversized request is refused.  It must pass alone in a fresh process
and after the rest of the suite; this file sorts last so that a run stopping
at the first failure has run every other test before it.
"""

import ctypes

import numpy as np
import pytest

from conftest import rel_fro

pytestmark = pytest.mark.gpu

# the tolerance of the inversion tests (test_gpu_core.py::test_zinv_batched)
TOL = 1e-12


def _inv_both(negf, mats):
    from libnegf_b200._lib import int_array, ptr_array, check
    lib = negf.load()
    n = [m.shape[0] for m in mats]
    dA = [negf.to_device(m) for m in mats]
    out_ref = [negf.dzeros(k, k) for k in n]
    out_na = [negf.dzeros(k, k) for k in n]
    info = (ctypes.c_int32 * len(mats))()
    args = (len(mats), int_array(n), ptr_array([a.data_ptr() for a in dA]), int_array(n))
    check(lib.negf_zinv_batched(*args, ptr_array([o.data_ptr() for o in out_ref]), int_array(n), info, None))
    check(lib.negf_zinv_batched_noalloc(*args, ptr_array([o.data_ptr() for o in out_na]), int_array(n), info, None))
    assert list(info) == [0] * len(mats)
    for a, da in zip(mats, dA):
        assert np.array_equal(negf.to_host(da), a)  # inputs untouched
    return [negf.to_host(o) for o in out_ref], [negf.to_host(o) for o in out_na]


@pytest.mark.parametrize("sizes", [[64, 17, 100], [256, 130, 300, 5]])
def test_noalloc_matches_allocating_entry_point_twice(negf, sizes):
    rng = np.random.default_rng(sum(sizes))
    for call in range(2):  # the second call reuses the scratch the first one left behind
        mats = [rng.standard_normal((k, k)) + 1j * rng.standard_normal((k, k)) for k in sizes]
        ref, na = _inv_both(negf, mats)
        for a, r, x in zip(mats, ref, na):
            assert rel_fro(x, r) < TOL
            assert rel_fro(x, np.linalg.inv(a)) < TOL * max(1.0, np.linalg.cond(a) / 1e2)


@pytest.mark.parametrize("b,limit", [(256, 51), (512, 15)])
def test_noalloc_documented_limit(negf, b, limit):
    """The header's limit: `limit` blocks of size b run and match the allocating
    entry point; one block more is refused."""
    from libnegf_b200._lib import int_array, ptr_array, check, NEGF_ERR_INVALID
    lib = negf.load()
    rng = np.random.default_rng(b)
    base = [rng.standard_normal((b, b)) + 1j * rng.standard_normal((b, b)) + 4.0 * np.sqrt(b) * np.eye(b)
            for _ in range(3)]
    mats = [base[i % 3] for i in range(limit)]
    ref, na = _inv_both(negf, mats)
    for r, x in zip(ref, na):
        assert rel_fro(x, r) < TOL
    n = [b] * (limit + 1)
    dA = negf.to_device(base[0])
    dO = [negf.dzeros(b, b) for _ in n]
    rc = lib.negf_zinv_batched_noalloc(len(n), int_array(n), ptr_array([dA.data_ptr()] * len(n)), int_array(n),
                                       ptr_array([o.data_ptr() for o in dO]), int_array(n), None, None)
    assert rc == NEGF_ERR_INVALID
    assert b"scratch" in lib.negf_last_error()


def test_noalloc_rejects_oversized_request(negf):
    from libnegf_b200._lib import int_array, ptr_array, NEGF_ERR_INVALID
    lib = negf.load()
    n = [1024] * 20  # 20 blocks of 1024 need far more than the fixed scratch
    a = negf.dzeros(8, 8)
    rc = lib.negf_zinv_batched_noalloc(len(n), int_array(n), ptr_array([a.data_ptr()] * len(n)), int_array(n),
                                       ptr_array([a.data_ptr()] * len(n)), int_array(n), None, None)
    assert rc == NEGF_ERR_INVALID
    assert b"scratch" in lib.negf_last_error()
