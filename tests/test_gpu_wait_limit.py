"""The bounded waits of the INT8 tensor-core product kernel run out cleanly.

Every mbarrier wait of ozaki_mma_kernel (stage copies, tensor-core
completion, accumulator drains) is bounded.  With the limit set to about
100 ns (negf_set_tensor_wait_limit) the pipeline waits of a mixed-precision
product expire: the kernel raises its abort flag, waits (with the default
limit) for its own copies and tensor-core operations in flight, releases its
tensor memory and returns, and the call reports NEGF_ERR_TIMEOUT.  No trap,
no fault: with the default limit restored, the same call on the same context
succeeds and matches the FP64 product (bar 1e-12 relative to |A| |B|).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rand(rng, m, n):
    return rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))


def test_product_wait_limit_runs_out_and_context_stays_usable(negf):
    from libnegf_b200._lib import NEGF_ERR_TIMEOUT, NegfError
    lib = negf.load()
    rng = np.random.default_rng(9)
    A, B = _rand(rng, 512, 512), _rand(rng, 512, 512)
    dA, dB = negf.to_device(A), negf.to_device(B)
    try:
        assert lib.negf_set_tensor_wait_limit(1e-7) == 0
        dC = negf.dzeros(512, 512)
        with pytest.raises(NegfError) as exc:
            negf.be_gemm_batched_("N", "N", [(1.0, dA, dB, 0.0, dC)], precision="mixed")
        assert exc.value.code == NEGF_ERR_TIMEOUT
        assert b"timed out" in lib.negf_last_error()
    finally:
        assert lib.negf_set_tensor_wait_limit(0.0) == 0
    for _ in range(2):
        dC = negf.dzeros(512, 512)
        negf.be_gemm_batched_("N", "N", [(1.0, dA, dB, 0.0, dC)], precision="mixed")
        AB = A @ B
        assert np.linalg.norm(negf.to_host(dC) - AB) / np.linalg.norm(AB) < 1e-12
