"""CPU oracle for the block-tridiagonal NEGF hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product path (the CUDA library, the
host API in ``libnegf.jl_b200``) imports or calls this package.  It is used by
``tests/``, by ``__graft_entry__.smoke()`` as the checker and by ``bench.py``'s
``cpu_baseline`` leg / ``--impl reference`` arm as the timed CPU baseline.

It restates, in numpy + scipy LAPACK/BLAS, the exact call sequence that
LibNEGF.jl's CPU backend executes (``src/backend_cpu.jl``: zgetrf / zgetrs /
zgemm / zgetri / ztrsm on dense column-major blocks).  Each function cites the
reference file:line it follows.

Pinning: the reference is Julia and no Julia toolchain exists in this image, so
no output of the reference itself can be produced here, and the reference ships
no golden vectors.  The oracle is pinned instead against the reference's own
test oracles -- a dense inverse (``test_matinvertndiag_general_rgf.jl``,
``test_keldyshndiag.jl:80-95``) and sequential RGF
(``test_matinvertndiag_ddrgf.jl:245-293``) -- at the reference's tolerances,
and through committed fixtures under ``tests/golden/`` made by
``tests/golden/make_golden.py``.  Parity with the reference itself is therefore
"unpinned" in the strict sense.

Two modules are not restatements of the reference: ``ddtruth`` (a
double-double truth for the parity tests) and ``ozaki`` (a host model of the
library's mixed-precision digit products, which the reference does not have,
used to check their accuracy claims against that truth).
"""

from .blockmatrix import BlockMatrix, bm_convert_dense, bm_from_dense, bm_copy  # noqa: F401
from . import backend_cpu, generators, rgf, general_rgf, keldysh, selected_inverse, ddrgf, physics, direct  # noqa: F401
