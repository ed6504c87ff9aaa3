"""Oracle restatement of the retarded RGF sweep.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows ``bndiag_of_inv_rgf_local!`` (src/matinvertndiag_rgf.jl:114-200) call
by call.  Names: ``lu[i]`` is the LU of the right-connected Schur complement
X_i held in the diagonal of ``buffM1``; ``R[i]`` = buffM1[i, i+1] =
M[i,i+1] X_{i+1}^{-1}; ``L[i+1]`` = buffM1[i+1, i] = X_{i+1}^{-1} M[i+1,i].
"""

import numpy as np

from .backend_cpu import be_lu, be_mldivide, be_gemm, be_ctranspose, be_identity
from .blockmatrix import BlockMatrix


def rgf_upward(M):
    """Upward pass (matinvertndiag_rgf.jl:143-162; the same as
    keldyshndiag.jl:191-219).  Returns (lu, R, L)."""
    npl = M.npl
    lu = [None] * npl
    R = [None] * npl
    L = [None] * npl
    lu[npl - 1] = be_lu(M.M[(npl - 1, npl - 1)])                       # rgf.jl:144
    for ix in range(npl - 2, -1, -1):                                   # rgf.jl:147
        t = be_ctranspose(M.M[(ix, ix + 1)])                            # rgf.jl:152
        y = be_mldivide("C", t, lu[ix + 1])                             # rgf.jl:153
        R[ix] = be_ctranspose(y)                                        # rgf.jl:154
        L[ix + 1] = be_mldivide("N", M.M[(ix + 1, ix)], lu[ix + 1])     # rgf.jl:157
        X = M.M[(ix, ix)].copy()                                        # rgf.jl:159
        X = be_gemm("N", "N", -1.0, M.M[(ix, ix + 1)], L[ix + 1], 1.0, X)  # rgf.jl:160
        lu[ix] = be_lu(X)                                               # rgf.jl:161
    return lu, R, L


def bndiag_of_inv_rgf_local(M, build_full_inv=False, upward=None):
    """Block tridiagonal of M^{-1} (matinvertndiag_rgf.jl:114-200).

    Returns a BlockMatrix with blocks (i,i), (i,i+1), (i+1,i); with
    ``build_full_inv`` every block of the inverse (rgf.jl:185-199).
    ``upward`` reuses a precomputed (lu, R, L) of ``rgf_upward``."""
    npl = M.npl
    lu, R, L = upward if upward is not None else rgf_upward(M)
    out = BlockMatrix(M.blockSizes, {"in": 3, "out": 3}, False)
    G = out.M
    G[(0, 0)] = be_mldivide("N", be_identity(M.blockSizes[0]), lu[0])   # rgf.jl:169
    for ix in range(1, npl):                                            # rgf.jl:172
        G[(ix - 1, ix)] = be_gemm("N", "N", -1.0, G[(ix - 1, ix - 1)], R[ix - 1], 0.0, None)   # :174
        G[(ix, ix - 1)] = be_gemm("N", "N", -1.0, L[ix], G[(ix - 1, ix - 1)], 0.0, None)       # :177
        d = be_mldivide("N", be_identity(M.blockSizes[ix]), lu[ix])                           # :180
        G[(ix, ix)] = be_gemm("N", "N", -1.0, L[ix], G[(ix - 1, ix)], 1.0, d)                 # :181
    if build_full_inv and npl > 2:                                      # rgf.jl:185-199
        # buffM1.M[ix+kx, jx] with ix+kx == jx-1 is R_{jx-1}; buffM1.M[jx, ix+kx] is L_jx
        out.ndiag = {"in": 3, "out": 2 * npl - 1}
        for ix in range(npl):
            for jx in range(ix + 2, npl):
                G[(ix, jx)] = be_gemm("N", "N", -1.0, G[(ix, jx - 1)], R[jx - 1], 0.0, None)   # :190
                G[(jx, ix)] = be_gemm("N", "N", -1.0, L[jx], G[(jx - 1, ix)], 0.0, None)       # :192
    return out
