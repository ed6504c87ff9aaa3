"""Oracle restatement of the block selected inverse.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

``Block_factorization!`` (src/selected_inverse.jl:9-55): block LU without
inter-block pivoting; the diagonal getrf pivots are discarded
(backend_cpu.jl:255-265).  ``Block_inverse!`` (selected_inverse.jl:139-206):
Takahashi-style selected inverse on the factored pattern, with at most two
upper neighbours per block row (the two ``Uij``/``Lji`` buffers, :146-152).

Blocks are a dict {(i, j): array} (the reference's ``Matrix{Block}`` with
unassigned entries absent); arithmetic is complex128.
"""

import numpy as np

from .backend_cpu import be_getrf, be_trsm, be_gemm, be_getri, lu_nopivot


def block_factorization(A_in, npl, nopivot=False):
    """``nopivot``: factor the diagonal blocks by lu(NoPivot()) (the
    factorisation selected_inverse.jl:17 names) instead of be_getrf!."""
    A = {k: np.array(v, dtype=np.complex128) for k, v in A_in.items()}
    for i in range(npl):
        A[(i, i)] = lu_nopivot(A[(i, i)]) if nopivot else be_getrf(A[(i, i)])     # :18
        for j in range(i + 1, npl):
            if (j, i) in A:
                A[(j, i)] = be_trsm("R", "U", "N", "N", 1.0, A[(i, i)], A[(j, i)])  # :23
            if (i, j) in A:
                A[(i, j)] = be_trsm("L", "L", "N", "U", 1.0, A[(i, i)], A[(i, j)])  # :27
        for k in range(i + 1, npl):                                               # :32
            if (i, k) in A:
                A[(k, k)] = be_gemm("N", "N", -1.0, A[(k, i)], A[(i, k)], 1.0, A[(k, k)])   # :34
                for l in range(k + 1, npl):
                    if (i, l) in A:
                        if (k, l) in A:
                            A[(k, l)] = be_gemm("N", "N", -1.0, A[(k, i)], A[(i, l)], 1.0, A[(k, l)])  # :39
                            A[(l, k)] = be_gemm("N", "N", -1.0, A[(l, i)], A[(i, k)], 1.0, A[(l, k)])  # :40
                        else:
                            A[(k, l)] = be_gemm("N", "N", -1.0, A[(k, i)], A[(i, l)], 0.0, None)     # :43,45
                            A[(l, k)] = be_gemm("N", "N", -1.0, A[(l, i)], A[(i, k)], 0.0, None)     # :44,46
    return A


def block_inverse(A_in, npl):
    A = {k: np.array(v, dtype=np.complex128) for k, v in A_in.items()}
    b0 = A[(0, 0)].shape
    U = [np.zeros(b0, dtype=np.complex128) for _ in range(2)]                    # :146-152
    Lb = [np.zeros(b0, dtype=np.complex128) for _ in range(2)]
    vidx = [0, 0]
    A[(npl - 1, npl - 1)] = be_getri(A[(npl - 1, npl - 1)])                      # :158
    for i in range(npl - 2, -1, -1):                                              # :160
        vid = 0
        Aii = np.zeros(b0, dtype=np.complex128)
        for j in range(i + 1, npl):
            if (i, j) in A:
                for k in range(i + 1, npl):
                    if (i, k) in A and (k, j) in A:
                        U[vid] = be_gemm("N", "N", 1.0, A[(i, k)], A[(k, j)], 1.0, U[vid])    # :165
                        vidx[vid] = j
                        Lb[vid] = be_gemm("N", "N", 1.0, A[(j, k)], A[(k, i)], 1.0, Lb[vid])  # :167
                U[vid] = be_trsm("L", "U", "N", "N", -1.0, A[(i, i)], U[vid])                 # :172
                Lb[vid] = be_trsm("R", "L", "N", "U", -1.0, A[(i, i)], Lb[vid])               # :174
                vid += 1
        for vj in range(vid):                                                      # :180
            j = vidx[vj]
            if (j, i) in A:
                Aii = be_gemm("N", "N", 1.0, U[vj], A[(j, i)], 1.0, Aii)                      # :183
                A[(j, i)] = Lb[vj].copy()                                                     # :185
                A[(i, j)] = U[vj].copy()                                                      # :187
                U[vj] = np.zeros(b0, dtype=np.complex128)                                     # :188
                Lb[vj] = np.zeros(b0, dtype=np.complex128)                                    # :189
        Aii = be_trsm("R", "L", "N", "U", 1.0, A[(i, i)], Aii)                                # :195
        A[(i, i)] = be_getri(A[(i, i)])                                                       # :197
        A[(i, i)] = A[(i, i)] - Aii                                                           # :199
    return A
