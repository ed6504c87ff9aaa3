"""Device-resident ``BlockMatrix`` / ``Block`` and the ``be_*`` backend layer.

Mirror of LibNEGF.jl's data types and backend API for the B200 library:

* ``BlockMatrix`` -- src/blockmatrix.jl:10-17: block sizes, the banded block
  table ``M`` (dict keyed by 0-based (i, j); only the band is assigned; a
  Hermitian matrix stores the diagonal and upper blocks), ``ndiag`` and the
  ``isArrayOrLU`` / ``isHermitian`` flags.
* ``Block`` -- src/block.jl:9-34: a dense block used by the selected inverse.
* ``be_*`` -- src/backend_cpu.jl:26-289 re-targeted at device memory: every
  block is a complex128 CUDA tensor stored column-major (a transposed view of
  a row-major allocation), exactly the layout of a Julia Matrix{ComplexF64};
  the arithmetic runs in libnegf_b200.so.  ``DeviceLU`` stands in for
  ``CpuLU`` (backend_cpu.jl:7-10): it holds the explicit inverse of the
  factored block, which is how the CUDA library applies ``be_mldivide!``.

Indices are 0-based (Julia's are 1-based).  PyTorch provides device memory and
the current stream only; no torch arithmetic runs on the product path.
"""

import ctypes

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib
from ._lib import check, ptr_array, int_array, load

DTYPE = torch.complex128


def _dev():
    if not torch.cuda.is_available():
        raise RuntimeError("libnegf_b200 needs a CUDA device (there is no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def stream_handle():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def dzeros(m, n):
    """Column-major complex128 zero block on the current device."""
    return torch.zeros((n, m), dtype=DTYPE, device=_dev()).t()


def dempty(m, n):
    return torch.empty((n, m), dtype=DTYPE, device=_dev()).t()


def to_device(a):
    """Host array (m x n) -> column-major device block."""
    a = np.asarray(a, dtype=np.complex128)
    t = torch.from_numpy(np.ascontiguousarray(a.T)).to(_dev())
    return t.t()


def to_host(t):
    return t.detach().cpu().numpy()


def ld(t):
    """Leading dimension of a column-major block."""
    if t.dim() != 2 or t.stride(0) != 1:
        raise ValueError("blocks must be column-major 2-D tensors")
    return max(1, t.stride(1))


def dptr(t):
    return t.data_ptr()


class DeviceLU:
    """``CpuLU`` stand-in: the factored block's inverse (used by be_mldivide!)."""

    def __init__(self, n):
        self.inv = dzeros(n, n)
        self.n = n


class BlockMatrix:
    """src/blockmatrix.jl:10-17."""

    def __init__(self, blockSizes, M=None, ndiag=None, isArrayOrLU=False, isHermitian=False):
        self.blockSizes = [int(b) for b in blockSizes]
        self.M = {} if M is None else M
        self.ndiag = dict(ndiag or {"in": 3, "out": 3})
        self.isArrayOrLU = bool(isArrayOrLU)
        self.isHermitian = bool(isHermitian)

    @property
    def npl(self):
        return len(self.blockSizes)

    def band(self, key="out"):
        return (self.ndiag[key] - 1) // 2

    def offsets(self):
        return np.concatenate([[0], np.cumsum(self.blockSizes)]).astype(int)

    def pattern(self, key="out"):
        """Assigned (i, j) pairs (blockmatrix.jl:44-69 visiting order)."""
        w = self.band(key)
        out = []
        for i in range(self.npl):
            if not self.isHermitian:
                for j in range(i - 1, max(0, i - w) - 1, -1):
                    out.append((i, j))
            out.append((i, i))
            for j in range(i + 1, min(self.npl, i + w + 1)):
                out.append((i, j))
        return out


# --------------------------------------------------------------------------
# backend primitives (src/backend_cpu.jl)

def be_copy_to_hw(a):
    """backend_cpu.jl:30-32."""
    return to_device(a)


def be_copy_from_hw(t):
    """backend_cpu.jl:38-40."""
    return to_host(t)


def be_copy_in_hw_(out, inp):
    """backend_cpu.jl:42-44."""
    out.copy_(inp)


def be_copy_in_hw(t):
    c = dempty(t.shape[0], t.shape[1])
    c.copy_(t)
    return c


def be_zero_array(dims):
    """backend_cpu.jl:50-52."""
    return dzeros(dims[0], dims[1])


def be_identity(n):
    """backend_cpu.jl:54-56."""
    t = dzeros(n, n)
    t.diagonal().fill_(1.0)
    return t


def be_fill_(t, x):
    """backend_cpu.jl:86-88."""
    t.fill_(complex(x))


def be_random_array(dims, rng=None):
    """backend_cpu.jl:82-84 (uniform [0,1) real and imaginary parts)."""
    rng = rng or np.random.default_rng()
    return to_device(rng.random(dims) + 1j * rng.random(dims))


def _gemm_problem(tA, tB, alpha, A, B, beta, C):
    m = C.shape[0]
    n = C.shape[1]
    k = A.shape[1] if tA == "N" else A.shape[0]
    p = _lib.ZGemmProblem()
    p.A, p.B, p.C = dptr(A), dptr(B), dptr(C)
    p.Cin = dptr(C) if beta != 0 else None
    p.m, p.n, p.k = m, n, k
    p.lda, p.ldb, p.ldc, p.ldcin = ld(A), ld(B), ld(C), ld(C)
    a, b = complex(alpha), complex(beta)
    p.alpha[0], p.alpha[1] = a.real, a.imag
    p.beta[0], p.beta[1] = b.real, b.imag
    p.diag[0] = p.diag[1] = 0.0
    return p


def be_gemm_(tA, tB, alpha, A, B, beta, C, td=None, cd=None):
    """be_gemm! (backend_cpu.jl:208-219): C = alpha op(A) op(B) + beta C."""
    p = _gemm_problem(tA, tB, alpha, A, B, beta, C)
    arr = (_lib.ZGemmProblem * 1)(p)
    check(load().negf_zgemm_batched(tA.encode(), tB.encode(), 1, arr, stream_handle()))


def be_gemm_batched_(tA, tB, items, precision="fp64"):
    """Many be_gemm! calls with the same ops in one launch: items are tuples
    (alpha, A, B, beta, C).  precision "mixed" runs the products on the INT8
    tensor cores with FP64-accurate digit splitting."""
    if not items:
        return
    arr = (_lib.ZGemmProblem * len(items))(*[_gemm_problem(tA, tB, *it) for it in items])
    fn = load().negf_zgemm_batched_mixed if precision == "mixed" else load().negf_zgemm_batched
    check(fn(tA.encode(), tB.encode(), len(items), arr, stream_handle()))


def be_ctranspose_(out, inp, td=None, cd=None):
    """be_ctranspose! (backend_cpu.jl:58-68): out = inp^H."""
    check(load().negf_zcopy_batched(b"C", 1, int_array([out.shape[0]]), int_array([out.shape[1]]),
                                    ptr_array([dptr(inp)]), int_array([ld(inp)]), ptr_array([dptr(out)]),
                                    int_array([ld(out)]), stream_handle()))


def be_ctranspose(inp, td=None, cd=None):
    out = dempty(inp.shape[1], inp.shape[0])
    be_ctranspose_(out, inp)
    return out


def be_lu_(Mout, Min, td=None, cd=None):
    """be_lu! (backend_cpu.jl:147-169): factor Min into the DeviceLU Mout.

    The library keeps the factored block as its inverse; a zero pivot raises
    SingularError (the reference prints and exits)."""
    be_inv_batched_([Min], [Mout.inv])


def be_lu(M, td=None, cd=None):
    lu = DeviceLU(M.shape[0])
    be_lu_(lu, M)
    return lu


def be_zero_lu(n):
    """backend_cpu.jl:130-136."""
    return DeviceLU(n)


def be_mldivide_(trans, Mout, Min, Mlu, td=None, cd=None):
    """be_mldivide! (backend_cpu.jl:193-206): Mout = X^{-1} Min ('N') or
    X^{-H} Min ('C') with X the factored block of Mlu."""
    tA = "N" if trans == "N" else "C"
    if trans == "T":
        tA = "T"
    be_gemm_(tA, "N", 1.0, Mlu.inv, Min, 0.0, Mout)


def be_inv_from_lu_(Mout, Min):
    """be_inv_from_lu! (backend_cpu.jl:187-190)."""
    Mout.copy_(Min.inv)


def be_inv(M):
    """be_inv (backend_cpu.jl:143-145)."""
    out = dzeros(M.shape[0], M.shape[0])
    be_inv_batched_([M], [out])
    return out


def be_inv_batched_(As, outs):
    """Batched inversion outs[i] = As[i]^{-1} (one launch)."""
    n = len(As)
    ns = int_array([a.shape[0] for a in As])
    info = (ctypes.c_int32 * max(1, n))()
    check(load().negf_zinv_batched(n, ns, ptr_array([dptr(a) for a in As]), int_array([ld(a) for a in As]),
                                   ptr_array([dptr(o) for o in outs]), int_array([ld(o) for o in outs]), info,
                                   stream_handle()))


def be_getrf_(A, td=None, cd=None):
    """be_getrf! (backend_cpu.jl:255-265): LU with partial pivoting in place,
    the pivots discarded as the reference does (its callers, the selected
    inverse, treat the factors as unpivoted).  Returns LAPACK's info (0, or
    the first zero pivot, 1-based)."""
    info = (ctypes.c_int32 * 1)()
    check(load().negf_zgetrf_batched(1, int_array([A.shape[0]]), ptr_array([dptr(A)]), int_array([ld(A)]),
                                     ptr_array([None]), info, stream_handle()))
    return int(info[0])


def be_trsm_(side, ul, tA, dA, alpha, A, B, td=None, cd=None):
    """be_trsm! (backend_cpu.jl:241-253): B = alpha op(T)^{-1} B (side 'L') or
    alpha B op(T)^{-1} (side 'R') with T the 'U' or 'L' triangle of A,
    unit ('U') or non-unit ('N') diagonal; op = 'N' (the form the selected
    inverse uses)."""
    if tA != "N":
        raise ValueError("be_trsm_: only tA = 'N' is supported (the reference's callers use 'N')")
    a = complex(alpha)
    al = (ctypes.c_double * 2)(a.real, a.imag)
    check(load().negf_ztrsm_batched(side.encode(), ul.encode(), b"N", dA.encode(), al, 1, int_array([B.shape[0]]),
                                    int_array([B.shape[1]]), ptr_array([dptr(A)]), int_array([ld(A)]),
                                    ptr_array([dptr(B)]), int_array([ld(B)]), stream_handle()))


def be_getri_(A, td=None, cd=None):
    """be_getri! (backend_cpu.jl:229-239): the inverse from L\\U factors with
    identity pivots, in place."""
    check(load().negf_zgetri_nopiv_batched(1, int_array([A.shape[0]]), ptr_array([dptr(A)]), int_array([ld(A)]),
                                           stream_handle()))


def be_mul(M1, M2):
    """be_mul (backend_cpu.jl:221-223)."""
    out = dzeros(M1.shape[0], M2.shape[1])
    be_gemm_("N", "N", 1.0, M1, M2, 0.0, out)
    return out


def be_A_from_LU(lu):
    """be_A_from_LU (backend_cpu.jl:96-128): the factored matrix itself."""
    return be_inv(lu.inv)


# --------------------------------------------------------------------------
# BlockMatrix operations (src/blockmatrix.jl)

def bm_convert(A, blockSizes=None, ndiag=None, isHermitian=False):
    """``bm_convert`` both ways (blockmatrix.jl:34-127).

    * sparse/dense host matrix + sizes -> device BlockMatrix;
    * BlockMatrix -> scipy CSC host matrix (Hermitian lower blocks are the
      conjugate transposes of the stored upper blocks)."""
    if isinstance(A, BlockMatrix):
        return sp.csc_matrix(bm_to_dense(A))
    dense = A.toarray() if sp.issparse(A) else np.asarray(A)
    bm = BlockMatrix(blockSizes, None, ndiag, False, isHermitian)
    off = bm.offsets()
    for (i, j) in bm.pattern("out"):
        bm.M[(i, j)] = to_device(dense[off[i]:off[i + 1], off[j]:off[j + 1]])
    return bm


def bm_to_dense(bm):
    off = bm.offsets()
    n = off[-1]
    A = np.zeros((n, n), dtype=np.complex128)
    w = bm.band("out")
    for i in range(bm.npl):
        for j in range(max(0, i - w), min(bm.npl, i + w + 1)):
            if j < i and bm.isHermitian:
                A[off[i]:off[i + 1], off[j]:off[j + 1]] = np.conj(to_host(bm.M[(j, i)])).T
            elif (i, j) in bm.M and isinstance(bm.M[(i, j)], torch.Tensor):
                A[off[i]:off[i + 1], off[j]:off[j + 1]] = to_host(bm.M[(i, j)])
    return A


def bm_copy(bm):
    """blockmatrix.jl:231-262."""
    out = BlockMatrix(bm.blockSizes, None, bm.ndiag, bm.isArrayOrLU, bm.isHermitian)
    for k, v in bm.M.items():
        out.M[k] = be_copy_in_hw(v) if isinstance(v, torch.Tensor) else v
    return out


def bm_copy_(out, inp):
    """blockmatrix.jl:270-298."""
    for k in inp.pattern("out"):
        if k in inp.M:
            out.M[k].copy_(inp.M[k])


def bm_blocks_define_(bm, filling, rng=None):
    """blockmatrix.jl:334-391: 1 zero blocks, 2 random blocks."""
    if filling == 2 and bm.isArrayOrLU:
        raise ValueError("filling up BlockMatrix with random blocks and block-diagonal LUs makes no sense")
    for (i, j) in bm.pattern("in"):
        if i == j and bm.isArrayOrLU:
            bm.M[(i, j)] = be_zero_lu(bm.blockSizes[i])
        elif filling == 1:
            bm.M[(i, j)] = be_zero_array((bm.blockSizes[i], bm.blockSizes[j]))
        else:
            bm.M[(i, j)] = be_random_array((bm.blockSizes[i], bm.blockSizes[j]), rng)


def bm_similar(bm, filling, rng=None):
    """blockmatrix.jl:307-319."""
    out = BlockMatrix(bm.blockSizes, None, bm.ndiag, bm.isArrayOrLU, bm.isHermitian)
    if filling != 0:
        bm_blocks_define_(out, filling, rng)
    return out


def bm_empty(blockSizes, npl, ndiag, isArrayOrLU, isHermitian):
    """blockmatrix.jl:321-323."""
    return BlockMatrix(blockSizes, None, {"in": ndiag, "out": ndiag}, isArrayOrLU, isHermitian)


def bm_reference_(M, B, iOffset=0, jOffset=0):
    """bm_reference! (blockmatrix.jl:974-998, :1011-1040): the band of M
    (ndiag["out"], diagonal and upper only when Hermitian) refers to the
    blocks B[(i + iOffset, j + jOffset)] -- no copies, as in the reference.
    B: a block table (dict keyed by (i, j)) or a BlockMatrix."""
    table = B.M if isinstance(B, BlockMatrix) else B
    for (i, j) in M.pattern("out"):
        M.M[(i, j)] = table[(i + iOffset, j + jOffset)]
    return M


def bm_blocks_define_identity_(bm):
    """blockmatrix.jl:700-719."""
    if bm.ndiag["in"] > 1:
        raise ValueError("this function is meant, for now, only for block-diagonal block matrices")
    for i in range(bm.npl):
        bm.M[(i, i)] = be_identity(bm.blockSizes[i])


def bm_fuse_to_tridiagonal(bm):
    """blockmatrix.jl:1075-1106: fuse groups of w layers into one, so a block
    (2w+1)-diagonal matrix becomes block tridiagonal.  The fused blocks are
    assembled on the device from the original blocks (no dense round trip)."""
    w = bm.band("in")
    if w <= 1:
        return bm_copy(bm)
    old = bm.npl
    new_npl = -(-old // w)
    sizes = [0] * new_npl
    for ix in range(old):
        sizes[ix // w] += bm.blockSizes[ix]
    starts = [0] * old
    for ix in range(old):
        g = ix // w
        starts[ix] = sum(bm.blockSizes[g * w:ix])
    out = BlockMatrix(sizes, None, {"in": 3, "out": 3}, False, bm.isHermitian)
    for (I, J) in out.pattern("out"):
        out.M[(I, J)] = dzeros(sizes[I], sizes[J])
    for (i, j), blk in bm.M.items():
        I, J = i // w, j // w
        if (I, J) not in out.M:
            continue
        r0, c0 = starts[i], starts[j]
        out.M[(I, J)][r0:r0 + bm.blockSizes[i], c0:c0 + bm.blockSizes[j]].copy_(blk)
        if bm.isHermitian and i != j and (J, I) in out.M:
            out.M[(J, I)][c0:c0 + bm.blockSizes[j], r0:r0 + bm.blockSizes[i]].copy_(blk.conj().t())
    return out


def bm_create_synthetic_random(nrLayers, blocksDim, isHermitian=False, ndiag=None, seed=None, uniform=False):
    """blockmatrix.jl:878-964 with numpy's generator in place of Julia's."""
    rng = np.random.default_rng(seed)
    nd = 3 if ndiag is None else (ndiag["in"] if isinstance(ndiag, dict) else int(ndiag))
    if uniform:
        sizes = [int(blocksDim)] * nrLayers
    else:
        sizes = [int(x) for x in np.round(8.0 * rng.random(nrLayers) + (blocksDim - 4.0))]
    bm = BlockMatrix(sizes, None, {"in": nd, "out": nd}, False, isHermitian)
    w = (nd - 1) // 2
    for i in range(nrLayers):
        if not isHermitian:
            for j in range(i - 1, max(0, i - w) - 1, -1):
                bm.M[(i, j)] = to_device(0.3 * (rng.random((sizes[i], sizes[j])) + 1j * rng.random((sizes[i], sizes[j]))))
        bm.M[(i, i)] = to_device(rng.random((sizes[i], sizes[i])) + 1j * rng.random((sizes[i], sizes[i])))
        for j in range(i + 1, min(nrLayers, i + w + 1)):
            bm.M[(i, j)] = to_device(0.3 * (rng.random((sizes[i], sizes[j])) + 1j * rng.random((sizes[i], sizes[j]))))
    return bm


# --------------------------------------------------------------------------
# Block (src/block.jl) -- dense blocks of the selected inverse

class Block:
    """src/block.jl:9-34: ``Full`` is a device block (or None), row/col sizes."""

    def __init__(self, M=None, row=-1, col=-1):
        if M is not None:
            self.Full = M if isinstance(M, torch.Tensor) else to_device(M)
            self.row, self.col = self.Full.shape[0], self.Full.shape[1]
        else:
            self.Full, self.row, self.col = None, row, col


def set_sparse_Block(b, rind, cind, s_flag=False, seed=None):
    """set_sparse_Block(b, rind, cind, s_flag) (block.jl:582-598): random real
    uniform [0,1) blocks at the 1-based positions (rind, cind)."""
    rng = np.random.default_rng(seed)
    A = {}
    for r, c in zip(rind, cind):
        i, j = r - 1, c - 1
        A[(i, j)] = Block(rng.random((b[i], b[j])).astype(np.complex128))
        if s_flag and i != j:
            A[(j, i)] = Block(rng.random((b[j], b[i])).astype(np.complex128))
    return A


def get_row_sizes(A, npl):
    return [A[(i, i)].row for i in range(npl)]


def _block_dims(A):
    """(rows, cols) of a block dict: one past its largest assigned indices
    (a Julia Matrix{Block} carries its size; the dict does not)."""
    if not A:
        return 0, 0
    return 1 + max(i for i, _ in A), 1 + max(j for _, j in A)


def _ends(A, rowE, colE):
    r, c = _block_dims(A)
    return (r - 1 if rowE is None else rowE), (c - 1 if colE is None else colE)


def get_rc_index(A, nrows=None, ncols=None):
    """get_rc_index (block.jl:348-364): the row and column indices (0-based)
    of the assigned blocks among the first nrows rows and ncols columns,
    row by row."""
    r, c = _block_dims(A)
    nrows = r if nrows is None else nrows
    ncols = c if ncols is None else ncols
    rows, cols = [], []
    for i in range(nrows):
        for j in range(ncols):
            if (i, j) in A:
                rows.append(i)
                cols.append(j)
    return rows, cols


def get_rc_index_at_(rcInd, A, rowB=0, rowE=None, colB=0, colE=None, flag_row=True):
    """get_rc_index_at! (block.jl:377-394): rcInd (emptied first) receives the
    row (flag_row) or column index of every assigned block in rows
    rowB..rowE and columns colB..colE (0-based, ends included as in the
    reference's ranges), row by row."""
    rowE, colE = _ends(A, rowE, colE)
    del rcInd[:]
    for i in range(rowB, rowE + 1):
        for j in range(colB, colE + 1):
            if (i, j) in A:
                rcInd.append(i if flag_row else j)


def get_rc_index_at(A, rowB=0, rowE=None, colB=0, colE=None, flag_row=True):
    """get_rc_index_at (block.jl:396-412): the list get_rc_index_at_ fills."""
    out = []
    get_rc_index_at_(out, A, rowB, rowE, colB, colE, flag_row)
    return out


def _index_at(A, rowB, rowE, colB, colE, flag_row):
    rowE, colE = _ends(A, rowE, colE)
    slots = (rowE - rowB + 1) if flag_row else (colE - colB + 1)
    out = get_rc_index_at(A, rowB, rowE, colB, colE, flag_row)
    if len(out) > max(slots, 0):
        # the reference writes into a vector of that many slots (BoundsError)
        raise IndexError("more assigned blocks than %s in the range" % ("rows" if flag_row else "columns"))
    return out


def get_row_index_at(A, rowB=0, rowE=None, colB=0, colE=None):
    """get_row_index_at (block.jl:414-430): the row index of every assigned
    block in the range, row by row; at most one per row of the range."""
    return _index_at(A, rowB, rowE, colB, colE, True)


def get_col_index_at(A, rowB=0, rowE=None, colB=0, colE=None):
    """get_col_index_at (block.jl:432-447): the column index of every
    assigned block in the range, row by row; at most one per column of the
    range."""
    return _index_at(A, rowB, rowE, colB, colE, False)


def get_colSizes(A, npl=None):
    """get_colSizes (block.jl:476-482): column sizes of the diagonal blocks."""
    npl = _block_dims(A)[0] if npl is None else npl
    return [A[(i, i)].col for i in range(npl)]


def get_blockSizes(A, npl=None):
    """get_blockSizes (block.jl:493-501): (row sizes, column sizes) of the
    diagonal blocks."""
    npl = _block_dims(A)[0] if npl is None else npl
    return get_row_sizes(A, npl), get_colSizes(A, npl)


def _host_block(x):
    return None if x is None else (to_host(x) if isinstance(x, torch.Tensor) else np.asarray(x))


def bm_equal(A, B):
    """bm_equal (block.jl:223-243): the same blocks assigned in A and B and
    every pair equal (shape and entries)."""
    if set(A) != set(B):
        return False
    for k in A:
        a, b = _host_block(A[k].Full), _host_block(B[k].Full)
        if (a is None) != (b is None):
            return False
        if a is not None and not (a.shape == b.shape and np.array_equal(a, b)):
            return False
    return True


def full(A, npl=None):
    """full(A) (block.jl:547-569): dense host matrix of a block dict."""
    if npl is None:
        npl = 1 + max(max(k) for k in A)
    b = get_row_sizes(A, npl)
    off = np.concatenate([[0], np.cumsum(b)]).astype(int)
    out = np.zeros((off[-1], off[-1]), dtype=np.complex128)
    for (i, j), blk in A.items():
        if blk.Full is not None:
            out[off[i]:off[i + 1], off[j]:off[j + 1]] = to_host(blk.Full)
    return out
