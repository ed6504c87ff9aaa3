"""Sweep-level mirror of LibNEGF.jl's hot-path functions on the B200 library.

Each function keeps the reference's name (``!`` becomes a trailing ``_``),
argument order and meaning, and runs the whole sweep as one call into
libnegf_b200.so (one batched launch per recursion step).  Errors: a zero pivot
raises ``SingularError`` where the reference prints and calls ``exit()``
(src/backend_cpu.jl:151-155).

Batched forms (``*_batched``) take lists of systems with the same layer count
and run them in the same launches.
"""

import ctypes

import numpy as np
import scipy.sparse as sp

from ._lib import check, ptr_array, int_array, load
from .blockmatrix import (BlockMatrix, Block, bm_copy, bm_blocks_define_, dzeros, dptr, stream_handle,
                          to_device, to_host)


class TimingData:
    """Placeholder for src/utils/full_timings.jl:14 (timing is done with CUDA
    events and ncu in this library)."""


class CountingData:
    """Placeholder for src/utils/full_timings.jl:20."""


class AuxDataRGF:
    """src/matinvertndiag_rgf.jl:10-14.  The device workspace (LU/R/L blocks,
    identity) lives inside the library for the duration of a sweep."""

    def __init__(self, M, buildFullInv=False):
        self.blockSizes = list(M.blockSizes)
        self.ndiag = dict(M.ndiag)
        self.buildFullInv = bool(buildFullInv)


def allocate_aux_data_RGF(M, buildFullInv=False):
    """src/matinvertndiag_rgf.jl:80-97."""
    return AuxDataRGF(M, buildFullInv)


def required_mem_non_symm(npl, itemsize, N1diag, N3diag, avgBlockSize):
    """src/matinvertndiag_rgf.jl:39-67 (MB)."""
    req = 0.0
    for ix in range(npl):
        if ix > 0:
            req += N3diag * avgBlockSize * avgBlockSize
        req += N3diag * avgBlockSize * avgBlockSize + N1diag * avgBlockSize * avgBlockSize
        if ix < npl - 1:
            req += N3diag * avgBlockSize * avgBlockSize
    return req * (2 * itemsize / 2 ** 20)


def required_mem_symm(npl, itemsize, N1diag, N3diag, avgBlockSize):
    """src/keldyshndiag.jl:49-77 (MB)."""
    req = 0.0
    for ix in range(npl):
        req += N3diag * avgBlockSize * avgBlockSize + N1diag * avgBlockSize * avgBlockSize
        if ix < npl - 1:
            req += N3diag * avgBlockSize * avgBlockSize
    return req * (2 * itemsize / 2 ** 20)


def _free_hbm_mb():
    import torch
    free, _ = torch.cuda.mem_get_info()
    return free / 2 ** 20


def check_if_enough_mem_rgf(npl, blockSize, itemsize=8):
    """src/matinvertndiag_rgf.jl:16-33, against 80% of free HBM."""
    if required_mem_non_symm(npl, itemsize, 1, 3, blockSize) > 0.8 * _free_hbm_mb():
        raise MemoryError("The required memory exceeds 80% of the total memory")


def check_if_enough_mem_rkd(npl, blockSize, itemsize=8):
    """src/keldyshndiag.jl:14-43, against 80% of free HBM."""
    req = required_mem_non_symm(npl, itemsize, 1, 5, blockSize) + required_mem_symm(npl, itemsize, 0, 3, blockSize)
    if req > 0.8 * _free_hbm_mb():
        raise MemoryError("The required memory exceeds 80% of the total memory")


def _tri_tables(systems):
    npl = systems[0].npl
    for s in systems:
        if s.npl != npl:
            raise ValueError("all systems of a batched call need the same number of layers")
    sizes, Md, Mu, Ml = [], [], [], []
    for s in systems:
        sizes += s.blockSizes
        for i in range(npl):
            Md.append(dptr(s.M[(i, i)]))
        for i in range(npl - 1):
            Mu.append(dptr(s.M[(i, i + 1)]))
            Ml.append(dptr(s.M[(i + 1, i)]))
    return npl, sizes, Md, Mu, Ml


def _ensure_out(Mout, full=False):
    w = Mout.npl if full else 1
    Mout.ndiag = dict(Mout.ndiag)
    for i in range(Mout.npl):
        for j in range(max(0, i - w), min(Mout.npl, i + w + 1)):
            blk = Mout.M.get((i, j))
            if blk is None or not hasattr(blk, "data_ptr") or tuple(blk.shape) != (Mout.blockSizes[i], Mout.blockSizes[j]):
                Mout.M[(i, j)] = dzeros(Mout.blockSizes[i], Mout.blockSizes[j])


def bndiag_of_inv_rgf_local_batched_(Mouts, Mins, buildFullInv=False):
    npl, sizes, Md, Mu, Ml = _tri_tables(Mins)
    for o in Mouts:
        _ensure_out(o, buildFullInv)
    Gd = [dptr(o.M[(i, i)]) for o in Mouts for i in range(npl)]
    Gu = [dptr(o.M[(i, i + 1)]) for o in Mouts for i in range(npl - 1)]
    Gl = [dptr(o.M[(i + 1, i)]) for o in Mouts for i in range(npl - 1)]
    gfull = None
    if buildFullInv:
        gfull = ptr_array([dptr(o.M[(i, j)]) for o in Mouts for i in range(npl) for j in range(npl)])
        for o in Mouts:
            o.ndiag = {"in": 3, "out": 2 * npl - 1}
    check(load().negf_rgf(len(Mins), npl, int_array(sizes), ptr_array(Md), ptr_array(Mu), ptr_array(Ml),
                          ptr_array(Gd), ptr_array(Gu), ptr_array(Gl), gfull, stream_handle()))


def bndiag_of_inv_rgf_local_(Mout, Min, auxData=None, td=None, cd=None):
    """bndiag_of_inv_rgf_local! (src/matinvertndiag_rgf.jl:114-200): Mout gets
    the block tridiagonal of Min^{-1} (every block with buildFullInv)."""
    full = bool(auxData.buildFullInv) if auxData is not None else False
    bndiag_of_inv_rgf_local_batched_([Mout], [Min], full)


def bndiag_of_inv_rgf_global_(Mout, Min, auxData=None, td=None, cd=None):
    """src/matinvertndiag_ddrgf_core.jl:32-46 (the same sweep; BLAS threading
    has no analogue on the GPU)."""
    bndiag_of_inv_rgf_local_(Mout, Min, auxData, td, cd)


class AuxDataKeldysh:
    """src/keldyshndiag.jl:7-12; ``buffS`` receives G^n."""

    def __init__(self, M, S):
        self.auxDataRGF = allocate_aux_data_RGF(M)
        self.buffS = bm_copy(S)


def allocate_aux_data_Keldysh(M, S):
    """src/keldyshndiag.jl:79-107."""
    return AuxDataKeldysh(M, S)


def keldyshndiag_batched_(Ms, auxs):
    npl, sizes, Md, Mu, Ml = _tri_tables(Ms)
    Sd = [dptr(a.buffS.M[(i, i)]) for a in auxs for i in range(npl)]
    Su = [dptr(a.buffS.M[(i, i + 1)]) for a in auxs for i in range(npl - 1)]
    check(load().negf_keldysh(len(Ms), npl, int_array(sizes), ptr_array(Md), ptr_array(Mu), ptr_array(Ml),
                              ptr_array(Sd), ptr_array(Su), stream_handle()))


def keldyshndiag_(M, S, auxData, td=None, cd=None):
    """keldyshndiag! (src/keldyshndiag.jl:120-131 -> v3 :166-188): the block
    tridiagonal of M^{-1} S M^{-H} lands in auxData.buffS (Hermitian storage)."""
    for k in S.M:
        auxData.buffS.M[k].copy_(S.M[k])
    keldyshndiag_batched_([M], [auxData])


def allocate_aux_data_general_RGF(M):
    """src/matinvertndiag_general_rgf.jl:8-24."""
    return AuxDataRGF(M, False)


def bndiag_of_inv_general_rgf_(Mout, Min, auxData=None, td=None, cd=None):
    """bndiag_of_inv_general_rgf! (src/matinvertndiag_general_rgf.jl:31-146):
    Mout gets the block n-diagonal of Min^{-1} (n = Min.ndiag["in"]).  Min is
    left unchanged (the reference overwrites it with Schur-updated blocks)."""
    npl = Min.npl
    nd = Min.ndiag["in"]
    w = (nd - 1) // 2
    Mout.ndiag = {"in": nd, "out": nd}
    Mb, Gb = [], []
    for i in range(npl):
        for j in range(npl):
            if abs(i - j) <= w:
                Mb.append(dptr(Min.M[(i, j)]))
                blk = Mout.M.get((i, j))
                if blk is None or tuple(blk.shape) != (Min.blockSizes[i], Min.blockSizes[j]):
                    Mout.M[(i, j)] = dzeros(Min.blockSizes[i], Min.blockSizes[j])
                Gb.append(dptr(Mout.M[(i, j)]))
            else:
                Mb.append(None)
                Gb.append(None)
    check(load().negf_general_rgf(1, npl, nd, int_array(Min.blockSizes), ptr_array(Mb), ptr_array(Gb),
                                  stream_handle()))


# --------------------------------------------------------------------------
# selected inverse (src/selected_inverse.jl)

def _selinv(A, mode):
    npl = 1 + max(max(k) for k in A)
    b = A[(0, 0)].row
    for (i, j), blk in A.items():
        if blk.row != b or blk.col != b:
            raise ValueError("the selected inverse assumes a uniform block size (selected_inverse.jl:146-152)")
    # fill-in blocks created by the factorisation (selected_inverse.jl:41-46)
    pattern = set(A.keys())
    fill = set()
    if mode & 1:
        for i in range(npl):
            for k in range(i + 1, npl):
                if (i, k) in pattern:
                    for l in range(k + 1, npl):
                        if (i, l) in pattern and (k, l) not in pattern:
                            pattern.add((k, l))
                            pattern.add((l, k))
                            fill.add((k, l))
                            fill.add((l, k))
    for k in fill:
        A[k] = Block(dzeros(b, b))
    tab = [None] * (npl * npl)
    fl = (ctypes.c_uint8 * (npl * npl))()
    for (i, j), blk in A.items():
        tab[i * npl + j] = dptr(blk.Full)
        fl[i * npl + j] = 1 if (i, j) in fill else 0
    check(load().negf_selected_inverse(npl, b, ptr_array(tab), fl, mode, stream_handle()))
    return A


def _copy_blocks(A):
    out = {}
    for k, v in A.items():
        c = Block(dzeros(v.row, v.col))
        c.Full.copy_(v.Full)
        out[k] = c
    return out


def Block_factorization_(A, td=None, cd=None):
    """Block_factorization! (selected_inverse.jl:9-55): block LU in place
    (diagonal pivots discarded, as the reference's be_getrf! does)."""
    return _selinv(A, 1)


def Block_factorization_noT_(A):
    """Block_factorization_noT! (selected_inverse.jl:57-104): the same block LU
    without the timing / counting wrappers."""
    return _selinv(A, 1)


def Block_factorization(A, td=None, cd=None):
    """selected_inverse.jl:124-128."""
    return Block_factorization_(_copy_blocks(A), td, cd)


def Block_inverse_(A, td=None, cd=None):
    """Block_inverse! (selected_inverse.jl:139-206): selected inverse of a
    factored block matrix, in place."""
    return _selinv(A, 2)


def Block_inverse(A, td=None, cd=None):
    """selected_inverse.jl:222-226."""
    return Block_inverse_(_copy_blocks(A), td, cd)


# --------------------------------------------------------------------------
# DDRGF (src/matinvertndiag_ddrgf_*.jl)

def bndiag_of_inv_ddrgf_get_nr_tasks(npl, blockSizeD1, blockSizeD2=1):
    """src/matinvertndiag_ddrgf_utils.jl:278-312."""
    if blockSizeD2 != 1:
        raise ValueError("The value of blockSizeD2 should be set to 1")
    nr = ctypes.c_int32()
    last = ctypes.c_int32()
    check(load().negf_ddrgf_get_nr_tasks(npl, blockSizeD1, ctypes.byref(nr), ctypes.byref(last)))
    return [nr.value, last.value]


class AuxDataDDRGF:
    """One DDRGF level (src/matinvertndiag_ddrgf_core.jl:1-30): the layer sizes
    of the matrix this level partitions (the original matrix at level 1, the
    previous level's separator Schur complement below), its interior size and
    task count, and -- at level 1 -- the output buffer ``buffMout``.  The
    coarse levels' Schur complements live inside the library's plan."""

    def __init__(self, blockSizes, blockSizeD1, level=1):
        self.level = level
        self.blockSizes = list(blockSizes)
        self.blockSizeD1 = int(blockSizeD1)
        self.blockSizeD2 = 1
        self.nrTasks, self.lastSizeD1 = bndiag_of_inv_ddrgf_get_nr_tasks(len(self.blockSizes), self.blockSizeD1)
        self.permVecInv, self.sizeDomains, self.permVec = [], [], []
        if self.nrTasks >= 1 and self.blockSizeD1 < len(self.blockSizes):
            self.permVecInv, self.sizeDomains = bndiag_of_inv_ddrgf_create_permutation_vector(
                len(self.blockSizes), self.blockSizeD1)
            self.permVec = bndiag_of_inv_ddrgf_transpose_permutation_vector(self.permVecInv)
        self.buffMout = None
        if level == 1:
            self.buffMout = BlockMatrix(self.blockSizes, None, {"in": 3, "out": 3}, False, False)
            bm_blocks_define_(self.buffMout, 1)

    def separator_sizes(self):
        """Layer sizes of this level's Schur complement (one per separator)."""
        if self.nrTasks < 1:
            return []
        return [self.blockSizes[t * (self.blockSizeD1 + 1)] for t in range(self.nrTasks)]


def bndiag_of_inv_ddrgf_create_permutation_vector(M, nrBlocksInNonPivots):
    """bndiag_of_inv_ddrgf_create_permutation_vector (ddrgf_utils.jl:478-575),
    0-based: permVecInv lists the old layer index of every new position --
    first the separators ("D2", one layer at the start of each task), then
    the interior layers ("D1") task by task -- and sizeDomains the sizes of
    those subdomains in the same order.  M: a BlockMatrix or its layer count."""
    npl = M if isinstance(M, int) else len(M.blockSizes)
    d1 = int(nrBlocksInNonPivots)
    nr, last = bndiag_of_inv_ddrgf_get_nr_tasks(npl, d1)
    if nr < 1:
        raise ValueError("DDRGF partition impossible for %d layers and interior size %d" % (npl, d1))
    sizes1 = [d1] * nr
    if last:
        sizes1[-1] = last
    perm_inv, size_domains = [], []
    x = 0
    for t in range(nr):  # region 2: the pivots
        perm_inv.append(x)
        size_domains.append(1)
        x += 1 + sizes1[t]
    x = 0
    for t in range(nr):  # region 1: the interiors
        x += 1
        perm_inv.extend(range(x, x + sizes1[t]))
        size_domains.append(sizes1[t])
        x += sizes1[t]
    return perm_inv, size_domains


def bndiag_of_inv_ddrgf_transpose_permutation_vector(permVec):
    """ddrgf_utils.jl:579-587: the inverse permutation (0-based)."""
    inv = list(permVec)
    for i, p in enumerate(permVec):
        inv[p] = i
    return inv


def bndiag_of_inv_ddrgf_create_permuted_matrix(M, permVec):
    """ddrgf_utils.jl:591-624: the block matrix P M P^T whose blocks are the
    blocks of M (references, no copies): block (i, j) of the band of M lands
    at (permVec[i], permVec[j]), and the block sizes move with it."""
    sizes = [0] * len(M.blockSizes)
    for i, b in enumerate(M.blockSizes):
        sizes[permVec[i]] = b
    Mhat = BlockMatrix(sizes, None, M.ndiag, False, M.isHermitian)
    for (i, j) in M.pattern("out"):
        if (i, j) in M.M:
            Mhat.M[(permVec[i], permVec[j])] = M.M[(i, j)]
    return Mhat


def bndiag_of_inv_ddrgf_create_sparse_permutator(permVec, blockSizes):
    """bndiag_of_inv_ddrgf_create_sparse_permutator (blockmatrix.jl:194-222):
    the sparse permutation matrix P (n x n, n the sum of the block sizes)
    whose identity block for layer j sits at the rows of its new position
    permVec[j] (0-based), so that P M P^T is the element form of
    bndiag_of_inv_ddrgf_create_permuted_matrix(M, permVec)."""
    npl = len(blockSizes)
    sizes_perm = [0] * npl
    for i in range(npl):
        sizes_perm[permVec[i]] = blockSizes[i]
    off_p = np.concatenate([[0], np.cumsum(sizes_perm)]).astype(int)
    off = np.concatenate([[0], np.cumsum(blockSizes)]).astype(int)
    rows, cols = [], []
    for j in range(npl):
        i = permVec[j]
        rows.extend(range(off_p[i], off_p[i + 1]))
        cols.extend(range(off[j], off[j + 1]))
    n = int(off[-1])
    return sp.csc_matrix((np.ones(n, dtype=np.complex128), (rows, cols)), shape=(n, n))


def check_if_enough_mem_ddrgf(npl, blockSize, itemsize=8):
    """check_if_enough_mem_ddrgf (ddrgf_utils.jl:1-34): the memory estimate
    of DDRGF in MB -- the RGF buffers (1 block-diagonal, 3 block-tridiagonal)
    plus DDRGF's own (buffTHat and buffMout, and one block diagonal for its
    other allocations).  The reference's comparison against 80 % of the
    memory is disabled there, so this raises nothing either; it returns the
    estimate."""
    return (required_mem_non_symm(npl, itemsize, 1, 3, blockSize) +
            required_mem_non_symm(npl, itemsize, 1, 2, blockSize))


def bndiag_of_inv_ddrgf_check_nr_threads(nrThreads, nrTasks):
    """bndiag_of_inv_ddrgf_check_nr_threads (ddrgf_utils.jl:455-465):
    (threads used, tasks per thread, tasks of the last thread)."""
    t, m, l = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    check(load().negf_ddrgf_check_nr_threads(int(nrThreads), int(nrTasks), ctypes.byref(t), ctypes.byref(m),
                                             ctypes.byref(l)))
    return t.value, m.value, l.value


def cost_rgf(L, rLU, rMLDIV, doFull):
    """cost_rgf (ddrgf_utils.jl:221-247), in units of one GEMM."""
    c = ctypes.c_double()
    check(load().negf_ddrgf_cost_rgf(int(L), float(rLU), float(rMLDIV), int(bool(doFull)), ctypes.byref(c)))
    return c.value


def cost_ddrgf(rLU, rMLDIV, nrTasks, nrThreads, blockSizeD1):
    """cost_ddrgf (ddrgf_utils.jl:249-276), in units of one GEMM."""
    c = ctypes.c_double()
    check(load().negf_ddrgf_cost_ddrgf(float(rLU), float(rMLDIV), int(nrTasks), int(nrThreads), int(blockSizeD1),
                                       ctypes.byref(c)))
    return c.value


def allocate_aux_data_DDRGF_single_level(M, nrBlocksInNonPivots, auxDataSeq=None, nrTasks=None):
    """allocate_aux_data_DDRGF_single_level (ddrgf_setup.jl:63-220): one level's
    partition, permutation and (for a BlockMatrix input) output buffer."""
    sizes = M.blockSizes if hasattr(M, "blockSizes") else list(M)
    a = AuxDataDDRGF(sizes, nrBlocksInNonPivots, level=1)
    if nrTasks is not None and nrTasks != a.nrTasks:
        raise ValueError("nrTasks %d does not match the partition (%d)" % (nrTasks, a.nrTasks))
    return a


def bndiag_of_inv_ddrgf_error_inv_of_T11(Min, Mout, auxData, td=None, cd=None):
    """bndiag_of_inv_ddrgf_error_inv_of_T11 (ddrgf_utils.jl:776-824): the
    diagnostic sqrt(sum ||(T11 T11^{-1})_{ij} - delta_ij I||_F^2 / sum_i b_i)
    over the interior domains of auxData's partition.  The domains' full
    inverses are recomputed by the library's RGF (buildFullInv); Mout is not
    needed (the reference uses one of its blocks as scratch).  Unlike the
    reference's rough version, domains of different sizes are handled."""
    from .blockmatrix import be_gemm_
    perm_inv, sizes = auxData.permVecInv, auxData.sizeDomains
    nr = auxData.nrTasks
    layers1 = perm_inv[nr:]
    num, den, o = 0.0, 0.0, 0
    for nd in sizes[nr:]:
        d = layers1[o:o + nd]
        o += nd
        bs = [Min.blockSizes[i] for i in d]
        full = {(a, b): dzeros(bs[a], bs[b]) for a in range(nd) for b in range(nd)}
        Gd = [full[(a, a)] for a in range(nd)]
        check(load().negf_rgf(1, nd, int_array(bs), ptr_array([dptr(Min.M[(i, i)]) for i in d]),
                              ptr_array([dptr(Min.M[(d[a], d[a + 1])]) for a in range(nd - 1)]),
                              ptr_array([dptr(Min.M[(d[a + 1], d[a])]) for a in range(nd - 1)]),
                              ptr_array([dptr(g) for g in Gd]), None, None,
                              ptr_array([dptr(full[(a, b)]) for a in range(nd) for b in range(nd)]),
                              stream_handle()))
        for a in range(nd):
            for b in range(nd):
                acc = dzeros(bs[a], bs[b])
                for k in (a - 1, a, a + 1):
                    if 0 <= k < nd:
                        be_gemm_("N", "N", 1.0, Min.M[(d[a], d[k])], full[(k, b)], 1.0, acc)
                x = to_host(acc)
                if a == b:
                    x = x - np.eye(bs[a])
                    den += bs[a]
                num += float(np.linalg.norm(x)) ** 2
    return float(np.sqrt(num / den)) if den else 0.0


def _probe_samples(M):
    # the reference's sample count (ddrgf_utils.jl:42-44), capped for the GPU
    avg = max(1, sum(M.blockSizes) // len(M.blockSizes))
    return avg, min(64, int(1.0e4 * 1.0e5 / avg ** 3) + 10)


def _time_ratio(M, op):
    """Per-sample ratios t(op)/t(GEMM) on blocks of the average size, timed with
    CUDA events around single-block library calls (one sample = one call)."""
    import torch
    from .blockmatrix import be_random_array, be_zero_lu, be_gemm_
    avg, n = _probe_samples(M)
    rng = np.random.default_rng(0)
    A = be_random_array((avg, avg), rng) + to_device(avg * np.eye(avg))
    B = be_random_array((avg, avg), rng)
    C = dzeros(avg, avg)
    lu = be_zero_lu(avg)
    be_gemm_("N", "N", 1.0, A, B, 1.0, C)
    op(A, B, C, lu)
    st = torch.cuda.current_stream()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    ratios = []
    for _ in range(n):
        e0.record(st)
        be_gemm_("N", "N", 1.0, A, B, 1.0, C)
        e1.record(st)
        op(A, B, C, lu)
        e2.record(st)
        e2.synchronize()
        ratios.append(e1.elapsed_time(e2) / max(1e-6, e0.elapsed_time(e1)))
    return np.array(ratios)


def get_rLU(M, td=None, cd=None):
    """get_rLU (src/matinvertndiag_ddrgf_utils.jl:158-219): [mean, std] of
    t(be_lu!)/t(be_gemm!) on blocks of the average size, on the GPU."""
    from .blockmatrix import be_lu_
    r = _time_ratio(M, lambda A, B, C, lu: be_lu_(lu, A))
    return [float(r.mean()), float(r.std())]


def get_rMLDIV(M, td=None, cd=None):
    """get_rMLDIV (src/matinvertndiag_ddrgf_utils.jl:95-156): [mean, std] of
    t(be_mldivide!)/t(be_gemm!) with an already factored block, on the GPU."""
    from .blockmatrix import be_mldivide_
    r = _time_ratio(M, lambda A, B, C, lu: be_mldivide_("N", C, B, lu))
    return [float(r.mean()), float(r.std())]


def get_dampRGF(M, td=None, cd=None):
    """get_dampRGF (src/matinvertndiag_ddrgf_utils.jl:36-93) measures how much
    slower a GEMM runs on one BLAS thread than on all of them, the share of
    the machine the coarse sequential RGF gets.  A GPU step has no such split
    (every launch of the Schur RGF gets the whole GPU): [1.0, 0.0]."""
    return [1.0, 0.0]


def _max_levels():
    from ._lib import NEGF_DDRGF_MAX_LEVELS
    return NEGF_DDRGF_MAX_LEVELS


def opt_params(Min, rLU, rMLDIV, dampRGF, nrThreads=None):
    """opt_params (src/matinvertndiag_ddrgf_utils.jl:357-453), the reference's
    partition search restated in the library: returns (nrLevels,
    nrTasksList, blockSizeD1List, optCost) for nrThreads CPU threads
    (default: all host cores).  Min: a BlockMatrix or its layer count."""
    import os
    K = _max_levels()
    nl = ctypes.c_int32()
    tasks = (ctypes.c_int32 * K)()
    d1 = (ctypes.c_int32 * K)()
    cost = ctypes.c_double()
    npl = Min if isinstance(Min, int) else len(Min.blockSizes)
    check(load().negf_ddrgf_opt_params(npl, int(nrThreads or os.cpu_count() or 1), float(rLU), float(rMLDIV),
                                       float(dampRGF), ctypes.byref(nl), tasks, d1, ctypes.byref(cost)))
    return nl.value, list(tasks[:nl.value]), list(d1[:nl.value]), cost.value


def choose_levels(npl, blockSize, nsys=1, maxLevels=None):
    """Interior sizes per level from the library's GPU cost model ([] when
    sequential RGF is cheapest)."""
    nl = ctypes.c_int32()
    d1 = (ctypes.c_int32 * _max_levels())()
    check(load().negf_ddrgf_choose_levels(npl, blockSize, nsys, int(maxLevels or _max_levels()), ctypes.byref(nl),
                                          d1))
    return list(d1[:nl.value])


def allocate_aux_data_DDRGF(Min, td=None, cd=None, blockSizeD1=None, costModel="gpu", nrThreads=None):
    """allocate_aux_data_DDRGF (src/matinvertndiag_ddrgf_setup.jl:4-51): one
    ``AuxDataDDRGF`` per level.

    blockSizeD1: an interior size (one level) or a list (one per level).
    Without it the levels come from a cost model: ``costModel="reference"``
    runs the reference's probes (get_rLU / get_rMLDIV / get_dampRGF, timed on
    the GPU) and its opt_params search, and builds max(1, nrLevels - 1)
    levels from the result as the reference does (setup.jl:36-48);
    ``costModel="gpu"`` (default) uses the library's GPU model (serial
    launch depth against batched GEMM work).  An empty choice (sequential RGF
    is cheapest) gives one level with blockSizeD1 = npl."""
    npl = Min.npl
    if blockSizeD1 is not None:
        d1s = [int(blockSizeD1)] if np.isscalar(blockSizeD1) else [int(d) for d in blockSizeD1]
    elif costModel == "reference":
        rLU = get_rLU(Min, td, cd)[0]
        rMLDIV = get_rMLDIV(Min, td, cd)[0]
        damp = get_dampRGF(Min, td, cd)[0]
        nrLevels, _, d1List, _ = opt_params(Min, rLU, rMLDIV, damp, nrThreads)
        d1s = d1List[:max(1, nrLevels - 1)]
    else:
        d1s = choose_levels(npl, max(Min.blockSizes), 1) or [npl]
    aux, sizes = [], list(Min.blockSizes)
    for k, d1 in enumerate(d1s):
        a = AuxDataDDRGF(sizes, d1, level=k + 1)
        aux.append(a)
        if a.nrTasks < 2 or d1 >= len(sizes):
            break
        sizes = a.separator_sizes()
    return aux


def bndiag_of_inv_ddrgf_(Min, listOfAuxData, td=None, cd=None, depth=1):
    """bndiag_of_inv_ddrgf! (src/matinvertndiag_ddrgf_core.jl:719-758) over
    the levels listOfAuxData[depth-1:], in one library call: the block
    tridiagonal of Min^{-1} lands in listOfAuxData[depth-1].buffMout."""
    aux = listOfAuxData[depth - 1]
    if aux.buffMout is None:
        raise ValueError("the output of a coarse DDRGF level stays inside the library")
    npl, sizes, Md, Mu, Ml = _tri_tables([Min])
    out = aux.buffMout
    Gd = [dptr(out.M[(i, i)]) for i in range(npl)]
    Gu = [dptr(out.M[(i, i + 1)]) for i in range(npl - 1)]
    Gl = [dptr(out.M[(i + 1, i)]) for i in range(npl - 1)]
    d1s = [a.blockSizeD1 for a in listOfAuxData[depth - 1:]]
    check(load().negf_ddrgf_levels(1, npl, int_array(sizes), ptr_array(Md), ptr_array(Mu), ptr_array(Ml),
                                   len(d1s), int_array(d1s), ptr_array(Gd), ptr_array(Gu), ptr_array(Gl),
                                   stream_handle()))


# --------------------------------------------------------------------------
# Dense debug path (src/matinvertndiag_direct.jl)

def _csc_direct(M, blockSizes, ndiag):
    import scipy.sparse as sp
    from ._lib import CCscMatrix
    A = sp.csc_matrix(M, dtype=np.complex128, copy=True)
    A.sort_indices()
    n = A.shape[0]
    if A.shape[1] != n:
        raise ValueError("bndiag_of_inv_direct needs a square matrix")
    colptr = np.ascontiguousarray(A.indptr, dtype=np.int32)
    rowval = np.ascontiguousarray(A.indices, dtype=np.int32)
    nz = np.ascontiguousarray(A.data, dtype=np.complex128)
    res = CCscMatrix()
    c_int32_p = ctypes.POINTER(ctypes.c_int32)
    check(load().negf_bndiag_of_inv_direct(n, A.nnz, colptr.ctypes.data_as(c_int32_p),
                                           rowval.ctypes.data_as(c_int32_p), nz.ctypes.data, len(blockSizes),
                                           int_array([int(b) for b in blockSizes]), int(ndiag.get("out", 3)),
                                           ctypes.byref(res)))
    libc = ctypes.CDLL(None)
    try:
        cp = np.ctypeslib.as_array(res.colptr, shape=(n + 1,)).copy()
        rv = np.ctypeslib.as_array(res.rowval, shape=(max(1, res.nnz),))[:res.nnz].copy()
        vals = np.ctypeslib.as_array(ctypes.cast(res.nzval, ctypes.POINTER(ctypes.c_double)),
                                     shape=(2 * max(1, res.nnz),))[:2 * res.nnz].copy()
    finally:
        for p in (res.colptr, res.rowval, res.nzval):
            libc.free(ctypes.cast(p, ctypes.c_void_p))
    return sp.csc_matrix((vals[0::2] + 1j * vals[1::2], rv, cp), shape=(n, n))


def bndiag_of_inv_direct(M, blockSizes, ndiag):
    """bndiag_of_inv_direct (src/matinvertndiag_direct.jl:78-85, and the
    catch-all form :100-140 for dense input): the block n-diagonal part of
    M^{-1} (ndiag["out"]) through the whole inverse, computed on the GPU; M is
    a scipy sparse matrix or a dense array, the result a scipy CSC matrix."""
    return _csc_direct(M, blockSizes, ndiag)


def bndiag_of_inv_direct_(M, blockSizes, ndiag):
    """bndiag_of_inv_direct! (src/matinvertndiag_direct.jl:17-61): M (scipy
    CSC) becomes itself with its out band replaced by the inverse's."""
    R = _csc_direct(M, blockSizes, ndiag)
    M.data, M.indices, M.indptr = R.data, R.indices, R.indptr
    M.has_sorted_indices = True


# --------------------------------------------------------------------------
# Input preparation (src/matloader.jl)

def build_M_from_HS(H, S, Se, energVal):
    """build_M_from_HS (matloader.jl:85-95): M = E S - H - S_e for host
    matrices (scipy sparse or dense), as the reference's loader prepares the
    input of the direct / C-interface paths.  The batched solver assembles
    M(E) = (E + i eta) S - H - Sigma(E) on the device instead
    (Device.set_overlap, Solver.set_self_energies)."""
    return energVal * S - H - Se
