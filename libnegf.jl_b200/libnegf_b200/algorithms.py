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
    """src/matinvertndiag_ddrgf_core.jl:1-30 (one level): the partition and
    the output buffer ``buffMout``."""

    def __init__(self, M, blockSizeD1):
        self.blockSizeD1 = int(blockSizeD1)
        self.blockSizeD2 = 1
        self.nrTasks, self.lastSizeD1 = bndiag_of_inv_ddrgf_get_nr_tasks(M.npl, self.blockSizeD1)
        self.buffMout = BlockMatrix(M.blockSizes, None, {"in": 3, "out": 3}, False, False)
        bm_blocks_define_(self.buffMout, 1)


def allocate_aux_data_DDRGF(Min, td=None, cd=None, blockSizeD1=None):
    """allocate_aux_data_DDRGF (src/matinvertndiag_ddrgf_setup.jl:4-51): the
    reference times LAPACK probes and searches a cost model
    (ddrgf_utils.jl:357-453); here the library's cost model for the GPU picks
    the interior domain size unless blockSizeD1 is given."""
    if blockSizeD1 is None:
        d1 = ctypes.c_int32()
        check(load().negf_ddrgf_choose_d1(Min.npl, max(Min.blockSizes), 1, ctypes.byref(d1)))
        blockSizeD1 = d1.value
    return [AuxDataDDRGF(Min, blockSizeD1)]


def bndiag_of_inv_ddrgf_(Min, listOfAuxData, td=None, cd=None, depth=1):
    """bndiag_of_inv_ddrgf! (src/matinvertndiag_ddrgf_core.jl:719-758): the
    block tridiagonal of Min^{-1} lands in listOfAuxData[0].buffMout."""
    aux = listOfAuxData[depth - 1]
    npl, sizes, Md, Mu, Ml = _tri_tables([Min])
    out = aux.buffMout
    Gd = [dptr(out.M[(i, i)]) for i in range(npl)]
    Gu = [dptr(out.M[(i, i + 1)]) for i in range(npl - 1)]
    Gl = [dptr(out.M[(i + 1, i)]) for i in range(npl - 1)]
    check(load().negf_ddrgf(1, npl, int_array(sizes), ptr_array(Md), ptr_array(Mu), ptr_array(Ml),
                            aux.blockSizeD1, ptr_array(Gd), ptr_array(Gu), ptr_array(Gl), stream_handle()))
