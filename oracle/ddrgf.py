"""Oracle restatement of domain-decomposed RGF (DDRGF), one or more levels.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Partition and permutation follow ``bndiag_of_inv_ddrgf_get_nr_tasks``
(src/matinvertndiag_ddrgf_utils.jl:278-312) and
``bndiag_of_inv_ddrgf_create_permutation_vector`` (:478-575): separators
("D2", one layer each) sit at layers t*(D1+1), interiors ("D1") fill the layers
between.  The phases follow ``bndiag_of_inv_ddrgf!``
(src/matinvertndiag_ddrgf_core.jl:719-758):

1. ``_inv_of_T11!`` (:437-498): full inverse of every interior domain, by RGF
   with ``buildFullInv``.
2. ``_compute_THat11Inv_x_THat12!`` (:48-114), ``_compute_THat21_x_THat11Inv!``
   (:203-266) and ``_build_Schur_compl!`` (:500-654): the separator Schur
   complement S = T22 - T21 T11^{-1} T12 (block tridiagonal over separators).
3. ``_inv_Schur_compl!`` (:656-680): the separator Schur complement is itself
   block tridiagonal; at the last level it is inverted by sequential RGF, else
   by DDRGF with the next level's interior size (the recursive call at
   :673-679).
4. ``_compute_minus_THat11Inv_x_THat12_x_THatSInv!`` (:116-201),
   ``_compute_minus_x_THatSInv_THat21_x_THat11Inv!`` (:268-344) and
   ``_compute_11_part!`` (:346-435): the 12, 21 and 11 parts.

The result is returned in the original (unpermuted) layer order, as
``listAux[1].buffMout`` is in the reference tests.

The partition search of ``allocate_aux_data_DDRGF`` is restated too:
``cost_rgf`` / ``cost_ddrgf`` (src/matinvertndiag_ddrgf_utils.jl:221-276),
``check_nr_threads`` (:455-465) and ``opt_params`` (:357-453).
"""

import numpy as np

from .backend_cpu import be_gemm
from .blockmatrix import BlockMatrix
from .rgf import bndiag_of_inv_rgf_local


def get_nr_tasks(npl, block_size_d1, block_size_d2=1):
    """``bndiag_of_inv_ddrgf_get_nr_tasks`` (matinvertndiag_ddrgf_utils.jl:278-312)."""
    if block_size_d2 != 1:
        raise ValueError("The value of blockSizeD2 should be set to 1")
    per = block_size_d1 + block_size_d2
    nr = npl // per + 1
    left = npl - (nr - 1) * per
    d1_left = left - 1
    if left == 0:
        return nr - 1, 0
    if d1_left == 0:
        return -1, 0
    return nr, d1_left


def partition(npl, block_size_d1):
    """Separator layers and interior domains (0-based, original order), plus
    ``permVecInv`` of ``_create_permutation_vector`` (utils.jl:478-575)."""
    nr, last = get_nr_tasks(npl, block_size_d1)
    if nr < 1:
        raise ValueError("DDRGF partition impossible for npl=%d, D1=%d" % (npl, block_size_d1))
    seps, doms = [], []
    x = 0
    for t in range(nr):
        seps.append(x)
        size = last if (t == nr - 1 and last != 0) else block_size_d1
        doms.append(list(range(x + 1, x + 1 + size)))
        x += 1 + size
    perm_inv = seps + [i for d in doms for i in d]
    return seps, doms, perm_inv


def _sub(M, layers):
    sub = BlockMatrix([M.blockSizes[i] for i in layers], {"in": 3, "out": 3}, False)
    for a, i in enumerate(layers):
        for b, j in enumerate(layers):
            if (i, j) in M.M and abs(a - b) <= 1:
                sub.M[(a, b)] = M.M[(i, j)]
    return sub


def bndiag_of_inv_ddrgf(M, block_size_d1):
    """Block tridiagonal of M^{-1} by DDRGF; returns (G, S) with S the first
    level's separator Schur complement as a dict {(t, u): block}.

    block_size_d1: the interior size (one level), or a list of them, one per
    level, the k-th partitioning the Schur complement of level k-1."""
    d1s = [block_size_d1] if np.isscalar(block_size_d1) else list(block_size_d1)
    npl = M.npl
    if d1s[0] >= npl:
        return bndiag_of_inv_rgf_local(M), None
    seps, doms, _ = partition(npl, d1s[0])
    T = len(seps)
    if T == 1:
        # matinvertndiag_ddrgf_core.jl:726-729: nrTasks == 1 runs sequential RGF
        return bndiag_of_inv_rgf_local(M), None
    A = M.M
    # 1. full inverse of every interior domain
    Tinv = []
    for d in doms:
        sub = _sub(M, d)
        g = bndiag_of_inv_rgf_local(sub, build_full_inv=True).M
        if len(d) <= 2:
            # the full inverse of a 1- or 2-layer domain is its tridiagonal
            pass
        Tinv.append(g)
    # 2. Schur complement on separators
    S = {}
    for t in range(T):
        s = seps[t]
        X = A[(s, s)].copy()
        f, l = 0, len(doms[t]) - 1
        fl, ll = doms[t][0], doms[t][-1]
        # THat21 x THat11Inv restricted to the corner blocks, then x THat12
        X = be_gemm("N", "N", -1.0, be_gemm("N", "N", 1.0, A[(s, fl)], Tinv[t][(f, f)], 0.0, None),
                    A[(fl, s)], 1.0, X)
        if t > 0:
            p = t - 1
            lp = len(doms[p]) - 1
            llp = doms[p][-1]
            X = be_gemm("N", "N", -1.0, be_gemm("N", "N", 1.0, A[(s, llp)], Tinv[p][(lp, lp)], 0.0, None),
                        A[(llp, s)], 1.0, X)
        S[(t, t)] = X
        if t < T - 1:
            sn = seps[t + 1]
            S[(t, t + 1)] = be_gemm("N", "N", -1.0, be_gemm("N", "N", 1.0, A[(s, fl)], Tinv[t][(f, l)], 0.0, None),
                                    A[(ll, sn)], 0.0, None)
            S[(t + 1, t)] = be_gemm("N", "N", -1.0, be_gemm("N", "N", 1.0, A[(sn, ll)], Tinv[t][(l, f)], 0.0, None),
                                    A[(fl, s)], 0.0, None)
    # 3. the Schur complement's tridiagonal inverse: RGF at the last level,
    #    else DDRGF one level down (matinvertndiag_ddrgf_core.jl:673-679)
    Sbm = BlockMatrix([M.blockSizes[s] for s in seps], {"in": 3, "out": 3}, False)
    Sbm.M = dict(S)
    if len(d1s) > 1:
        GS = bndiag_of_inv_ddrgf(Sbm, d1s[1:])[0].M
    else:
        GS = bndiag_of_inv_rgf_local(Sbm).M
    out = BlockMatrix(M.blockSizes, {"in": 3, "out": 3}, False)
    G = out.M
    for t in range(T):
        G[(seps[t], seps[t])] = GS[(t, t)]
    # 4. 12, 21 and 11 parts
    for t in range(T):
        d = doms[t]
        s = seps[t]
        nd = len(d)
        fl, ll = d[0], d[-1]
        has_next = t < T - 1
        sn = seps[t + 1] if has_next else None
        # B12[i] = -(T11inv T12 S^{-1})[i, sep_t], B12n[i] = ... [i, sep_{t+1}]
        a1 = [be_gemm("N", "N", 1.0, Tinv[t][(i, 0)], A[(fl, s)], 0.0, None) for i in range(nd)]
        a2 = [be_gemm("N", "N", 1.0, Tinv[t][(i, nd - 1)], A[(ll, sn)], 0.0, None) if has_next else None
              for i in range(nd)]
        B12, B12n = [], []
        for i in range(nd):
            x = be_gemm("N", "N", -1.0, a1[i], GS[(t, t)], 0.0, None)
            if has_next:
                x = be_gemm("N", "N", -1.0, a2[i], GS[(t + 1, t)], 1.0, x)
            B12.append(x)
            if has_next:
                y = be_gemm("N", "N", -1.0, a1[i], GS[(t, t + 1)], 0.0, None)
                y = be_gemm("N", "N", -1.0, a2[i], GS[(t + 1, t + 1)], 1.0, y)
                B12n.append(y)
        G[(fl, s)] = B12[0]
        if has_next:
            G[(ll, sn)] = B12n[nd - 1]
        # C21[j] = (T21 T11inv)[sep_t, j], C21n[j] = (T21 T11inv)[sep_{t+1}, j]
        C21 = [be_gemm("N", "N", 1.0, A[(s, fl)], Tinv[t][(0, j)], 0.0, None) for j in range(nd)]
        C21n = [be_gemm("N", "N", 1.0, A[(sn, ll)], Tinv[t][(nd - 1, j)], 0.0, None) if has_next else None
                for j in range(nd)]
        x = be_gemm("N", "N", -1.0, GS[(t, t)], C21[0], 0.0, None)
        if has_next:
            x = be_gemm("N", "N", -1.0, GS[(t, t + 1)], C21n[0], 1.0, x)
        G[(s, fl)] = x
        if has_next:
            y = be_gemm("N", "N", -1.0, GS[(t + 1, t)], C21[nd - 1], 0.0, None)
            y = be_gemm("N", "N", -1.0, GS[(t + 1, t + 1)], C21n[nd - 1], 1.0, y)
            G[(sn, ll)] = y
        for i in range(nd):
            for j in (i - 1, i, i + 1):
                if 0 <= j < nd:
                    x = Tinv[t][(i, j)].copy()
                    x = be_gemm("N", "N", -1.0, B12[i], C21[j], 1.0, x)
                    if has_next:
                        x = be_gemm("N", "N", -1.0, B12n[i], C21n[j], 1.0, x)
                    G[(d[i], d[j])] = x
    return out, S


# ---------------------------------------------------------------------------
# The reference's partition search (CPU cost model in units of one GEMM)

def cost_rgf(L, rLU, rMLDIV, do_full):
    """``cost_rgf`` (matinvertndiag_ddrgf_utils.jl:221-247)."""
    if do_full and L > 4:
        raise ValueError("a block tridiagonal matrix with L>4 is being fully inverted with RGF")
    n_full = 0
    if do_full and L == 3:
        n_full += 1 + 2
    elif do_full and L == 4:
        n_full += 3 + 6
    n_gemm = (L - 1) + 3 * (L - 1) + n_full
    n_mldiv = 2 * (L - 1) + 1 + (L - 1)
    return n_gemm + rLU * L + rMLDIV * n_mldiv


def cost_ddrgf(rLU, rMLDIV, nr_tasks, nr_threads, d1):
    """``cost_ddrgf`` (matinvertndiag_ddrgf_utils.jl:249-276)."""
    f = 1.0 / nr_threads
    c = f * nr_tasks * cost_rgf(d1, rLU, rMLDIV, True)
    c += 2.0 * f * 2 * nr_tasks * d1
    c += f * 4 * nr_tasks
    c += f * 4 * nr_tasks * d1
    c += f * 4 * nr_tasks
    c += f * nr_tasks * (4 * (d1 - 1) + 2 * d1)
    return c


def check_nr_threads(nr_threads, nr_tasks):
    """``bndiag_of_inv_ddrgf_check_nr_threads`` (matinvertndiag_ddrgf_utils.jl:455-465)."""
    while True:
        per = -(-nr_tasks // nr_threads)
        rest = nr_tasks - (nr_threads - 1) * per
        if rest > 0:
            return nr_threads, per, rest
        nr_threads -= 1


def opt_params(npl, rLU, rMLDIV, damp_rgf, nr_threads, max_levels=6, d1_max=4):
    """``opt_params`` (matinvertndiag_ddrgf_utils.jl:357-453): exhaustive search
    over per-level interior sizes d1 in {4, 3, 2, 1} for 1..6 levels, in the
    reference's enumeration order (Julia's ``Iterators.product``, first level
    fastest) with its strict-minimum tie rule and its pruning of level-1
    sizes below 4 once a finite cost is known.  Returns (nr_levels,
    nr_tasks_list, d1_list, cost)."""
    best = (0, [], [], float("inf"))
    for levels in range(1, max_levels + 1):
        arr = [d1_max] * levels
        while True:
            tasks_prev = npl
            nr_list, d1_list = [], []
            cost_new = cost_coarse = 0.0
            for lev in range(levels):
                d1 = arr[lev]
                if best[3] != float("inf") and lev == 0 and d1 < d1_max:
                    break
                cost_new -= cost_coarse
                nr, _ = get_nr_tasks(tasks_prev, d1)
                if nr == -1:
                    break
                tasks_prev = nr
                thr, _, _ = check_nr_threads(nr_threads, nr)
                cost_new += cost_ddrgf(rLU, rMLDIV, nr, thr, d1)
                cost_coarse = damp_rgf * cost_rgf(nr, rLU, rMLDIV, False)
                cost_new += cost_coarse
                nr_list.append(nr)
                d1_list.append(d1)
                if cost_new < best[3]:
                    best = (lev + 1, list(nr_list), list(d1_list), cost_new)
            # next combination: the first level varies fastest
            k = 0
            while k < levels:
                if arr[k] > 1:
                    arr[k] -= 1
                    break
                arr[k] = d1_max
                k += 1
            if k == levels:
                break
    return best


def levels_used(nr_levels, d1_list):
    """Interior sizes of the DDRGF levels that ``allocate_aux_data_DDRGF``
    (matinvertndiag_ddrgf_setup.jl:36-48) builds from ``opt_params``: one
    level for the finest grid, then one per coarse grid up to nr_levels - 1
    levels in all (at least one)."""
    return list(d1_list[:max(1, nr_levels - 1)])
