"""CPU tests: the oracle against the reference's own test oracles and the
committed golden fixtures; the DDRGF partition helper; the C ABI exports."""

import os
import re

import numpy as np
import pytest

from conftest import ROOT, rel_fro
from oracle import rgf, general_rgf, keldysh, selected_inverse, ddrgf, physics, direct
from oracle.blockmatrix import bm_convert_dense, band_of_dense, bm_from_dense, bm_fuse_to_tridiagonal
from oracle.generators import bm_create_synthetic_random, hermitian_random_like, set_sparse_block, full_of_blocks

GOLD = os.path.join(ROOT, "tests", "golden")
ROUNDOFF64 = 1e-15  # test/common_to_test.jl:25-27


def _gold(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


@pytest.mark.parametrize("npl,b", [(10, 32), (1, 7), (2, 5), (6, 17)])
def test_rgf_vs_dense(npl, b):
    M = bm_create_synthetic_random(npl, b, seed=npl)
    G = bm_convert_dense(rgf.bndiag_of_inv_rgf_local(M))
    ref = band_of_dense(np.linalg.inv(bm_convert_dense(M)), M.blockSizes, {"in": 3, "out": 3})
    assert rel_fro(G, ref) < ROUNDOFF64 * 1e3


def test_rgf_full_inverse_vs_dense():
    M = bm_create_synthetic_random(7, 12, seed=3)
    G = bm_convert_dense(rgf.bndiag_of_inv_rgf_local(M, build_full_inv=True))
    assert rel_fro(G, np.linalg.inv(bm_convert_dense(M))) < ROUNDOFF64 * 1e3


def test_keldysh_vs_dense():
    # test_keldyshndiag.jl:60-95
    M = bm_create_synthetic_random(10, 32, seed=1)
    S = hermitian_random_like(M, seed=2)
    Gn = bm_convert_dense(keldysh.keldyshndiag(M, S))
    Gr = np.linalg.inv(bm_convert_dense(M))
    bf = Gr @ bm_convert_dense(S) @ Gr.conj().T
    assert rel_fro(Gn, band_of_dense(bf, M.blockSizes, {"in": 3, "out": 3}, True)) < ROUNDOFF64 * 1e3


@pytest.mark.parametrize("nd", [5, 7])
def test_general_rgf_vs_dense_and_fused(nd):
    # test_matinvertndiag_general_rgf.jl and _fused.jl
    M = bm_create_synthetic_random(10, 32, seed=nd, ndiag=nd)
    G = bm_convert_dense(general_rgf.bndiag_of_inv_general_rgf(M))
    nd_ = {"in": nd, "out": nd}
    ref = band_of_dense(np.linalg.inv(bm_convert_dense(M)), M.blockSizes, nd_)
    assert rel_fro(G, ref) < ROUNDOFF64 * 1e3
    F = bm_fuse_to_tridiagonal(M)
    Gf = band_of_dense(bm_convert_dense(rgf.bndiag_of_inv_rgf_local(F)), M.blockSizes, nd_)
    assert rel_fro(G, Gf) < ROUNDOFF64 * 1e3


def test_selected_inverse_reference_cases():
    # test_selected_inverse.jl:6-55
    rind = [1, 1, 1, 2, 3, 3, 3, 4, 5]
    cind = [1, 3, 5, 2, 3, 4, 5, 4, 5]
    A = set_sparse_block([100] * 5, rind, cind, True, seed=0)
    F = full_of_blocks(selected_inverse.block_factorization(A, 5), [100] * 5)
    T = full_of_blocks(A, [100] * 5)
    import scipy.linalg as sl
    P, L, U = sl.lu(T)
    assert np.allclose(P, np.eye(500))
    assert rel_fro(F, np.tril(L, -1) + U) <= 1e-14
    assert rel_fro((np.tril(F, -1) + np.eye(500)) @ np.triu(F), T) <= 1e-14
    A1 = set_sparse_block([1] * 5, rind, cind, True, seed=1)
    Z = selected_inverse.block_inverse(selected_inverse.block_factorization(A1, 5), 5)
    T1 = full_of_blocks(A1, [1] * 5)
    invT = np.linalg.inv(T1)
    d = np.diag(T1 @ full_of_blocks(Z, [1] * 5))
    for (i, j), z in Z.items():
        assert abs(z[0, 0] - invT[i, j]) < 1e-13


@pytest.mark.parametrize("npl,d1", [(128, 15), (64, 15), (32, 6), (8, 1), (18, 3)])
def test_ddrgf_vs_sequential(npl, d1):
    # test_matinvertndiag_ddrgf.jl:245-293 (2.5e-10)
    b = 8 if npl > 60 else 16
    M = bm_create_synthetic_random(npl, b, seed=npl + d1)
    Gs = bm_convert_dense(rgf.bndiag_of_inv_rgf_local(M))
    Gp, S = ddrgf.bndiag_of_inv_ddrgf(M, d1)
    assert rel_fro(bm_convert_dense(Gp), Gs) < ROUNDOFF64 * 2.5e5


def test_ddrgf_schur_complement_exact():
    # test_matinvertndiag_ddrgf.jl:209-241: Schur complement vs exact
    M = bm_create_synthetic_random(20, 10, seed=5)
    D = bm_convert_dense(M)
    seps, doms, perm = ddrgf.partition(20, 4)
    off = M.offsets()
    idx = lambda layers: np.concatenate([np.arange(off[l], off[l + 1]) for l in layers])
    i2 = idx(seps)
    i1 = idx([l for d in doms for l in d])
    exact = D[np.ix_(i2, i2)] - D[np.ix_(i2, i1)] @ np.linalg.solve(D[np.ix_(i1, i1)], D[np.ix_(i1, i2)])
    _, S = ddrgf.bndiag_of_inv_ddrgf(M, 4)
    sb = [M.blockSizes[s] for s in seps]
    so = np.concatenate([[0], np.cumsum(sb)])
    approx = np.zeros_like(exact)
    for (t, u), blk in S.items():
        approx[so[t]:so[t + 1], so[u]:so[u + 1]] = blk
    assert rel_fro(approx, exact) < ROUNDOFF64 * 2.5e5


@pytest.mark.parametrize("npl,b,d1s", [(128, 6, [4, 3]), (64, 8, [3, 1, 1]), (40, 10, [3, 1, 2]), (128, 6, [7, 7])])
def test_ddrgf_multilevel_vs_sequential(npl, b, d1s):
    # the Schur complement recursion (matinvertndiag_ddrgf_core.jl:656-680):
    # every level's partition is possible, the result matches sequential RGF
    # at test_matinvertndiag_ddrgf.jl's tolerance (2.5e-10)
    n = npl
    for d1 in d1s:
        nr, _ = ddrgf.get_nr_tasks(n, d1)
        assert nr >= 2
        n = nr
    M = bm_create_synthetic_random(npl, b, seed=npl + sum(d1s))
    Gs = bm_convert_dense(rgf.bndiag_of_inv_rgf_local(M))
    Gp, _ = ddrgf.bndiag_of_inv_ddrgf(M, d1s)
    assert rel_fro(bm_convert_dense(Gp), Gs) < ROUNDOFF64 * 2.5e5


def test_ddrgf_cost_model_known_answers():
    # worked by hand from matinvertndiag_ddrgf_utils.jl:221-276, :357-465:
    # cost_rgf(3, full): 4*2 + 3 GEMMs + 2*3 LU + 1.5*7 solves = 27.5
    assert ddrgf.cost_rgf(3, 2.0, 1.5, True) == 27.5
    # cost_rgf(4, coarse): 12 GEMMs + 2*4 + 1.5*10 = 35
    assert ddrgf.cost_rgf(4, 2.0, 1.5, False) == 35.0
    # 4 tasks on 8 threads: check_nr_threads settles at 4 threads, 1 task each
    assert ddrgf.check_nr_threads(8, 4) == (4, 1, 1)
    assert ddrgf.check_nr_threads(3, 10) == (3, 4, 2)
    # npl = 16: D1 = 4 is impossible (get_nr_tasks = -1), D1 = 3 gives 4 tasks
    # at 73.5 + coarse 35 = 108.5; smaller level-1 sizes are pruned after that
    assert ddrgf.cost_ddrgf(2.0, 1.5, 4, 4, 3) == 73.5
    assert ddrgf.opt_params(16, 2.0, 1.5, 1.0, 8) == (1, [4], [3], 108.5)
    # allocate_aux_data_DDRGF builds max(1, nrLevels - 1) levels (setup.jl:36-48)
    assert ddrgf.levels_used(1, [3]) == [3]
    assert ddrgf.levels_used(2, [4, 3]) == [4]
    assert ddrgf.levels_used(4, [4, 1, 1, 2]) == [4, 1, 1]


def test_library_ddrgf_partition_search_matches_oracle():
    # host-only entry points: negf_ddrgf_opt_params against the oracle's
    # restatement; negf_ddrgf_choose_levels gives possible partitions
    import sys
    sys.path.insert(0, os.path.join(ROOT, "libnegf.jl_b200"))
    import libnegf_b200 as L
    for npl in list(range(2, 40)) + [64, 128, 500, 2048]:
        for thr in (1, 3, 8, 64):
            for r in ((2.0, 1.5, 1.0), (0.5, 3.0, 0.3), (7.0, 0.2, 4.0)):
                a = L.opt_params(npl, *r, nrThreads=thr)
                o = ddrgf.opt_params(npl, *r, thr)
                assert a[:3] == o[:3], (npl, thr, r)
                assert abs(a[3] - o[3]) <= 1e-12 * abs(o[3])
    for npl, b in ((64, 512), (128, 64), (1024, 32), (4096, 32), (7, 16)):
        n = npl
        d1s = L.choose_levels(npl, b)
        assert len(d1s) <= 6
        for d1 in d1s:
            nr, _ = ddrgf.get_nr_tasks(n, d1)
            assert nr >= 2
            n = nr
    assert L.choose_levels(4096, 32), "a long device with small blocks should decompose"


@pytest.mark.parametrize("npl,d1,expect", [(64, 15, (4, 0)), (128, 15, (8, 0)), (40, 6, (6, 4)), (17, 3, (-1, 0)),
                                           (18, 3, (5, 1)), (9, 1, (-1, 0)), (8, 1, (4, 0)), (10, 4, (2, 0)),
                                           (32, 6, (5, 3))])
def test_ddrgf_get_nr_tasks(npl, d1, expect):
    # matinvertndiag_ddrgf_utils.jl:278-312, worked by hand
    assert ddrgf.get_nr_tasks(npl, d1) == expect


def test_physics_oracle_vs_dense():
    sysm = physics.physics_system(5, 20, seed=3)
    for E in (-0.5, 0.25):
        r = physics.solve_energy(sysm, E)
        D = bm_convert_dense(sysm.M_of_E(E))
        Gi = np.linalg.inv(D)
        nd = {"in": 3, "out": 3}
        assert rel_fro(bm_convert_dense(r["GR"]), band_of_dense(Gi, sysm.sizes, nd)) < 1e-12
        Sin = bm_convert_dense(sysm.sigma_in(E))
        assert rel_fro(bm_convert_dense(r["Gn"]), band_of_dense(Gi @ Sin @ Gi.conj().T, sysm.sizes, nd, True)) < 1e-12
        b = sysm.sizes[0]
        g1n = Gi[:b, -b:]
        T = np.trace(sysm.gamma(sysm.sigL) @ g1n @ sysm.gamma(sysm.sigR) @ g1n.conj().T).real
        assert abs(r["T"] - T) < 1e-10 * max(1, abs(T))


# -- golden fixtures --------------------------------------------------------

def test_golden_rgf_keldysh():
    g = _gold("rgf_npl10_b32")
    M = bm_from_dense(g["M"], list(g["sizes"]), {"in": 3, "out": 3})
    assert rel_fro(bm_convert_dense(rgf.bndiag_of_inv_rgf_local(M)), g["G"]) < 1e-14
    k = _gold("keldysh_npl10_b32")
    S = bm_from_dense(k["S"], list(g["sizes"]), {"in": 3, "out": 3}, True)
    assert rel_fro(bm_convert_dense(keldysh.keldyshndiag(M, S)), k["Gn"]) < 1e-14


def test_golden_general_rgf():
    g = _gold("general_rgf_npl8_b24_n5")
    M = bm_from_dense(g["M"], list(g["sizes"]), {"in": 5, "out": 5})
    assert rel_fro(bm_convert_dense(general_rgf.bndiag_of_inv_general_rgf(M)), g["G"]) < 1e-14


def test_golden_selected_inverse():
    g = _gold("selinv_5x40")
    A = {}
    for (i, j) in g["pattern"]:
        blk = g["A"][i * 40:(i + 1) * 40, j * 40:(j + 1) * 40]
        if np.any(blk != 0):
            A[(int(i), int(j))] = blk
    F = selected_inverse.block_factorization(A, 5)
    assert rel_fro(full_of_blocks(F, [40] * 5).real, g["F"]) < 1e-14
    Z = selected_inverse.block_inverse(F, 5)
    assert rel_fro(full_of_blocks(Z, [40] * 5).real, g["Z"]) < 1e-14


def test_golden_ddrgf():
    g = _gold("ddrgf_npl24_b12_d6")
    M = bm_from_dense(g["M"], list(g["sizes"]), {"in": 3, "out": 3})
    G, _ = ddrgf.bndiag_of_inv_ddrgf(M, int(g["d1"]))
    assert rel_fro(bm_convert_dense(G), g["G"]) < 1e-14


def test_golden_negf():
    g = _gold("negf_npl6_b24")
    sysm = physics.DeviceSystem(list(g["Hd"]), list(g["Hu"]), g["sigL"], g["sigR"], eta=float(g["eta"]))
    for e, E in enumerate(g["E"]):
        r = physics.solve_energy(sysm, E)
        for i in range(6):
            assert rel_fro(r["GR"].M[(i, i)], g["GR"][e][i]) < 1e-14
            assert rel_fro(1j * r["Gn"].M[(i, i)], g["GL"][e][i]) < 1e-14
        assert abs(r["T"] - g["T"][e]) < 1e-13


# -- C ABI ------------------------------------------------------------------

def _declared_functions():
    src = open(os.path.join(ROOT, "include", "negf_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)
    skip = {"sizeof", "defined"}
    return sorted({n for n in names if (n.startswith("negf_") or n == "run_bndiag_wrapper") and n not in skip})


def test_library_exports_every_declared_symbol():
    import ctypes
    import sys
    sys.path.insert(0, os.path.join(ROOT, "libnegf.jl_b200"))
    from libnegf_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares a prototype for each of them
    assert set(names) <= set(_lib.PROTOTYPES), set(names) - set(_lib.PROTOTYPES)


def test_library_fails_loudly_without_device():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "libnegf.jl_b200"))
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import libnegf_b200
    lib = libnegf_b200.load()
    assert lib.negf_version() == 100
    with pytest.raises(libnegf_b200.NegfError):
        libnegf_b200._lib.check(lib.negf_probe_fp64_peak(None, None))


def test_oracle_overlap_and_energy_dependent_sigma_vs_dense():
    # M(E) = (E + i eta) S - H - Sigma(E) (build_M_from_HS, src/matloader.jl:89-95)
    from oracle import physics
    base = physics.physics_system(5, 12, seed=17)
    s = physics.with_overlap_and_sigma_of_E(base, seed=3)
    for E in (-0.4, 0.35):
        M = s.M_of_E(E)
        D = bm_convert_dense(M)
        G = np.linalg.inv(D)
        r = physics.solve_energy(s, E)
        off = np.cumsum([0] + s.sizes)
        Sin = bm_convert_dense(s.sigma_in(E))
        Gn = G @ Sin @ np.conj(G).T
        for i in range(5):
            blk = np.s_[off[i]:off[i + 1], off[i]:off[i + 1]]
            assert np.linalg.norm(r["GR"].M[(i, i)] - G[blk]) < 1e-11 * np.linalg.norm(G[blk])
            assert np.linalg.norm(r["Gn"].M[(i, i)] - Gn[blk]) < 1e-11 * np.linalg.norm(Gn[blk])
        sL, sR = s.sig(E)
        g1n = G[off[0]:off[1], off[4]:off[5]]
        T = np.real(np.trace(s.gamma(sL) @ g1n @ s.gamma(sR) @ np.conj(g1n).T))
        assert abs(T - r["T"]) < 1e-11 * max(1.0, abs(T))


def test_direct_oracle_band_and_outside_entries():
    # bndiag_of_inv_direct! (matinvertndiag_direct.jl:17-61): the out band of
    # inv(M) written into M; M's entries outside the band stay
    M = bm_create_synthetic_random(6, 8, seed=2, ndiag=5)
    D = bm_convert_dense(M)
    out, inv = direct.bndiag_of_inv_direct(D, M.blockSizes, {"in": 5, "out": 3})
    band = band_of_dense(inv, M.blockSizes, {"in": 3, "out": 3})
    assert np.array_equal(out[band != 0], band[band != 0])
    off = np.concatenate([[0], np.cumsum(M.blockSizes)])
    assert np.array_equal(out[0:off[1], off[2]:off[3]], D[0:off[1], off[2]:off[3]])
    # on a tridiagonal matrix the band agrees with sequential RGF
    T = bm_create_synthetic_random(6, 8, seed=3)
    out3, _ = direct.bndiag_of_inv_direct(bm_convert_dense(T), T.blockSizes, {"in": 3, "out": 3})
    assert rel_fro(out3, bm_convert_dense(rgf.bndiag_of_inv_rgf_local(T))) < 1e-12


def test_golden_ddrgf_multilevel():
    g = _gold("ddrgf_ml_npl40_b8")
    M = bm_from_dense(g["M"], list(g["sizes"]), {"in": 3, "out": 3})
    G, _ = ddrgf.bndiag_of_inv_ddrgf(M, [int(x) for x in g["d1"]])
    assert rel_fro(bm_convert_dense(G), g["G"]) < 1e-14
    exact = band_of_dense(np.linalg.inv(g["M"]), list(g["sizes"]), {"in": 3, "out": 3})
    assert rel_fro(g["G"], exact) < ROUNDOFF64 * 2.5e5


def test_golden_opt_params_grid():
    # the reference's search (matinvertndiag_ddrgf_utils.jl:357-453), frozen; the
    # library's restatement gives the same rows
    import sys
    sys.path.insert(0, os.path.join(ROOT, "libnegf.jl_b200"))
    import libnegf_b200 as L
    for row in _gold("ddrgf_opt_params_grid")["grid"]:
        npl, thr, rlu, rml, damp, lev, cost = int(row[0]), int(row[1]), row[2], row[3], row[4], int(row[5]), row[6]
        d1s = [int(x) for x in row[7:7 + lev]]
        tasks = [int(x) for x in row[13:13 + lev]]
        assert ddrgf.opt_params(npl, rlu, rml, damp, thr) == (lev, tasks, d1s, cost)
        a = L.opt_params(npl, rlu, rml, damp, nrThreads=thr)
        assert a[:3] == (lev, tasks, d1s) and abs(a[3] - cost) <= 1e-12 * cost


def test_golden_direct():
    g = _gold("direct_npl6_b8_in5_out3")
    sizes = [int(x) for x in g["sizes"]]
    R, inv = direct.bndiag_of_inv_direct(g["M"], sizes, {"in": 5, "out": 3})
    assert np.array_equal(R, g["R"])
    band = band_of_dense(np.ones_like(g["M"]), sizes, {"in": 3, "out": 3}) != 0
    assert np.array_equal(g["R"][~band], g["M"][~band])
    assert rel_fro(g["R"][band], np.linalg.inv(g["M"])[band]) < 1e-13


def test_golden_overlap_sigma_of_E():
    g = _gold("negf_overlap_sigmaE_npl5_b16")
    Es = list(g["E"])
    sig = {float(E): (g["sigL"][k], g["sigR"][k]) for k, E in enumerate(Es)}
    sysm = physics.DeviceSystem(list(g["Hd"]), list(g["Hu"]), g["sigL"][0], g["sigR"][0], eta=float(g["eta"]),
                                Sd=list(g["Sd"]), Su=list(g["Su"]), sigma_fn=lambda E: sig[float(E)])
    for k, E in enumerate(Es):
        r = physics.solve_energy(sysm, E)
        for i in range(5):
            assert rel_fro(r["GR"].M[(i, i)], g["GR"][k][i]) < 1e-14
            assert rel_fro(1j * r["Gn"].M[(i, i)], g["GL"][k][i]) < 1e-14
        assert abs(r["T"] - g["T"][k]) <= 1e-14 * max(1.0, abs(g["T"][k]))


# ---------------------------------------------------------------------------
# the double-double truth (oracle/ddtruth.py) used by the configuration parity tests

def test_ddtruth_products_and_inverse_are_exact_to_dd_level():
    from oracle import ddtruth as dd
    rng = np.random.default_rng(7)
    A = dd.DD(rng.standard_normal((48, 48)) + 1j * rng.standard_normal((48, 48)))
    X = dd.inv(A)
    R = dd.sub(dd.identity(48), dd.matmul(A, X))
    assert np.abs(R.hi).max() < 1e-28
    # a product of exactly representable integer matrices is exact
    B = dd.DD(np.round(64 * rng.standard_normal((48, 20))) + 1j * np.round(64 * rng.standard_normal((48, 20))))
    C = dd.DD(np.round(64 * rng.standard_normal((20, 30))) + 0j)
    P = dd.matmul(B, C)
    assert np.array_equal(P.hi, B.hi @ C.hi) and not np.any(P.lo)


@pytest.mark.parametrize("npl,b", [(5, 12), (1, 9), (3, 20)])
def test_ddtruth_vs_dense_and_oracle(npl, b):
    from oracle import ddtruth as dd
    sysm = physics.physics_system(npl, b, seed=npl + b)
    E = 0.21
    t = dd.physics_truth(sysm, E)
    r = physics.solve_energy(sysm, E)
    D = bm_convert_dense(sysm.M_of_E(E))
    Gd = np.linalg.inv(D)
    o = 0
    for i, bi in enumerate(sysm.sizes):
        assert rel_fro(t["GR"][i], Gd[o:o + bi, o:o + bi]) < 1e-13
        assert rel_fro(t["GR"][i], r["GR"].M[(i, i)]) < 1e-13
        assert rel_fro(t["GL"][i], 1j * r["Gn"].M[(i, i)]) < 1e-13
        o += bi
    assert abs(t["T"] - r["T"]) < 1e-12 * max(1.0, abs(r["T"]))
