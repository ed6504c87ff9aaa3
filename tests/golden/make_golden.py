"""Generate the golden fixtures of the parity tests from the CPU oracle.

    python tests/golden/make_golden.py

Every fixture is a small seeded case (inputs + oracle outputs) saved as a
compressed .npz next to this script.  The oracle restates the reference's
LAPACK/BLAS call sequences (oracle/); the reference itself (Julia) cannot run
in this image.  The shapes and tolerances follow the reference's tests:
test_keldyshndiag.jl (npl=10, b~32), test_matinvertndiag_general_rgf*.jl
(npl=10, b~32, n=5), test_selected_inverse.jl (5 blocks, pattern rind/cind),
test_matinvertndiag_ddrgf.jl (sequential vs domain decomposed, one and several
levels; the partition search opt_params), test_matinvertndiag_direct.jl (the
dense path's output), and build_M_from_HS with an overlap matrix and
energy-dependent self-energies (matloader.jl:89-95).
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import rgf, general_rgf, keldysh, selected_inverse, ddrgf, physics, direct  # noqa: E402
from oracle.blockmatrix import bm_convert_dense  # noqa: E402
from oracle.generators import (bm_create_synthetic_random, hermitian_random_like, set_sparse_block,  # noqa: E402
                               full_of_blocks)

RIND = [1, 1, 1, 2, 3, 3, 3, 4, 5]
CIND = [1, 3, 5, 2, 3, 4, 5, 4, 5]


def cases():
    out = {}
    M = bm_create_synthetic_random(10, 32, seed=1234)
    out["rgf_npl10_b32"] = dict(sizes=np.array(M.blockSizes), M=bm_convert_dense(M),
                                G=bm_convert_dense(rgf.bndiag_of_inv_rgf_local(M)))
    S = hermitian_random_like(M, seed=4321)
    # the Keldysh fixture shares M with the RGF fixture
    out["keldysh_npl10_b32"] = dict(S=bm_convert_dense(S), Gn=bm_convert_dense(keldysh.keldyshndiag(M, S)))
    M5 = bm_create_synthetic_random(8, 24, seed=1234, ndiag=5)
    out["general_rgf_npl8_b24_n5"] = dict(sizes=np.array(M5.blockSizes), M=bm_convert_dense(M5),
                                           G=bm_convert_dense(general_rgf.bndiag_of_inv_general_rgf(M5)))
    A = set_sparse_block([40] * 5, RIND, CIND, True, seed=1234)
    F = selected_inverse.block_factorization(A, 5)
    Z = selected_inverse.block_inverse(F, 5)
    out["selinv_5x40"] = dict(A=full_of_blocks(A, [40] * 5, np.float64), F=full_of_blocks(F, [40] * 5).real,
                              Z=full_of_blocks(Z, [40] * 5).real,
                               pattern=np.array(sorted(Z.keys()), dtype=np.int32))
    Md = bm_create_synthetic_random(24, 12, seed=1234)
    Gd, _ = ddrgf.bndiag_of_inv_ddrgf(Md, 6)
    out["ddrgf_npl24_b12_d6"] = dict(sizes=np.array(Md.blockSizes), M=bm_convert_dense(Md), d1=np.array(6),
                                     G=bm_convert_dense(Gd))
    sysm = physics.physics_system(6, 24, seed=0)
    Es = np.array([-0.6, 0.0, 0.3, 0.7])
    gr, gl, T = [], [], []
    for E in Es:
        r = physics.solve_energy(sysm, E)
        gr.append(np.stack([r["GR"].M[(i, i)] for i in range(6)]))
        gl.append(np.stack([1j * r["Gn"].M[(i, i)] for i in range(6)]))
        T.append(r["T"])
    out["negf_npl6_b24"] = dict(Hd=np.stack(sysm.Hd), Hu=np.stack(sysm.Hu), sigL=sysm.sigL, sigR=sysm.sigR,
                                E=Es, eta=np.array(sysm.eta), GR=np.stack(gr), GL=np.stack(gl), T=np.array(T))
    # DDRGF over three levels: 40 layers -> 10 separators -> 5 -> 2 (+ RGF)
    Mm = bm_create_synthetic_random(40, 8, seed=77)
    Gm, _ = ddrgf.bndiag_of_inv_ddrgf(Mm, [3, 1, 2])
    out["ddrgf_ml_npl40_b8"] = dict(sizes=np.array(Mm.blockSizes), M=bm_convert_dense(Mm), d1=np.array([3, 1, 2]),
                                    G=bm_convert_dense(Gm))
    # the reference's partition search on a grid of layer counts / threads / ratios
    grid = []
    for npl in (16, 32, 64, 128, 500):
        for thr in (1, 8, 64):
            for r in ((2.0, 1.5, 1.0), (0.5, 3.0, 0.3)):
                lev, tasks, d1s, cost = ddrgf.opt_params(npl, r[0], r[1], r[2], thr)
                row = [npl, thr, r[0], r[1], r[2], lev, cost] + d1s + [0] * (6 - len(d1s)) + tasks + \
                    [0] * (6 - len(tasks))
                grid.append(row)
    out["ddrgf_opt_params_grid"] = dict(grid=np.array(grid, dtype=np.float64))
    # the dense path: pentadiagonal input, tridiagonal output (entries outside the band stay)
    Mp = bm_create_synthetic_random(6, 8, seed=2, ndiag=5)
    Dp = bm_convert_dense(Mp)
    res, _ = direct.bndiag_of_inv_direct(Dp, Mp.blockSizes, {"in": 5, "out": 3})
    out["direct_npl6_b8_in5_out3"] = dict(sizes=np.array(Mp.blockSizes), M=Dp, R=res)
    # overlap S and Sigma(E): M(E) = (E + i eta) S - H - Sigma(E)
    base = physics.physics_system(5, 16, seed=23)
    full = physics.with_overlap_and_sigma_of_E(base, seed=5)
    Es = np.array([-0.5, 0.2, 0.6])
    gr, gl, T, sl, sr = [], [], [], [], []
    for E in Es:
        r = physics.solve_energy(full, E)
        gr.append(np.stack([r["GR"].M[(i, i)] for i in range(5)]))
        gl.append(np.stack([1j * r["Gn"].M[(i, i)] for i in range(5)]))
        T.append(r["T"])
        a, b = full.sigma_fn(E)
        sl.append(a)
        sr.append(b)
    out["negf_overlap_sigmaE_npl5_b16"] = dict(Hd=np.stack(base.Hd), Hu=np.stack(base.Hu), Sd=np.stack(full.Sd),
                                               Su=np.stack(full.Su), sigL=np.stack(sl), sigR=np.stack(sr), E=Es,
                                               eta=np.array(base.eta), GR=np.stack(gr), GL=np.stack(gl),
                                               T=np.array(T))
    return out


def main():
    for name, arrs in cases().items():
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
        print("wrote", name)


if __name__ == "__main__":
    main()
