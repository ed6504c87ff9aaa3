"""Uneven batches: one resident plan over devices of different layer counts
and (ragged) block sizes, several energies each, against the oracle per
device and energy.  The reference solves one system per call; this is its
RGF + RKD + transmission (src/matinvertndiag_rgf.jl:114-200,
src/keldyshndiag.jl:120-317) batched over systems."""

import numpy as np
import pytest

from conftest import rel_fro
from oracle import physics as o_phys

pytestmark = pytest.mark.gpu

SPECS = [  # (layers, block sizes or a uniform size, energies, seed)
    (4, 48, 3, 1),
    (7, [32, 40, 24, 32, 48, 16, 32], 2, 2),
    (2, 64, 2, 3),
    (9, 16, 4, 4),
]


def _systems():
    out = []
    for npl, b, ne, seed in SPECS:
        sizes = b if isinstance(b, list) else None
        s = o_phys.physics_system(npl, b if sizes is None else 0, seed=seed, block_sizes=sizes)
        out.append((s, np.linspace(-0.8, 0.6, ne) + 0.01 * seed))
    return out


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-10)])
def test_batch_solver_vs_oracle(negf, precision, tol):
    systems = _systems()
    devs = [negf.Device(s.Hd, s.Hu, s.sigL, s.sigR) for s, _ in systems]
    solver = negf.BatchSolver(devs, [len(E) for _, E in systems], eta=systems[0][0].eta, precision=precision)
    solver.set_energies(np.concatenate([E for _, E in systems]))
    for _ in range(2):  # the second pass replays the captured graph
        solver.run()
    solver.check()
    gr, gl, t = solver.host_outputs()
    for k, (s, Es) in enumerate(systems):
        for e, E in enumerate(Es):
            r = o_phys.solve_energy(s, E)
            for i in range(len(s.Hd)):
                assert rel_fro(gr[k][e][i], r["GR"].M[(i, i)]) < tol
                assert rel_fro(gl[k][e][i], 1j * r["Gn"].M[(i, i)]) < tol
            assert abs(t[k][e] - r["T"]) <= tol * max(1.0, abs(r["T"]))
    solver.close()
    for d in devs:
        d.close()


def test_batch_of_one_matches_single_solver(negf):
    s = o_phys.physics_system(5, 40, seed=9)
    E = np.linspace(-0.5, 0.5, 3)
    dev = negf.Device(s.Hd, s.Hu, s.sigL, s.sigR)
    a = negf.BatchSolver([dev], [3], eta=s.eta)
    a.set_energies(E)
    a.run()
    ga, la, ta = a.host_outputs()
    g1, l1, t1 = dev.solve(E, eta=s.eta)
    for e in range(3):
        for i in range(5):
            assert np.array_equal(ga[0][e][i], g1[e][i])
            assert np.array_equal(la[0][e][i], l1[e][i])
    assert np.array_equal(ta[0], t1)
    a.close()
    dev.close()
