"""Uneven batches through the scheduler (budget-packed groups, autotuned
knobs) and the request server, against the oracle."""

import numpy as np
import pytest

from conftest import rel_fro
from oracle import physics as o_phys

pytestmark = pytest.mark.gpu


def _systems(specs):
    return [o_phys.physics_system(npl, b, seed=seed) for npl, b, seed in specs]


def test_solve_uneven_small_budget_splits_and_matches(negf):
    from libnegf_b200.batch import bytes_per_energy, solve_uneven
    systems = _systems([(3, 32, 1), (6, 48, 2), (2, 160, 3), (5, 24, 4)])
    devs = [negf.Device(s.Hd, s.Hu, s.sigL, s.sigR) for s in systems]
    energies = [np.linspace(-0.7, 0.5, n) for n in (3, 2, 3, 4)]
    per = [bytes_per_energy(d, precision="fp64") for d in devs]
    budget = 2 * max(per)  # forces several groups and split devices
    got = {}

    def consume(solver, parts):
        gr, gl, t = solver.host_outputs()
        for j, (k, s, c) in enumerate(parts):
            for e in range(c):
                got[(k, s + e)] = (gr[j][e], gl[j][e], t[j][e])

    st = solve_uneven(devs, energies, budget_bytes=budget, on_group=consume, eta=systems[0].eta)
    assert st["groups"] > 1
    assert len(got) == sum(len(e) for e in energies)
    for k, s in enumerate(systems):
        for e, E in enumerate(energies[k]):
            r = o_phys.solve_energy(s, E)
            gr, gl, t = got[(k, e)]
            for i in range(len(s.Hd)):
                assert rel_fro(gr[i], r["GR"].M[(i, i)]) < 1e-12
                assert rel_fro(gl[i], 1j * r["Gn"].M[(i, i)]) < 1e-12
            assert abs(t - r["T"]) <= 1e-12 * max(1.0, abs(r["T"]))
    for d in devs:
        d.close()


def test_server_requests_of_different_sizes(negf):
    from libnegf_b200.server import NegfServer
    systems = _systems([(4, 32, 11), (3, 64, 12), (7, 16, 13)])
    energies = [np.linspace(-0.6, 0.6, n) for n in (5, 3, 6)]
    srv = NegfServer(precision="fp64", eta=systems[0].eta)
    try:
        reqs = [srv.submit(s.Hd, s.Hu, s.sigL, s.sigR, E, want_blocks=(k == 1))
                for k, (s, E) in enumerate(zip(systems, energies))]
        for r in reqs:
            r.wait(timeout=300)
        for k, (r, s, E) in enumerate(zip(reqs, systems, energies)):
            for e, En in enumerate(E):
                ref = o_phys.solve_energy(s, En)
                assert abs(r.t[e] - ref["T"]) <= 1e-12 * max(1.0, abs(ref["T"]))
                if k == 1:
                    for i in range(len(s.Hd)):
                        assert rel_fro(r.gr[e][i], ref["GR"].M[(i, i)]) < 1e-12
                        assert rel_fro(r.gl[e][i], 1j * ref["Gn"].M[(i, i)]) < 1e-12
        stats = srv.latency_stats()
        assert stats["requests"] == 3 and stats["p99_s"] >= stats["p50_s"] > 0
    finally:
        srv.close()


@pytest.mark.parametrize("budget_gb", [0.0, 1e-6])
def test_native_server_matches_oracle(negf, budget_gb):
    # negf_server_*: three requests of different shapes from the host; with the
    # default budget they share one batch plan, with a tiny one each request is
    # solved alone (through negf_solve)
    from libnegf_b200.server import NativeServer
    systems = _systems([(4, 32, 11), (6, 24, 12), (3, 48, 13)])
    energies = [np.linspace(-0.6, 0.5, n) for n in (3, 4, 2)]
    srv = NativeServer(budget_gb=budget_gb, eta=systems[0].eta)
    try:
        tickets = [srv.submit(s.Hd, s.Hu, s.sigL, s.sigR, E) for s, E in zip(systems, energies)]
        for s, E, tk in zip(systems, energies, tickets):
            gr, gl, t = tk.wait(timeout=120.0)
            assert tk.latency > 0.0
            for e, En in enumerate(E):
                r = o_phys.solve_energy(s, En)
                for i in range(s.npl):
                    assert rel_fro(gr[e][i], r["GR"].M[(i, i)]) < 1e-12
                    assert rel_fro(gl[e][i], 1j * r["Gn"].M[(i, i)]) < 1e-12
                assert abs(t[e] - r["T"]) <= 1e-12 * max(1.0, abs(r["T"]))
        st = srv.stats()
        assert st["requests"] == 3 and st["p99_s"] >= st["p50_s"] > 0.0
        # requests submitted while the worker is busy join one group; the first may go alone
        assert st["groups"] == 3 if budget_gb > 0.0 else 1 <= st["groups"] <= 3
    finally:
        srv.close()
