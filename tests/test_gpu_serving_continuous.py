"""Continuous batching in the native request server (negf_server_*).

A request that arrives while another group is on the GPU is admitted at once
by a free lane (the HBM budget has room) and runs beside it on its own
stream: the server reports two groups in flight, and the small late request
completes before the large early one.  Its G^R / G^< diagonal blocks and T(E)
are the same alone and inside that mixed stream (same plan arithmetic per
(device, energy) item; bar 1e-13 relative Frobenius per block), for the FP64
and the mixed precision mode, and they match the oracle at the mode's bar
(1e-12 FP64, 1e-10 mixed).
"""

import time

import numpy as np
import pytest

from conftest import rel_fro
from oracle import physics as o_phys

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,bar", [("fp64", 1e-12), ("mixed", 1e-10)])
def test_same_alone_and_in_the_mix_and_overlap(negf, precision, bar):
    from libnegf_b200.server import NativeServer
    x = o_phys.physics_system(6, 64, seed=41)
    Ex = np.linspace(-0.6, 0.6, 5)
    big = o_phys.physics_system(24, 256, seed=42)
    Ebig = np.linspace(-0.9, 0.9, 48)
    others = [(o_phys.physics_system(n, b, seed=43 + k), np.linspace(-0.5, 0.4, ne))
              for k, (n, b, ne) in enumerate([(5, 32, 4), (9, 96, 3)])]

    srv = NativeServer(lanes=2, precision=precision, eta=x.eta)
    try:
        alone = srv.submit(x.Hd, x.Hu, x.sigL, x.sigR, Ex).wait(timeout=300)
        # the mix: a long request first, then x and two more while it runs
        tb = srv.submit(big.Hd, big.Hu, big.sigL, big.sigR, Ebig, want_blocks=False)
        time.sleep(0.05)
        tx = srv.submit(x.Hd, x.Hu, x.sigL, x.sigR, Ex)
        to = [srv.submit(s.Hd, s.Hu, s.sigL, s.sigR, E) for s, E in others]
        mixed = tx.wait(timeout=300)
        x_done = time.perf_counter()
        big_out = tb.wait(timeout=600)
        big_done = time.perf_counter()
        other_out = [t.wait(timeout=300) for t in to]
        st = srv.stats()
    finally:
        srv.close()

    assert st["peak_inflight_groups"] >= 2, st
    assert x_done < big_done  # admitted and finished while the long request was on the GPU
    for e in range(len(Ex)):
        for i in range(x.npl):
            assert rel_fro(mixed[0][e][i], alone[0][e][i]) < 1e-13
            assert rel_fro(mixed[1][e][i], alone[1][e][i]) < 1e-13
        assert abs(mixed[2][e] - alone[2][e]) <= 1e-13 * max(1.0, abs(alone[2][e]))
    for e, E in enumerate(Ex):
        r = o_phys.solve_energy(x, E)
        for i in range(x.npl):
            assert rel_fro(mixed[0][e][i], r["GR"].M[(i, i)]) < bar
            assert rel_fro(mixed[1][e][i], 1j * r["Gn"].M[(i, i)]) < bar
        assert abs(mixed[2][e] - r["T"]) <= bar * max(1.0, abs(r["T"]))
    for (s, E), out in zip(others, other_out):
        r = o_phys.solve_energy(s, E[0])
        for i in range(s.npl):
            assert rel_fro(out[0][0][i], r["GR"].M[(i, i)]) < bar
    for k in (0, len(Ebig) - 1):
        r = o_phys.solve_energy(big, Ebig[k], want_keldysh=False)
        assert abs(big_out[2][k] - r["T"]) <= bar * max(1.0, abs(r["T"]))


def test_one_lane_runs_one_group_at_a_time(negf):
    from libnegf_b200.server import NativeServer
    s = o_phys.physics_system(8, 128, seed=44)
    srv = NativeServer(lanes=1, eta=s.eta)
    try:
        ts = [srv.submit(s.Hd, s.Hu, s.sigL, s.sigR, np.linspace(-0.5, 0.5, 6)) for _ in range(3)]
        for t in ts:
            t.wait(timeout=300)
        st = srv.stats()
    finally:
        srv.close()
    assert st["peak_inflight_groups"] == 1 and st["requests"] == 3


def test_caller_output_buffers_and_cached_memory_release(negf):
    """Results delivered into caller-owned (here pinned) output arrays equal the
    default ones; handing the library's cached device chunks back to the driver
    leaves later solves unchanged."""
    import ctypes
    import torch
    from libnegf_b200.server import NativeServer
    x = o_phys.physics_system(6, 48, seed=41)
    E = np.linspace(-0.4, 0.4, 5)
    srv = NativeServer(lanes=2, precision="mixed", eta=x.eta)
    try:
        gr0, gl0, t0 = srv.submit(x.Hd, x.Hu, x.sigL, x.sigR, E).wait()
        n = len(E) * sum(h.shape[0] ** 2 for h in x.Hd)
        pg = torch.empty(n, dtype=torch.complex128, pin_memory=True)
        pl = torch.empty(n, dtype=torch.complex128, pin_memory=True)
        tt = np.empty(len(E))
        gr1, gl1, t1 = srv.submit(x.Hd, x.Hu, x.sigL, x.sigR, E, out=(pg.numpy(), pl.numpy(), tt)).wait()
        negf._lib.check(negf.load().negf_release_cached_memory())
        gr2, gl2, t2 = srv.submit(x.Hd, x.Hu, x.sigL, x.sigR, E).wait()
    finally:
        srv.close()
    for e in range(len(E)):
        for i in range(len(x.Hd)):
            assert np.array_equal(gr1[e][i], gr0[e][i]) and np.array_equal(gl1[e][i], gl0[e][i])
            assert np.array_equal(gr2[e][i], gr0[e][i]) and np.array_equal(gl2[e][i], gl0[e][i])
    assert np.array_equal(t1, t0) and np.array_equal(t2, t0)
    assert np.shares_memory(gr1[0][0], pg.numpy())
    with pytest.raises(ValueError):
        NativeServer.submit(srv, x.Hd, x.Hu, x.sigL, x.sigR, E, out=(pg.numpy()[:3], pl.numpy(), tt))
