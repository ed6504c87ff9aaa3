"""Overlapped downloads (negf_solver_run_download): the G^R / G^< layers are
copied to pinned host memory while the rest of the pass runs; the outputs
equal those of run + download, for one device, an uneven batch (one pitched
copy per device group and layer), pageable buffers (the fallback) and the
one-call negf_solve (full chunks overlap, a partial last chunk does not)."""

import numpy as np
import pytest
import torch

from conftest import rel_fro
from oracle import physics as o_phys

pytestmark = pytest.mark.gpu


def _pinned(n):
    return torch.empty(n, dtype=torch.float64, pin_memory=True)


def _compare(solver, precision):
    lay, total = solver.layout()
    a = [_pinned(2 * total), _pinned(2 * total), _pinned(2 * solver.nE)]
    b = [_pinned(2 * total), _pinned(2 * total), _pinned(2 * solver.nE)]
    solver.run()
    solver.download(*(x.data_ptr() for x in a))
    for x in b:
        x.fill_(np.nan)
    solver.run_download(*(x.data_ptr() for x in b))
    for x, y in zip(a, b):
        # the same launches in the same order (graph against eager replay)
        assert torch.equal(x, y), float((x - y).abs().max())
    # pageable numpy buffers: the run-then-download fallback
    c = [np.full(2 * total, np.nan), np.full(2 * total, np.nan), np.full(2 * solver.nE, np.nan)]
    solver.run_download(*(x.ctypes.data for x in c))
    for x, y in zip(a, c):
        assert np.array_equal(x.numpy(), y)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_run_download_single_device(negf, precision):
    s = o_phys.physics_system(6, 64, seed=5)
    dev = negf.Device(s.Hd, s.Hu, s.sigL, s.sigR)
    solver = negf.Solver(dev, 8, eta=s.eta, precision=precision)
    solver.set_energies(np.linspace(-0.7, 0.7, 8))
    _compare(solver, precision)
    # and against the oracle
    lay, total = solver.layout()
    gr, gl, t2 = _pinned(2 * total), _pinned(2 * total), _pinned(16)
    solver.run_download(gr.data_ptr(), gl.data_ptr(), t2.data_ptr())
    per = sum(b * b for b in dev.sizes)
    g = gr.numpy().view(np.complex128)
    E = np.linspace(-0.7, 0.7, 8)
    tol = 1e-12 if precision == "fp64" else 1e-10
    for e in (0, 7):
        ref = o_phys.solve_energy(s, E[e])
        o = e * per
        for i, b in enumerate(dev.sizes):
            assert rel_fro(g[o:o + b * b].reshape(b, b, order="F"), ref["GR"].M[(i, i)]) < tol
            o += b * b
        assert abs(t2.numpy()[2 * e] - ref["T"]) <= tol * max(1.0, abs(ref["T"]))


def test_run_download_uneven_batch(negf):
    specs = [(4, 48, 3, 1), (7, [32, 40, 24, 32, 48, 16, 32], 2, 2), (9, 16, 4, 4)]
    devs, Es = [], []
    for npl, b, ne, seed in specs:
        sizes = b if isinstance(b, list) else None
        s = o_phys.physics_system(npl, b if sizes is None else 0, seed=seed, block_sizes=sizes)
        devs.append(negf.Device(s.Hd, s.Hu, s.sigL, s.sigR))
        Es.append(np.linspace(-0.8, 0.6, ne) + 0.01 * seed)
    solver = negf.BatchSolver(devs, [len(E) for E in Es])
    solver.set_energies(np.concatenate(Es))
    _compare(solver, "fp64")


def test_negf_solve_chunks_use_overlapped_downloads(negf):
    s = o_phys.physics_system(5, 32, seed=9)
    dev = negf.Device(s.Hd, s.Hu, s.sigL, s.sigR)
    E = np.linspace(-0.6, 0.6, 7)
    full = dev.solve(E, eta=s.eta)
    chunked = dev.solve(E, eta=s.eta, max_chunk=3)  # chunks of 3, 3 and 1
    for e in range(7):
        for i in range(5):
            assert rel_fro(chunked[0][e][i], full[0][e][i]) < 1e-13
            assert rel_fro(chunked[1][e][i], full[1][e][i]) < 1e-13
    assert np.allclose(chunked[2], full[2], rtol=1e-12, atol=0)
