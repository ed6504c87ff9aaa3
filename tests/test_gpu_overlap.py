"""Non-orthogonal bases and energy-dependent self-energies: M(E) =
(E + i eta) S - H - Sigma(E) assembled per energy on the device (the
reference's build_M_from_HS, src/matloader.jl:89-95), through RGF + RKD +
transmission, against the oracle."""

import numpy as np
import pytest

from conftest import rel_fro
from oracle import physics as o_phys

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("overlap,sigma_e,precision,tol", [
    (True, False, "fp64", 1e-12), (False, True, "fp64", 1e-12), (True, True, "fp64", 1e-12),
    (True, True, "mixed", 1e-10)])
def test_overlap_and_sigma_of_E(negf, overlap, sigma_e, precision, tol):
    base = o_phys.physics_system(6, 40, seed=23)
    full = o_phys.with_overlap_and_sigma_of_E(base, seed=5)
    ref_sys = o_phys.DeviceSystem(base.Hd, base.Hu, base.sigL, base.sigR, eta=base.eta,
                                  Sd=full.Sd if overlap else None, Su=full.Su if overlap else None,
                                  sigma_fn=full.sigma_fn if sigma_e else None)
    dev = negf.Device(base.Hd, base.Hu, base.sigL, base.sigR)
    if overlap:
        dev.set_overlap(full.Sd, full.Su)
    Es = np.linspace(-0.7, 0.6, 4)
    solver = negf.Solver(dev, len(Es), eta=base.eta, precision=precision, sigma_per_energy=sigma_e)
    solver.set_energies(Es)
    if sigma_e:
        sig = [full.sigma_fn(E) for E in Es]
        solver.set_self_energies([s[0] for s in sig], [s[1] for s in sig])
    solver.run()
    solver.run()  # graph replay: the per-energy assembly reruns from the inputs
    solver.check()
    gr, gl, t = solver.host_outputs()
    for e, E in enumerate(Es):
        r = o_phys.solve_energy(ref_sys, E)
        for i in range(6):
            assert rel_fro(gr[0][e][i], r["GR"].M[(i, i)]) < tol
            assert rel_fro(gl[0][e][i], 1j * r["Gn"].M[(i, i)]) < tol
        assert abs(t[0][e] - r["T"]) <= tol * max(1.0, abs(r["T"]))
    solver.close()
    dev.close()


def test_identity_overlap_matches_plain_path(negf):
    s = o_phys.physics_system(4, 32, seed=29)
    E = np.linspace(-0.5, 0.5, 3)
    dev = negf.Device(s.Hd, s.Hu, s.sigL, s.sigR)
    g0, l0, t0 = dev.solve(E, eta=s.eta)
    dev.set_overlap()  # S = I
    g1, l1, t1 = dev.solve(E, eta=s.eta)
    for e in range(3):
        for i in range(4):
            # same mathematics, different rounding order (explicit lower blocks)
            assert rel_fro(g1[e][i], g0[e][i]) < 1e-12
            assert rel_fro(l1[e][i], l0[e][i]) < 1e-12
    assert np.allclose(t1, t0, rtol=1e-12, atol=1e-14)
    dev.close()
