"""Seeded NEGF device systems and the per-energy G^R / G^< / transmission oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

The reference has no energy loop, self-energy, Fermi function or transmission;
they are built here from their textbook definitions on top of the reference's
own RGF (``rgf.py``) and RKD (``keldysh.py``) restatements, so their parity is
the dense-inverse cross-check only.

Generator (all draws from ``numpy.random.default_rng(seed)``, in this order):
* H_ii = (A + A^H)/2, A complex normal with E|a|^2 = 1, divided by sqrt(b);
* H_{i,i+1} complex normal with E|h|^2 = 0.25, divided by sqrt(b); H_{i+1,i} = H_{i,i+1}^H;
* Sigma_{L/R} = X - 0.05 i (Y Y^H + 0.1 I), X = (B + B^H)/2 with B complex normal
  of E|x|^2 = 0.1, Y complex normal of E|y|^2 = 1 divided by sqrt(b);
* M(E) = (E + i eta) I - H - Sigma (Sigma_L on layer 0, Sigma_R on layer N-1);
* Gamma = i (Sigma - Sigma^H), Sigma^in = f Gamma with the Fermi function
  f(E) = 1 / (1 + exp((E - mu)/kT)); G^< = i G^n with G^n = G^R Sigma^in G^A.
"""

import numpy as np

from .blockmatrix import BlockMatrix
from . import rgf as _rgf
from . import keldysh as _keldysh
from .backend_cpu import be_gemm


def _cn(rng, shape, var):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * np.sqrt(var / 2.0)


class DeviceSystem:
    """Energy-independent data of one device: H blocks and lead self-energies."""

    def __init__(self, Hd, Hu, sigL, sigR, eta=1e-6, muL=0.1, muR=-0.1, kT=0.025):
        self.Hd, self.Hu = Hd, Hu          # diagonal blocks, upper blocks H_{i,i+1}
        self.sigL, self.sigR = sigL, sigR
        self.eta, self.muL, self.muR, self.kT = eta, muL, muR, kT

    @property
    def npl(self):
        return len(self.Hd)

    @property
    def sizes(self):
        return [h.shape[0] for h in self.Hd]

    def gamma(self, sig):
        return 1j * (sig - np.conj(sig).T)

    def fermi(self, E, mu):
        return 1.0 / (1.0 + np.exp((E - mu) / self.kT))

    def M_of_E(self, E):
        """M(E) as a block-tridiagonal BlockMatrix."""
        n = self.npl
        bm = BlockMatrix(self.sizes, {"in": 3, "out": 3}, False)
        z = E + 1j * self.eta
        for i in range(n):
            d = z * np.eye(self.sizes[i]) - self.Hd[i]
            if i == 0:
                d = d - self.sigL
            if i == n - 1:
                d = d - self.sigR
            bm.M[(i, i)] = d
        for i in range(n - 1):
            bm.M[(i, i + 1)] = -self.Hu[i]
            bm.M[(i + 1, i)] = -np.conj(self.Hu[i]).T
        return bm

    def sigma_in(self, E):
        """Sigma^in(E) as a Hermitian BlockMatrix (diagonal + upper blocks)."""
        n = self.npl
        bm = BlockMatrix(self.sizes, {"in": 3, "out": 3}, True)
        for i in range(n):
            bm.M[(i, i)] = np.zeros((self.sizes[i], self.sizes[i]), dtype=np.complex128)
        for i in range(n - 1):
            bm.M[(i, i + 1)] = np.zeros((self.sizes[i], self.sizes[i + 1]), dtype=np.complex128)
        bm.M[(0, 0)] = bm.M[(0, 0)] + self.fermi(E, self.muL) * self.gamma(self.sigL)
        bm.M[(n - 1, n - 1)] = bm.M[(n - 1, n - 1)] + self.fermi(E, self.muR) * self.gamma(self.sigR)
        return bm


def physics_system(npl, b, seed=0, eta=1e-6, block_sizes=None):
    rng = np.random.default_rng(seed)
    sizes = block_sizes if block_sizes is not None else [int(b)] * npl
    Hd, Hu = [], []
    for i in range(npl):
        A = _cn(rng, (sizes[i], sizes[i]), 1.0) / np.sqrt(sizes[i])
        Hd.append((A + np.conj(A).T) / 2.0)
    for i in range(npl - 1):
        Hu.append(_cn(rng, (sizes[i], sizes[i + 1]), 0.25) / np.sqrt(sizes[i]))

    def sig(n):
        B = _cn(rng, (n, n), 0.1)
        X = (B + np.conj(B).T) / 2.0
        Y = _cn(rng, (n, n), 1.0) / np.sqrt(n)
        return X - 0.05j * (Y @ np.conj(Y).T + 0.1 * np.eye(n))

    sigL = sig(sizes[0])
    sigR = sig(sizes[-1])
    return DeviceSystem(Hd, Hu, sigL, sigR, eta=eta)


def energy_grid(n, lo=-1.0, hi=1.0):
    return np.linspace(lo, hi, n)


def solve_energy(sysm, E, want_keldysh=True):
    """One energy point through the reference algorithms: G^R tridiagonal by
    RGF, G^n by RKD, transmission from G^R_{1N}.

    Returns dict with 'GR' (BlockMatrix), 'Gn' (Hermitian BlockMatrix, or None)
    and 'T' (float)."""
    M = sysm.M_of_E(E)
    # one upward pass shared by G^R, G^n and the transmission chain
    up = _rgf.rgf_upward(M)
    lu, R, L = up
    GR = _rgf.bndiag_of_inv_rgf_local(M, upward=up)
    out = {"GR": GR}
    if want_keldysh:
        out["Gn"] = _keldysh.keldyshndiag(M, sysm.sigma_in(E), upward=up)
    # G^R_{1N} by the row recursion G_{1,j} = -G_{1,j-1} R_{j-1} (rgf.jl:185-199)
    g1 = GR.M[(0, 0)]
    for j in range(1, sysm.npl):
        g1 = be_gemm("N", "N", -1.0, g1, R[j - 1], 0.0, None)
    gL = sysm.gamma(sysm.sigL)
    gR = sysm.gamma(sysm.sigR)
    T = np.trace(gL @ g1 @ gR @ np.conj(g1).T)
    out["T"] = float(np.real(T))
    out["G1N"] = g1
    return out
