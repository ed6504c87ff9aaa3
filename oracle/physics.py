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
    """Data of one device: H blocks, lead self-energies (constant, or a
    function of the energy) and optionally an overlap matrix S (diagonal
    blocks Sd, upper blocks Su; S = I when absent), so that
    M(E) = (E + i eta) S - H - Sigma(E) as the reference's build_M_from_HS
    (src/matloader.jl:89-95) forms it."""

    def __init__(self, Hd, Hu, sigL, sigR, eta=1e-6, muL=0.1, muR=-0.1, kT=0.025, Sd=None, Su=None, sigma_fn=None):
        self.Hd, self.Hu = Hd, Hu          # diagonal blocks, upper blocks H_{i,i+1}
        self.sigL, self.sigR = sigL, sigR
        self.eta, self.muL, self.muR, self.kT = eta, muL, muR, kT
        self.Sd, self.Su, self.sigma_fn = Sd, Su, sigma_fn

    def sig(self, E):
        """(Sigma_L(E), Sigma_R(E))."""
        return self.sigma_fn(E) if self.sigma_fn is not None else (self.sigL, self.sigR)

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
        sL, sR = self.sig(E)
        for i in range(n):
            S = self.Sd[i] if self.Sd is not None else np.eye(self.sizes[i])
            d = z * S - self.Hd[i]
            if i == 0:
                d = d - sL
            if i == n - 1:
                d = d - sR
            bm.M[(i, i)] = d
        for i in range(n - 1):
            up, lo = -self.Hu[i], -np.conj(self.Hu[i]).T
            if self.Su is not None:
                up = up + z * self.Su[i]
                lo = lo + z * np.conj(self.Su[i]).T
            bm.M[(i, i + 1)] = up
            bm.M[(i + 1, i)] = lo
        return bm

    def sigma_in(self, E):
        """Sigma^in(E) as a Hermitian BlockMatrix (diagonal + upper blocks)."""
        n = self.npl
        bm = BlockMatrix(self.sizes, {"in": 3, "out": 3}, True)
        for i in range(n):
            bm.M[(i, i)] = np.zeros((self.sizes[i], self.sizes[i]), dtype=np.complex128)
        for i in range(n - 1):
            bm.M[(i, i + 1)] = np.zeros((self.sizes[i], self.sizes[i + 1]), dtype=np.complex128)
        sL, sR = self.sig(E)
        bm.M[(0, 0)] = bm.M[(0, 0)] + self.fermi(E, self.muL) * self.gamma(sL)
        bm.M[(n - 1, n - 1)] = bm.M[(n - 1, n - 1)] + self.fermi(E, self.muR) * self.gamma(sR)
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


def with_overlap_and_sigma_of_E(sysm, seed=0):
    """The same device with an overlap matrix S = I + a small Hermitian band
    (positive definite) and energy-dependent lead self-energies
    Sigma(E) = (1 + 0.1 E) X - 0.05 i (1 + 0.5 sin 2E)(Y Y^H + 0.1 I)."""
    rng = np.random.default_rng(seed)
    sizes = sysm.sizes
    Sd, Su = [], []
    for b in sizes:
        A = _cn(rng, (b, b), 1.0) / np.sqrt(b)
        Sd.append(np.eye(b) + 0.02 * (A + np.conj(A).T))
    for i in range(len(sizes) - 1):
        Su.append(0.01 * _cn(rng, (sizes[i], sizes[i + 1]), 1.0) / np.sqrt(sizes[i]))

    def parts(n):
        B = _cn(rng, (n, n), 0.1)
        Y = _cn(rng, (n, n), 1.0) / np.sqrt(n)
        return (B + np.conj(B).T) / 2.0, Y @ np.conj(Y).T + 0.1 * np.eye(n)

    XL, PL = parts(sizes[0])
    XR, PR = parts(sizes[-1])

    def sigma_fn(E):
        g = 0.05 * (1.0 + 0.5 * np.sin(2.0 * E))
        return (1.0 + 0.1 * E) * XL - 1j * g * PL, (1.0 + 0.1 * E) * XR - 1j * g * PR

    return DeviceSystem(sysm.Hd, sysm.Hu, sysm.sigL, sysm.sigR, eta=sysm.eta, muL=sysm.muL, muR=sysm.muR,
                        kT=sysm.kT, Sd=Sd, Su=Su, sigma_fn=sigma_fn)


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
    sL, sR = sysm.sig(E)
    gL = sysm.gamma(sL)
    gR = sysm.gamma(sR)
    T = np.trace(gL @ g1 @ gR @ np.conj(g1).T)
    out["T"] = float(np.real(T))
    out["G1N"] = g1
    return out
