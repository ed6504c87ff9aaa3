"""Double-double ("dd") truth for the NEGF parity tests.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Why: at the benchmark configuration (N = 32 layers of b = 256, kappa(M) ~ 1e4)
every FP64 algorithm -- the reference's LAPACK call sequence restated in
``rgf.py`` / ``keldysh.py`` and the GPU path alike -- is ~u kappa ~ 1e-12 from
the exact inverse, so comparing the GPU with the oracle alone cannot say which
of the two carries the error.  This module computes the same outputs with
~100-bit arithmetic so that both can be measured against a value whose own
error is far below theirs.

Representation: a matrix is a pair (hi, lo) of complex128 arrays whose value is
hi + lo (|lo| <= ulp(hi) / 2 after normalisation).  Products are formed with
the error-free splitting of Ozaki et al. ("Error-free transformations of
matrix multiplication by using fast routines of matrix multiplication", 2012):
each operand row (left) or column (right) is cut into slices whose entries are
small integers times a per-row power of two, so that every slice product is
computed EXACTLY by an ordinary complex128 BLAS GEMM; the exact slice products
are summed in dd.  Inverses are refined from an FP64 inverse by two Newton
steps X <- X + X (I - A X) in dd.

The math follows the definitions, not the reference's call order (it is an
independent third opinion, not a restatement):
* G^R = M^{-1}: right-connected g_i = (M_ii - M_{i,i+1} g_{i+1} M_{i+1,i})^{-1},
  then the tridiagonal blocks by the downward recursion
  (src/matinvertndiag_rgf.jl:114-200 computes the same quantities);
* G^n = G^R Sigma^in G^A with Sigma^in non-zero on the first and last layer
  only: G^n_ii = C_i S_L C_i^H + D_i S_R D_i^H with the first block column
  C_i = G_{i,0} and the last block column D_i = G_{i,N-1} of G^R
  (src/keldyshndiag.jl:120-317 computes the same blocks recursively);
* T = Re Tr[Gamma_L G_{0,N-1} Gamma_R G_{0,N-1}^H].
"""

import math

import numpy as np

_SPLITTER = 134217729.0  # 2^27 + 1 (Veltkamp)
_NSLICE = 4              # slices per operand; pairs s + t <= 3 are formed


class DD:
    """hi + lo, both complex128 arrays of one shape."""

    __slots__ = ("hi", "lo")

    def __init__(self, hi, lo=None):
        self.hi = np.asarray(hi, dtype=np.complex128)
        self.lo = np.zeros_like(self.hi) if lo is None else np.asarray(lo, dtype=np.complex128)

    @property
    def H(self):
        return DD(np.conj(self.hi).T, np.conj(self.lo).T)

    def value(self):
        """The FP64 rounding of hi + lo."""
        return self.hi + self.lo


def _two_sum(a, b):
    s = a + b
    bp = s - a
    return s, (a - (s - bp)) + (b - bp)


def _fast_two_sum(a, b):
    s = a + b
    return s, b - (s - a)


def add(a, b):
    s, e = _two_sum(a.hi, b.hi)
    e = e + (a.lo + b.lo)
    return DD(*_fast_two_sum(s, e))


def neg(a):
    return DD(-a.hi, -a.lo)


def sub(a, b):
    return add(a, neg(b))


def _split_real(x):
    c = _SPLITTER * x
    hi = c - (c - x)
    return hi, x - hi


def _two_prod_real(a, b):
    p = a * b
    ah, al = _split_real(a)
    bh, bl = _split_real(b)
    return p, ((ah * bh - p) + ah * bl + al * bh) + al * bl


def scale(a, f):
    """a times a real FP64 scalar f, in dd."""
    f = float(f)
    pr, er = _two_prod_real(a.hi.real, f)
    pi, ei = _two_prod_real(a.hi.imag, f)
    e = (er + 1j * ei) + a.lo * f
    return DD(*_fast_two_sum(pr + 1j * pi, e))


def times_i(a):
    """i a (exact)."""
    return DD(1j * a.hi, 1j * a.lo)


def identity(n):
    return DD(np.eye(n, dtype=np.complex128))


def _slice_bits(k):
    # entries of a slice are integers of magnitude <= 2^(beta-1); the real
    # (or imaginary) part of one complex dot product of length k is a sum of
    # 2k such products, exact in FP64 while k 2^(2 beta - 1) <= 2^53
    return max(8, (53 - int(math.ceil(math.log2(max(k, 2))))) // 2)


def _slices(x, axis, beta):
    """x = sum of _NSLICE slices (plus a remainder below 2^(e - 4 beta)
    relative to the row / column maximum 2^e); slice s holds integers of
    magnitude <= 2^(beta-1) times 2^(e + 1 - beta (s + 1)) along `axis`."""
    mu = np.maximum(np.abs(x.real), np.abs(x.imag)).max(axis=axis, keepdims=True)
    e = np.zeros_like(mu)
    nz = mu > 0
    e[nz] = np.ceil(np.log2(mu[nz]))
    out = []
    r = x.copy()
    for s in range(_NSLICE):
        u = np.exp2(e + 1 - beta * (s + 1))
        t = np.rint(r.real / u) * u + 1j * (np.rint(r.imag / u) * u)
        out.append(t)
        r = r - t  # exact
    return out


def matmul(a, b):
    """dd product a b (a: m x k, b: k x n), accurate to ~2^-84 relative to |a| |b|."""
    k = a.hi.shape[1]
    beta = _slice_bits(k)
    sa = _slices(a.hi, 1, beta)
    sb = _slices(b.hi, 0, beta)
    hi = None
    lo = None
    for s in range(_NSLICE):
        for t in range(_NSLICE - s):
            p = sa[s] @ sb[t]  # exact
            if hi is None:
                hi, lo = p, np.zeros_like(p)
            else:
                hi, e = _two_sum(hi, p)
                lo = lo + e
    lo = lo + (a.hi @ b.lo + a.lo @ b.hi)
    return DD(*_fast_two_sum(hi, lo))


def inv(a, steps=2):
    """a^{-1} by Newton refinement of the FP64 inverse of a.hi."""
    n = a.hi.shape[0]
    x = DD(np.linalg.inv(a.hi))
    eye = identity(n)
    for _ in range(steps):
        r = sub(eye, matmul(a, x))
        x = add(x, matmul(x, r))
    return x


def tri_inverse(Md, Mu, Ml, SinL=None, SinR=None, GammaL=None, GammaR=None):
    """Selected blocks of G^R = M^{-1} (and of G^n) for a block-tridiagonal M.

    Md[i] = M[i,i], Mu[i] = M[i,i+1], Ml[i] = M[i+1,i] as DD.  With SinL / SinR
    (DD, the Sigma^in blocks on the first / last layer) G^n's diagonal blocks
    are formed; with GammaL / GammaR (DD) the transmission.

    Returns a dict of FP64 blocks: 'd' (G^R_ii), 'u' (G^R_{i,i+1}),
    'l' (G^R_{i+1,i}), 'Gn' (G^n_ii, when requested), 'T' (when requested)."""
    n = len(Md)
    g = [None] * n
    R = [None] * n
    L = [None] * n
    g[n - 1] = inv(Md[n - 1])
    for i in range(n - 2, -1, -1):
        R[i] = matmul(Mu[i], g[i + 1])
        L[i + 1] = matmul(g[i + 1], Ml[i])
        g[i] = inv(sub(Md[i], matmul(Mu[i], L[i + 1])))
    d = [None] * n
    u = [None] * (n - 1)
    lo = [None] * (n - 1)
    d[0] = g[0]
    for i in range(1, n):
        u[i - 1] = neg(matmul(d[i - 1], R[i - 1]))
        lo[i - 1] = neg(matmul(L[i], d[i - 1]))
        d[i] = sub(g[i], matmul(L[i], u[i - 1]))
    out = {"d": [x.value() for x in d], "u": [x.value() for x in u], "l": [x.value() for x in lo]}
    want_gn = SinL is not None or SinR is not None
    want_t = GammaL is not None and GammaR is not None
    if not (want_gn or want_t):
        return out
    # first block column C_i = G_{i,0}: C_0 = G_00, C_i = -L_i C_{i-1}
    C = [d[0]]
    for i in range(1, n):
        C.append(neg(matmul(L[i], C[i - 1])))
    # last block column D_i = G_{i,N-1} = G_ii Q_i, Q_{N-1} = I, Q_i = -R_i Q_{i+1}
    Q = [None] * n
    Q[n - 1] = identity(Md[n - 1].hi.shape[0])
    for i in range(n - 2, -1, -1):
        Q[i] = neg(matmul(R[i], Q[i + 1]))
    D = [matmul(d[i], Q[i]) if i < n - 1 else d[n - 1] for i in range(n)]
    if want_gn:
        gn = []
        for i in range(n):
            acc = None
            if SinL is not None:
                acc = matmul(matmul(C[i], SinL), C[i].H)
            if SinR is not None:
                t = matmul(matmul(D[i], SinR), D[i].H)
                acc = t if acc is None else add(acc, t)
            gn.append(acc.value())
        out["Gn"] = gn
    if want_t:
        t = matmul(matmul(matmul(GammaL, D[0]), GammaR), D[0].H)
        out["T"] = float(np.real(np.trace(t.hi) + np.trace(t.lo)))
    return out


def physics_truth(sysm, E, want_keldysh=True):
    """Truth of one energy point of an ``oracle.physics.DeviceSystem`` (no
    overlap matrix, constant self-energies): M(E) = (E + i eta) I - H - Sigma
    formed exactly in dd from the FP64 inputs, then ``tri_inverse``.

    Returns {'GR': [G^R_ii], 'GRu', 'GRl', 'GL': [G^<_ii = i G^n_ii], 'T'}."""
    if sysm.Sd is not None or sysm.sigma_fn is not None:
        raise ValueError("physics_truth covers the plain generator (S = I, constant Sigma)")
    n = sysm.npl
    z = complex(E, sysm.eta)
    sL, sR = sysm.sigL, sysm.sigR
    Md = []
    for i in range(n):
        m = neg(DD(sysm.Hd[i]))
        if i == 0:
            m = sub(m, DD(sL))
        if i == n - 1:
            m = sub(m, DD(sR))
        zi = DD(np.zeros_like(m.hi))
        np.fill_diagonal(zi.hi, z)
        Md.append(add(m, zi))
    Mu = [neg(DD(h)) for h in sysm.Hu]
    Ml = [neg(DD(np.conj(h).T)) for h in sysm.Hu]

    def gamma(s):  # i (S - S^H), exact
        return times_i(sub(DD(s), DD(np.conj(s).T)))

    gL, gR = gamma(sL), gamma(sR)
    kw = {"GammaL": gL, "GammaR": gR}
    if want_keldysh:
        kw["SinL"] = scale(gL, sysm.fermi(E, sysm.muL))
        kw["SinR"] = scale(gR, sysm.fermi(E, sysm.muR))
    r = tri_inverse(Md, Mu, Ml, **kw)
    out = {"GR": r["d"], "GRu": r["u"], "GRl": r["l"], "T": r["T"]}
    if want_keldysh:
        out["GL"] = [1j * x for x in r["Gn"]]
    return out


def block_truth(Md, Mu, Ml):
    """Truth of the G^R tridiagonal of a block-tridiagonal matrix given by its
    FP64 blocks (the reference-API sweeps' input)."""
    return tri_inverse([DD(x) for x in Md], [DD(x) for x in Mu], [DD(x) for x in Ml])
