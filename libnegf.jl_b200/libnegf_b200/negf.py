"""Batched-energy NEGF solves on the B200 library.

The reference computes one energy point per call (RGF for G^R, RKD for G^n);
here a ``Device`` keeps H, Sigma_L, Sigma_R resident on the GPU and a
``Solver`` runs RGF + RKD + transmission for a whole list of energies in one
replayed launch sequence (CUDA graph).

Physics: M(E) = (E + i eta) I - H - Sigma (Sigma_L on layer 0, Sigma_R on layer
N-1), Gamma = i (Sigma - Sigma^H), Sigma^in = f_L Gamma_L (+) f_R Gamma_R with
Fermi functions at mu_L / mu_R and temperature kT, G^< = i G^R Sigma^in G^A,
T(E) = Re Tr[Gamma_L G^R_{1N} Gamma_R G^A_{N1}].
"""

import ctypes

import numpy as np

from . import _lib
from ._lib import check, load, ptr_array, int_array


def _host_blocks(blocks):
    """Keep column-major complex128 copies alive and return their addresses."""
    keep = [np.asfortranarray(np.asarray(b, dtype=np.complex128)) for b in blocks]
    return keep, [k.ctypes.data for k in keep]


def make_opts(eta=1e-6, mu_l=0.1, mu_r=-0.1, kT=0.025, want_gr=True, want_gl=True, want_t=True, max_chunk=0,
              hbm_budget_gb=0.0, precision="fp64", gemm_form=0, gj_nb=0, sigma_per_energy=False, gj_update=0):
    """precision: "fp64" (every product in FP64) or "mixed" (Schur products on
    the INT8 tensor cores with FP64-accurate digit splitting).  gemm_form /
    gj_nb: schedule knobs (0 = library default; see libnegf_b200.autotune).
    gj_update (mixed only): the Gauss-Jordan rank-nb updates as INT8 digit
    products with 34 pairs (2) or FP64 products (1); 0 = library default."""
    o = _lib.SolveOpts()
    o.eta, o.mu_l, o.mu_r, o.kT = eta, mu_l, mu_r, kT
    o.want_gr, o.want_gl, o.want_t = int(want_gr), int(want_gl), int(want_t)
    o.max_chunk = int(max_chunk)
    o.hbm_budget_gb = float(hbm_budget_gb)
    o.precision = {"fp64": _lib.NEGF_PREC_FP64, "mixed": _lib.NEGF_PREC_MIXED}[precision]
    o.gemm_form = int(gemm_form)
    o.gj_nb = int(gj_nb)
    o.sigma_per_energy = int(bool(sigma_per_energy))
    o.gj_update = int(gj_update)
    return o


class Device:
    """One device (block-tridiagonal H and lead self-energies) on the GPU."""

    def __init__(self, Hd, Hu, sigL, sigR):
        self.sizes = [int(h.shape[0]) for h in Hd]
        self.npl = len(Hd)
        self._handle = ctypes.c_void_p()
        kd, pd = _host_blocks(Hd)
        ku, pu = _host_blocks(Hu)
        sl = np.asfortranarray(np.asarray(sigL, dtype=np.complex128))
        sr = np.asfortranarray(np.asarray(sigR, dtype=np.complex128))
        check(load().negf_device_create(self.npl, int_array(self.sizes), ptr_array(pd), ptr_array(pu),
                                        sl.ctypes.data, sr.ctypes.data, ctypes.byref(self._handle)))

    def upload(self, Hd, Hu, sigL, sigR):
        kd, pd = _host_blocks(Hd)
        ku, pu = _host_blocks(Hu)
        sl = np.asfortranarray(np.asarray(sigL, dtype=np.complex128))
        sr = np.asfortranarray(np.asarray(sigR, dtype=np.complex128))
        check(load().negf_device_upload(self._handle, ptr_array(pd), ptr_array(pu), sl.ctypes.data, sr.ctypes.data))

    def set_overlap(self, Sd=None, Su=None):
        """Overlap matrix S (diagonal blocks Sd, upper blocks Su; None: identity /
        zero): solvers created afterwards use M(E) = (E + i eta) S - H - Sigma."""
        kd, pd = _host_blocks(Sd) if Sd is not None else (None, None)
        ku, pu = _host_blocks(Su) if Su is not None else (None, None)
        check(load().negf_device_set_overlap(self._handle, ptr_array(pd) if pd is not None else None,
                                             ptr_array(pu) if pu is not None else None))

    @property
    def handle(self):
        return self._handle

    def close(self):
        if self._handle:
            load().negf_device_destroy(self._handle)
            self._handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, energies, eta=1e-6, mu_l=0.1, mu_r=-0.1, kT=0.025, want_gr=True, want_gl=True, want_t=True,
              max_chunk=0, precision="fp64", gj_update=0):
        """G^R / G^< diagonal blocks and T(E) for every energy (host arrays).

        Returns (gr, gl, t): gr/gl are lists (per energy) of lists (per layer)
        of b_i x b_i arrays, or None."""
        E = np.ascontiguousarray(np.asarray(energies, dtype=np.float64))
        nE = len(E)
        per = sum(b * b for b in self.sizes)
        gr = np.empty(nE * per, dtype=np.complex128) if want_gr else None
        gl = np.empty(nE * per, dtype=np.complex128) if want_gl else None
        t = np.empty(nE, dtype=np.float64) if want_t else None
        o = make_opts(eta, mu_l, mu_r, kT, want_gr, want_gl, want_t, max_chunk, precision=precision,
                      gj_update=gj_update)
        check(load().negf_solve(self._handle, nE, E.ctypes.data_as(_lib.c_double_p), ctypes.byref(o),
                                gr.ctypes.data if gr is not None else None,
                                gl.ctypes.data if gl is not None else None,
                                t.ctypes.data_as(_lib.c_double_p) if t is not None else None, 0, None))
        return self._split(gr, nE), self._split(gl, nE), t

    def selected_inverse(self, energies, method="ddrgf", precision="fp64", eta=1e-6, levels=None, max_chunk=0,
                         want=("d", "u", "l")):
        """Blocks (i,i), (i,i+1), (i+1,i) of G^R(E) = M(E)^{-1} for every energy
        (negf_device_selected_inverse): method "rgf", "ddrgf" (levels: interior
        sizes per level, None = the library's cost model) or "selinv" (block LU
        selected inverse, no pivoting inside blocks).

        Returns (d, u, l): per energy lists of blocks (None where not wanted)."""
        E = np.ascontiguousarray(np.asarray(energies, dtype=np.float64))
        nE = len(E)
        sd = sum(b * b for b in self.sizes)
        su = sum(self.sizes[i] * self.sizes[i + 1] for i in range(self.npl - 1))
        gd = np.empty(nE * sd, dtype=np.complex128) if "d" in want else None
        gu = np.empty(max(1, nE * su), dtype=np.complex128) if "u" in want and su else None
        gl = np.empty(max(1, nE * su), dtype=np.complex128) if "l" in want and su else None
        o = make_opts(eta, max_chunk=max_chunk, precision=precision)
        m = {"rgf": _lib.NEGF_METHOD_RGF, "ddrgf": _lib.NEGF_METHOD_DDRGF, "selinv": _lib.NEGF_METHOD_SELINV}[method]
        lv = list(levels) if levels else []
        check(load().negf_device_selected_inverse(self._handle, nE, E.ctypes.data_as(_lib.c_double_p), ctypes.byref(o),
                                                  m, len(lv), int_array(lv) if lv else None,
                                                  gd.ctypes.data if gd is not None else None,
                                                  gu.ctypes.data if gu is not None else None,
                                                  gl.ctypes.data if gl is not None else None, 0, None))

        def split(flat, shapes):
            if flat is None:
                return None
            out = []
            for e in range(nE):
                o, row = e * sum(r * c for r, c in shapes), []
                for r, c in shapes:
                    row.append(flat[o:o + r * c].reshape(r, c, order="F"))
                    o += r * c
                out.append(row)
            return out

        b = self.sizes
        return (split(gd, [(x, x) for x in b]), split(gu, [(b[i], b[i + 1]) for i in range(self.npl - 1)]),
                split(gl, [(b[i + 1], b[i]) for i in range(self.npl - 1)]))

    def _split(self, flat, nE):
        if flat is None:
            return None
        per = sum(b * b for b in self.sizes)
        out = []
        for e in range(nE):
            o = e * per
            row = []
            for b in self.sizes:
                row.append(flat[o:o + b * b].reshape(b, b, order="F"))
                o += b * b
            out.append(row)
        return out


class Solver:
    """Resident plan for repeated solves of nE energies (device outputs)."""

    def __init__(self, device, nE, **kw):
        self.device = device
        self.devices = [device]
        self.counts = [int(nE)]
        self.nE = int(nE)
        self.opts = make_opts(**kw)
        self._h = ctypes.c_void_p()
        check(load().negf_solver_create(device.handle, self.nE, ctypes.byref(self.opts), ctypes.byref(self._h)))

    def set_energies(self, energies, stream=None):
        E = np.ascontiguousarray(np.asarray(energies, dtype=np.float64))
        assert len(E) == self.nE
        check(load().negf_solver_set_energies(self._h, E.ctypes.data_as(_lib.c_double_p), stream))

    def set_self_energies(self, sigL, sigR, stream=None):
        """Per-energy Sigma_L(E), Sigma_R(E) (lists of nE blocks in the energy
        order) for a solver made with sigma_per_energy=True."""
        kl, pl = _host_blocks(sigL)
        kr, pr = _host_blocks(sigR)
        check(load().negf_solver_set_self_energies(self._h, ptr_array(pl), ptr_array(pr), stream))

    def run(self, stream=None):
        check(load().negf_solver_run(self._h, stream))

    def check(self):
        check(load().negf_solver_check(self._h))

    KINDS = ["gemm", "gj_panel", "gj_unpermute", "blockop", "trace", "lu_panel", "lu_swap", "tri_diag",
             "oz_split", "oz_mma"]

    def run_profiled(self, stream=None):
        """One pass launch by launch with a CUDA event after each launch."""
        check(load().negf_solver_run_profiled(self._h, stream))

    def profile_read(self, reset=True):
        """Per kernel kind: (ms, flops, launches) summed over profiled passes."""
        K = len(self.KINDS)
        ms = (ctypes.c_double * K)()
        fl = (ctypes.c_double * K)()
        n = (ctypes.c_int64 * K)()
        check(load().negf_solver_profile_read(self._h, ms, fl, n, int(reset)))
        return {k: (ms[i], fl[i], n[i]) for i, k in enumerate(self.KINDS)}

    def download(self, gr_ptr, gl_ptr, t_ptr, stream=None):
        """Copy the outputs into host memory at the given addresses (None: skip)."""
        check(load().negf_solver_download(self._h, gr_ptr, gl_ptr,
                                          ctypes.cast(t_ptr, _lib.c_double_p) if t_ptr else None, stream))

    def run_download(self, gr_ptr, gl_ptr, t_ptr, stream=None):
        """One pass with the downloads into host memory at the given addresses
        (pinned; None: skip) overlapped with it, layer by layer; returns when
        done (negf_solver_run_download)."""
        check(load().negf_solver_run_download(self._h, gr_ptr, gl_ptr,
                                              ctypes.cast(t_ptr, _lib.c_double_p) if t_ptr else None, stream))

    def outputs(self):
        gr = ctypes.c_void_p()
        gl = ctypes.c_void_p()
        t = ctypes.POINTER(ctypes.c_double)()
        check(load().negf_solver_outputs(self._h, ctypes.byref(gr), ctypes.byref(gl), ctypes.byref(t)))
        return gr.value, gl.value, ctypes.cast(t, ctypes.c_void_p).value

    def stats(self):
        f = ctypes.c_double()
        n = ctypes.c_int64()
        w = ctypes.c_int64()
        check(load().negf_solver_stats(self._h, ctypes.byref(f), ctypes.byref(n), ctypes.byref(w)))
        return {"flops": f.value, "launches": n.value, "workspace_bytes": w.value}

    def layout(self):
        """(device index, energy index within the device, element offset) of every
        energy's output blocks in gr / gl (device-major)."""
        out, off = [], 0
        for k, (d, n) in enumerate(zip(self.devices, self.counts)):
            per = sum(b * b for b in d.sizes)
            for e in range(n):
                out.append((k, e, off))
                off += per
        return out, off

    def host_outputs(self, stream=None):
        """Download everything and split it: (gr, gl, t) with gr[k][e][i] the
        diagonal block i of energy e of device k (numpy), t[k][e] real."""
        lay, total = self.layout()
        gr = np.empty(total, dtype=np.complex128) if self.opts.want_gr else None
        gl = np.empty(total, dtype=np.complex128) if self.opts.want_gl else None
        t2 = np.empty(2 * self.nE, dtype=np.float64) if self.opts.want_t else None
        self.download(gr.ctypes.data if gr is not None else None, gl.ctypes.data if gl is not None else None,
                      t2.ctypes.data if t2 is not None else None, stream)

        def split(flat):
            if flat is None:
                return None
            res = [[None] * n for n in self.counts]
            for (k, e, off) in lay:
                row, o = [], off
                for b in self.devices[k].sizes:
                    row.append(flat[o:o + b * b].reshape(b, b, order="F"))
                    o += b * b
                res[k][e] = row
            return res

        t = None
        if t2 is not None:
            t, g = [], 0
            for n in self.counts:
                t.append(t2[0::2][g:g + n])
                g += n
        return split(gr), split(gl), t

    def close(self):
        if self._h:
            load().negf_solver_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchSolver(Solver):
    """One resident plan over several devices of different layer counts and
    block sizes (counts[k] energies of devices[k]); energies and outputs are
    device-major (see negf_solver_create_batch)."""

    def __init__(self, devices, counts, **kw):
        self.devices = list(devices)
        self.device = self.devices[0]
        self.counts = [int(c) for c in counts]
        self.nE = sum(self.counts)
        self.opts = make_opts(**kw)
        self._h = ctypes.c_void_p()
        handles = (ctypes.c_void_p * len(self.devices))(*[d.handle.value for d in self.devices])
        cnt = (ctypes.c_int32 * len(self.counts))(*self.counts)
        check(load().negf_solver_create_batch(len(self.devices), handles, cnt, ctypes.byref(self.opts),
                                              ctypes.byref(self._h)))

