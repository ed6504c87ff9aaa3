"""Request server: NEGF solves of different sizes as they arrive.

A request is (H blocks, Sigma_L, Sigma_R, energy list); its Hamiltonian is
uploaded once at submission and stays resident until the request completes.
A worker thread batches whenever the GPU is free: it takes the queued work
FIFO -- (request, chunk of its energies) items, split so that one group's
workspace fits the HBM budget (the library's own estimate,
``negf_batch_bytes``) -- and solves the group as one ``BatchSolver`` (one
launch per recursion step over every item) with autotuned schedule knobs
(tuned once per group signature and cached).  Requests arriving meanwhile
join the next group; this server runs one group at a time.  ``NativeServer``
(the library's negf_server_*) runs several groups at once on separate
streams, admitting new requests while others are on the GPU.  A request completes when its
last chunk is done; its latency (arrival to completion) feeds the p50 / p99
statistics.

The reference has no request loop (it solves one energy per call); this
serves its RGF + RKD + transmission (src/matinvertndiag_rgf.jl:114-200,
src/keldyshndiag.jl:120-317).  Responses carry T(E) for every energy and, when
asked for, the diagonal G^R / G^< blocks (host arrays).
"""

import collections
import threading
import time

import numpy as np

from ._lib import NEGF_ERR_NOMEM, NegfError
from .batch import bytes_per_energy, default_budget, pack
from .negf import BatchSolver, Device


class Request:
    def __init__(self, rid, device, energies, want_blocks):
        self.id = rid
        self.device = device
        self.energies = np.asarray(energies, dtype=np.float64)
        self.want_blocks = want_blocks
        self.arrival = time.perf_counter()
        self.done_at = None
        self.t = np.empty(len(self.energies))
        self.gr = [None] * len(self.energies) if want_blocks else None
        self.gl = [None] * len(self.energies) if want_blocks else None
        self.remaining = len(self.energies)
        self.error = None
        self._event = threading.Event()

    @property
    def latency(self):
        return None if self.done_at is None else self.done_at - self.arrival

    def wait(self, timeout=None):
        if not self._event.wait(timeout):
            raise TimeoutError("request %d not done" % self.id)
        if self.error is not None:
            raise self.error
        return self


def _device_view(ptr, n):
    """A device address as a flat float64 torch tensor (no copy)."""
    import torch

    class _P:
        def __init__(self):
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                             "strides": None}

    return torch.as_tensor(_P(), device="cuda")


class NegfServer:
    def __init__(self, precision="fp64", budget_bytes=None, tune=True, eta=1e-6, mu_l=0.1, mu_r=-0.1, kT=0.025):
        import torch
        self.precision = precision
        self.phys = dict(eta=eta, mu_l=mu_l, mu_r=mu_r, kT=kT)
        self.budget = budget_bytes or default_budget()
        self.tune = tune
        self._queue = collections.deque()  # (request, first energy, count)
        self._lock = threading.Condition()
        self._stop = False
        self._ids = 0
        self.completed = []
        self.groups = 0
        self.energy_points = 0
        self.device_ms = 0.0
        self._stream = torch.cuda.Stream()
        self._tuned = {}  # schedule knobs per group signature
        self._worker = threading.Thread(target=self._loop, daemon=True)
        self._worker.start()

    # -- client side -------------------------------------------------------
    def submit(self, Hd, Hu, sigL, sigR, energies, want_blocks=False):
        dev = Device(Hd, Hu, sigL, sigR)
        with self._lock:
            self._ids += 1
            req = Request(self._ids, dev, energies, want_blocks)
            req.per_energy = bytes_per_energy(dev, precision=self.precision, want_gr=want_blocks,
                                              want_gl=want_blocks, want_t=True, **self.phys)
            self._queue.append((req, 0, len(req.energies)))
            self._lock.notify()
        return req

    def close(self):
        with self._lock:
            self._stop = True
            self._lock.notify()
        self._worker.join()

    def latency_stats(self):
        lat = np.array([r.latency for r in self.completed if r.latency is not None])
        if lat.size == 0:
            return {"requests": 0}
        return {"requests": int(lat.size), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()), "max_s": float(lat.max())}

    # -- worker ------------------------------------------------------------
    def _take_group(self):
        """FIFO work under the budget: whole queued items, the last one split."""
        items = [(i, c, req.per_energy) for i, (req, s, c) in enumerate(self._queue)]
        groups = pack(items, self.budget)
        first = groups[0]
        taken = []
        for qi, start, count in first:
            req, s0, _ = self._queue[qi]
            taken.append((req, s0 + start, count))
        # drop what was taken from the queue (the head items, the last maybe in part)
        for qi, start, count in first:
            req, s0, c0 = self._queue[0]
            if start + count == c0:
                self._queue.popleft()
            else:
                self._queue[0] = (req, s0 + start + count, c0 - start - count)
        return taken

    def _loop(self):
        import torch
        sh = self._stream.cuda_stream
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        while True:
            with self._lock:
                while not self._queue and not self._stop:
                    self._lock.wait()
                if self._stop and not self._queue:
                    return
                group = self._take_group()
            want_blocks = any(r.want_blocks for r, _, _ in group)
            devs = [r.device for r, _, _ in group]
            knobs = {}
            if self.tune:
                from .autotune import autotune, signature
                sig = signature(devs, self.precision)
                if sig not in self._tuned:
                    self._tuned[sig], _ = autotune(devs, [c for _, _, c in group], precision=self.precision,
                                                   eta=self.phys["eta"])
                knobs = self._tuned[sig]
            try:
                try:
                    solver = BatchSolver(devs, [c for _, _, c in group], precision=self.precision,
                                         want_gr=want_blocks, want_gl=want_blocks, want_t=True, **self.phys, **knobs)
                except NegfError as exc:
                    if exc.code != NEGF_ERR_NOMEM or sum(c for _, _, c in group) <= 1:
                        raise
                    # the estimate was short: requeue the group, halve the budget
                    with self._lock:
                        for item in reversed(group):
                            self._queue.appendleft(item)
                        self.budget = max(1, self.budget // 2)
                    continue
                try:
                    solver.set_energies(np.concatenate([r.energies[s:s + c] for r, s, c in group]), sh)
                    ev0.record(self._stream)
                    solver.run(sh)
                    ev1.record(self._stream)
                    ev1.synchronize()
                    solver.check()
                    self.device_ms += ev0.elapsed_time(ev1)
                    self._deliver(solver, group)
                finally:
                    solver.close()
                self.groups += 1
            except Exception as exc:  # the group fails as a whole
                for r, s, c in group:
                    r.error = exc
                    self._finish(r, c)
                continue

    def _deliver(self, solver, group):
        gr_p, gl_p, t_p = solver.outputs()
        t = _device_view(t_p, 2 * solver.nE)[0::2].cpu().numpy()
        lay, total = solver.layout()
        g = 0
        for k, (r, s, c) in enumerate(group):
            r.t[s:s + c] = t[g:g + c]
            if r.want_blocks:
                sizes = r.device.sizes
                per = sum(b * b for b in sizes)
                for e in range(c):
                    off = lay[g + e][2]
                    for which, dst in ((gr_p, r.gr), (gl_p, r.gl)):
                        flat = _device_view(which, 2 * total)[2 * off:2 * (off + per)].cpu().numpy()
                        flat = flat.view(np.complex128)
                        blocks, o = [], 0
                        for b in sizes:
                            blocks.append(flat[o:o + b * b].reshape(b, b, order="F"))
                            o += b * b
                        dst[s + e] = blocks
            g += c
            self.energy_points += c
            self._finish(r, c)

    def _finish(self, r, count):
        r.remaining -= count
        if r.remaining <= 0 and r.done_at is None:
            r.done_at = time.perf_counter()
            r.device.close()
            self.completed.append(r)
            r._event.set()


class NativeServer:
    """The library's own request server (negf_server_*), for any host
    language: ``lanes`` native worker threads, each with its own CUDA stream,
    admit queued requests first in, first out, whenever the HBM budget has
    room beside the groups already on the GPU, so requests that arrive while
    others run start at once and their launches overlap (continuous
    batching).  ``submit`` returns a ticket object whose ``wait()`` gives
    (gr, gl, t) as host arrays."""

    def __init__(self, budget_gb=0.0, lanes=2, **opts):
        import ctypes
        from . import _lib
        from .negf import make_opts
        self._lib = _lib
        o = make_opts(**opts)
        self._h = ctypes.c_void_p()
        _lib.check(_lib.load().negf_server_create_ex(ctypes.byref(o), float(budget_gb), int(lanes),
                                                     ctypes.byref(self._h)))

    class Ticket:
        def __init__(self, server, tid, sizes, nE, keep):
            self.server, self.id, self.sizes, self.nE, self._keep = server, tid, sizes, nE, keep

        def done(self):
            import ctypes
            d = ctypes.c_int32()
            self.server._lib.check(self.server._lib.load().negf_server_poll(self.server._h, self.id, ctypes.byref(d)))
            return bool(d.value)

        def wait(self, timeout=600.0):
            """Block until done (at most ``timeout`` seconds); returns (gr, gl, t)
            with gr[e][i] the diagonal block i of energy e."""
            import ctypes
            lat = ctypes.c_double()
            self.server._lib.check(self.server._lib.load().negf_server_wait(self.server._h, self.id, float(timeout),
                                                                            ctypes.byref(lat)))
            self.latency = lat.value
            gr, gl, t = self._keep[:3]

            def split(flat):
                if flat is None:
                    return None
                out, o = [], 0
                for _ in range(self.nE):
                    row = []
                    for b in self.sizes:
                        row.append(flat[o:o + b * b].reshape(b, b, order="F"))
                        o += b * b
                    out.append(row)
                return out
            return split(gr), split(gl), t

    def submit(self, Hd, Hu, sigL, sigR, energies, want_blocks=True, out=None):
        """Queue one request.  ``out`` = (gr, gl, t): caller-owned flat output
        arrays (complex128 of len(energies) * sum b_i^2, float64 of
        len(energies)) that the results are written into -- e.g. views of
        pinned host memory reused across requests, which receive at DMA speed;
        by default fresh arrays are allocated (their pages are first touched by
        the copy, which costs several times the transfer itself)."""
        import ctypes
        from .negf import _host_blocks
        E = np.ascontiguousarray(np.asarray(energies, dtype=np.float64))
        sizes = [int(h.shape[0]) for h in Hd]
        per = sum(b * b for b in sizes)
        if out is not None:
            gr, gl, t = out
            for a, n, dt in ((gr, len(E) * per, np.complex128), (gl, len(E) * per, np.complex128),
                             (t, len(E), np.float64)):
                if a is not None and (a.dtype != dt or a.size < n or not a.flags.c_contiguous):
                    raise ValueError("out arrays: contiguous %s of at least %d elements" % (np.dtype(dt).name, n))
            if t is None:
                raise ValueError("out: t is required")
        else:
            gr = np.empty(len(E) * per, dtype=np.complex128) if want_blocks else None
            gl = np.empty(len(E) * per, dtype=np.complex128) if want_blocks else None
            t = np.empty(len(E), dtype=np.float64)
        kd, pd = _host_blocks(Hd)
        ku, pu = _host_blocks(Hu)
        sl = np.asfortranarray(np.asarray(sigL, dtype=np.complex128))
        sr = np.asfortranarray(np.asarray(sigR, dtype=np.complex128))
        lib, L = self._lib, self._lib.load()
        tid = ctypes.c_int64()
        lib.check(L.negf_server_submit(self._h, len(sizes), lib.int_array(sizes), lib.ptr_array(pd),
                                       lib.ptr_array(pu), sl.ctypes.data, sr.ctypes.data, len(E),
                                       E.ctypes.data_as(lib.c_double_p), gr.ctypes.data if gr is not None else None,
                                       gl.ctypes.data if gl is not None else None,
                                       t.ctypes.data_as(lib.c_double_p), ctypes.byref(tid)))
        # the output buffers (and energies) stay referenced until the ticket is dropped
        return NativeServer.Ticket(self, tid.value, sizes, len(E), (gr, gl, t, E))

    def stats(self):
        import ctypes
        c, g = ctypes.c_int64(), ctypes.c_int64()
        p50, p99 = ctypes.c_double(), ctypes.c_double()
        self._lib.check(self._lib.load().negf_server_stats(self._h, ctypes.byref(c), ctypes.byref(g),
                                                           ctypes.byref(p50), ctypes.byref(p99)))
        q, inf, peak, gb = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
        self._lib.check(self._lib.load().negf_server_stats_ex(self._h, ctypes.byref(q), ctypes.byref(inf),
                                                              ctypes.byref(peak), ctypes.byref(gb)))
        return {"requests": c.value, "groups": g.value, "p50_s": p50.value, "p99_s": p99.value, "queued": q.value,
                "inflight_groups": inf.value, "peak_inflight_groups": peak.value, "inflight_gb": gb.value}

    def close(self):
        if self._h:
            self._lib.load().negf_server_destroy(self._h)
            self._h = None


def group_sizes(bytes_per_request, budget):
    """The native worker's grouping rule (negf_server_group_sizes)."""
    import ctypes
    from . import _lib
    n = len(bytes_per_request)
    b = (ctypes.c_int64 * max(1, n))(*[int(x) for x in bytes_per_request])
    sizes = (ctypes.c_int32 * max(1, n))()
    ng = ctypes.c_int32()
    _lib.check(_lib.load().negf_server_group_sizes(n, b, float(budget), sizes, ctypes.byref(ng)))
    return list(sizes[:ng.value])
