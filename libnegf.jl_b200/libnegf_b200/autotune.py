"""Schedule autotuner for batched solves.

The reference picks its DDRGF partition with wall-clock probes of the LAPACK
kernels and a cost model (src/matinvertndiag_ddrgf_utils.jl:37-219, :357-453).
For batches of devices of uneven layer counts and block sizes the schedule
knobs of this library are

  * ``gemm_form``: FP64 complex products as four real DMMA products (1) or in
    the 3M (Gauss) form (2);
  * ``gj_nb``: the Gauss-Jordan panel width for blocks above 112 (8, 16, 32;
    wider panels need more shared memory, narrower ones more rank updates).

``autotune`` times every admissible candidate on a sample of the batch (a few
energies of a spread of its devices), with CUDA events around graph replays,
and returns the fastest; results are cached per batch signature (precision
and largest block size class), so a server pays for tuning once per class.
"""

import itertools

import numpy as np

from ._lib import NegfError
from .negf import BatchSolver

_CACHE = {}
_SMEM_PER_BLOCK = 227 * 1024


def _panel_fits(n, nb):
    # the panel kernel stages an n x nb slab of complex doubles plus pivot data
    return n * nb * 16 + 16 * 1024 <= _SMEM_PER_BLOCK


def signature(devices, precision):
    """Shape class of a batch: precision and its largest block size rounded up
    to a multiple of 64 (the knobs act per block size: panel width, GEMM
    tiles), so that a server tunes once per class, not per request mix."""
    maxb = max(max(d.sizes) for d in devices)
    return (precision, -(-maxb // 64) * 64)


def candidates(devices):
    maxb = max(max(d.sizes) for d in devices)
    nbs = [0]
    if maxb > 112:
        nbs += [nb for nb in (8, 16, 32) if _panel_fits(maxb, nb)]
    return [dict(gemm_form=f, gj_nb=nb) for f, nb in itertools.product((2, 1), nbs)]


def _sample(devices, counts, max_devices, per_device):
    idx = np.unique(np.linspace(0, len(devices) - 1, min(max_devices, len(devices))).round().astype(int))
    return [devices[i] for i in idx], [min(counts[i], per_device) for i in idx]


def autotune(devices, counts, precision="fp64", energies=None, max_devices=32, per_device=4, reps=3, eta=1e-6,
             use_cache=True):
    """Best schedule knobs for solving ``counts[k]`` energies of
    ``devices[k]``: returns (knobs, table) with knobs a dict for
    ``make_opts`` / ``BatchSolver`` and table the measured ms per pass of
    every candidate on the sample."""
    import torch

    key = signature(devices, precision)
    if use_cache and key in _CACHE:
        return _CACHE[key]
    devs, cnts = _sample(devices, counts, max_devices, per_device)
    E = np.concatenate([np.linspace(-0.9, 0.9, c) for c in cnts]) if energies is None else np.asarray(energies)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    table = []
    for cand in candidates(devs):
        try:
            s = BatchSolver(devs, cnts, eta=eta, precision=precision, want_t=False, **cand)
        except NegfError:  # not admissible for these block sizes (shared memory)
            continue
        try:
            s.set_energies(E[:s.nE], sh)
            s.run(sh)  # capture + warm
            stream.synchronize()
            ev0.record(stream)
            for _ in range(reps):
                s.run(sh)
            ev1.record(stream)
            ev1.synchronize()
            s.check()
            table.append((cand, ev0.elapsed_time(ev1) / reps))
        finally:
            s.close()
    best = min(table, key=lambda t: t[1])[0]
    result = (best, table)
    _CACHE[key] = result
    return result
