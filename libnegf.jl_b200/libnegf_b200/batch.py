"""Uneven batches: many devices of different layer counts and block sizes,
each with its own energy list, solved as a few resident batch plans.

The reference solves one system and one energy per call
(src/matinvertndiag_rgf.jl:114-200, src/keldyshndiag.jl:120-317) and budgets
memory per call against 80 % of the RAM (src/keldyshndiag.jl:14-77,
``check_if_enough_mem_rkd``).  Here the work items -- (device, chunk of its
energies) -- are packed in order into groups whose device workspace, as the
library estimates it (``negf_batch_bytes``), fits an HBM budget; every group
is one ``BatchSolver`` (one launch per recursion step over all its items) with
schedule knobs from the autotuner, and its outputs are handed to a consumer
while they are resident.
"""

import ctypes
import time

import numpy as np

from . import _lib
from ._lib import NegfError, check, load
from .negf import BatchSolver, make_opts


def bytes_per_energy(device, **opts):
    """Device bytes one energy of ``device`` needs in a batch plan."""
    o = make_opts(**opts)
    h = (ctypes.c_void_p * 1)(device.handle.value)
    n = (ctypes.c_int32 * 1)(1)
    out = ctypes.c_int64()
    check(load().negf_batch_bytes(1, h, n, ctypes.byref(o), ctypes.byref(out)))
    return int(out.value)


def pack(items, budget):
    """Greedy in-order packing of work items into groups.

    items: list of (key, count, bytes_per_unit); returns a list of groups, each
    a list of (key, start, count) with sum(count * bytes_per_unit) <= budget.
    Items are split into chunks when one alone does not fit; a single unit
    larger than the budget gets a group of its own (the caller's allocation
    then decides)."""
    groups, cur, used = [], [], 0
    for key, count, per in items:
        start = 0
        while start < count:
            room = (budget - used) // per if per > 0 else count - start
            if room <= 0:
                if cur:
                    groups.append(cur)
                    cur, used = [], 0
                    continue
                room = 1  # one unit above the budget: alone
            take = min(count - start, room)
            cur.append((key, start, take))
            used += take * per
            start += take
    if cur:
        groups.append(cur)
    return groups


def halve(group):
    """Split a group's energies into a first and a second half, in order (the
    item at the boundary is split)."""
    total = sum(c for _, _, c in group)
    half = max(1, total // 2)
    first, second, acc = [], [], 0
    for k, s, c in group:
        if acc >= half:
            second.append((k, s, c))
            continue
        take = min(c, half - acc)
        first.append((k, s, take))
        if take < c:
            second.append((k, s + take, c - take))
        acc += take
    return [g for g in (first, second) if g]


def default_budget():
    import torch
    free, _ = torch.cuda.mem_get_info()
    return int(0.8 * free)


def solve_uneven(devices, energies, precision="fp64", budget_bytes=None, tune=True, on_group=None, stream=None,
                 eta=1e-6, mu_l=0.1, mu_r=-0.1, kT=0.025, want_gr=True, want_gl=True, want_t=True):
    """Solve ``energies[k]`` of ``devices[k]`` for every k.

    on_group(solver, parts): called after each group with the resident
    ``BatchSolver`` (its device-major outputs) and ``parts``, the group's
    (device index, first energy, count) list, in the solver's order.
    Returns a dict of statistics (groups, device ms, energy points/s)."""
    phys = dict(eta=eta, mu_l=mu_l, mu_r=mu_r, kT=kT, want_gr=want_gr, want_gl=want_gl, want_t=want_t)
    budget = budget_bytes or default_budget()
    per = [bytes_per_energy(d, precision=precision, **phys) for d in devices]
    items = [(k, len(energies[k]), per[k]) for k in range(len(devices))]
    groups = pack(items, budget)
    knobs, table = {}, None
    if tune:
        from .autotune import autotune
        knobs, table = autotune(devices, [len(e) for e in energies], precision=precision, eta=eta)
    import torch
    st = stream or torch.cuda.Stream()
    sh = st.cuda_stream
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dev_ms, pts, solved = 0.0, 0, 0
    t0 = time.perf_counter()
    pending = list(groups)
    while pending:
        g = pending.pop(0)
        try:
            solver = BatchSolver([devices[k] for k, _, _ in g], [c for _, _, c in g], precision=precision, **phys,
                                 **knobs)
        except NegfError as exc:
            # the estimate was short: halve the group and retry
            if exc.code != _lib.NEGF_ERR_NOMEM or sum(c for _, _, c in g) <= 1:
                raise
            pending[:0] = halve(g)
            continue
        try:
            solver.set_energies(np.concatenate([np.asarray(energies[k][s:s + c], dtype=np.float64)
                                                for k, s, c in g]), sh)
            ev0.record(st)
            solver.run(sh)
            ev1.record(st)
            ev1.synchronize()
            solver.check()
            dev_ms += ev0.elapsed_time(ev1)
            pts += solver.nE
            solved += 1
            if on_group is not None:
                on_group(solver, g)
        finally:
            solver.close()
    wall = time.perf_counter() - t0
    return {"groups": solved, "energy_points": pts, "device_ms": dev_ms, "wall_s": wall,
            "pts_per_s_device": pts / (dev_ms / 1000.0) if dev_ms else None, "pts_per_s_wall": pts / wall,
            "knobs": knobs, "tuning": table, "budget_bytes": budget}
