#!/usr/bin/env python
"""Benchmark of the batched-energy NEGF hot path on B200.

Workload (the reference's metric configuration): Keldysh G^R + G^< batched
over energies, ComplexF64 plain form -- a Hermitian block-tridiagonal device of
N = 32 layers of b = 256 (H_ii = (A + A^H)/2, A complex normal / sqrt(b);
H_{i,i+1} complex normal of variance 0.25 / sqrt(b); lead self-energies
Sigma = X - 0.05 i (Y Y^H + 0.1 I)), 256 energies uniform in [-1, 1], eta = 1e-6,
Fermi occupations at mu_L = 0.1, mu_R = -0.1, kT = 0.025.  Outputs per energy:
all diagonal G^R and G^< blocks and T(E) = Tr[Gamma_L G^R_1N Gamma_R G^A_N1].
Seeded synthetic data (numpy default_rng(0)); no dataset is involved.

One step = one pass of RGF (shared upward pass) + downward G^R + RKD + the
transmission chain over all 256 energies, on device-resident inputs, replayed
as one CUDA graph.  The headline is the mixed-precision path (Schur products on
the INT8 tensor cores with FP64-grade digit splitting; inversions in FP64),
checked block by block against the FP64 path's outputs on every 8th energy
(bar 1e-10) and, on four energies, both paths against the oracle
("accuracy_vs_oracle"); the FP64 path is timed beside it ("fp64_path").  The
p50 / p99 solve latency comes from a short Poisson request stream through the
library's request server (continuous batching, mixed precision, "serving").

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload cfg2|cfg3|cfg4|cfg5]

Multi-GPU: one process per GPU (torchrun; --gpus N without a launcher starts
the N ranks itself); every rank solves its own 256 energies (weak scaling, no
data-path collective); the time is the max over ranks.  ``--impl reference``
times the CPU restatement of the reference's algorithm (the oracle: LibNEGF.jl
itself is Julia and cannot run here) on the host cores.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "libnegf.jl_b200"))

METRIC = "energy pts/s, RGF G^R+G^< mixed vs FP64 @1e-10 rel err; p50/p99 solve latency"
UNIT = "energy_pts/s"
WORKLOAD = "Keldysh G^R + G^< (+T) batched over energies, ComplexF64 plain form, N=32 layers x b=256, 256 energies"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--npl", type=int, default=None, help="layers (cfg2: 32, cfg3: 64)")
    ap.add_argument("--b", type=int, default=None, help="block size (cfg2: 256, cfg3: 512)")
    ap.add_argument("--ne", type=int, default=None, help="energies (cfg2: 256, cfg3: 128)")
    ap.add_argument("--cpu-budget-s", type=float, default=12.0, help="time budget of each CPU baseline mode")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the request-stream latency sample")
    ap.add_argument("--serve-requests", type=int, default=12, help="requests in the latency sample")
    ap.add_argument("--serve-rate", type=float, default=4.0, help="arrival rate of the latency sample, requests/s")
    ap.add_argument("--workload", default="cfg2", choices=["cfg2", "cfg3", "cfg4", "cfg5"],
                    help="cfg2 (default, the headline line); cfg4: a bounded sample of the uneven batch (systems "
                         "of N in U{8..96}, b in {32..384}, 16 energies each); cfg5: a bounded sample of the "
                         "Poisson-arrival request stream through the server (p50/p99 latency)")
    ap.add_argument("--chunk", type=int, default=8, help="cfg3: energies per device-resident chunk")
    ap.add_argument("--methods", default="ddrgf,selinv,rgf", help="cfg3: methods to time (ddrgf, selinv, rgf)")
    ap.add_argument("--systems", type=int, default=96, help="cfg4: number of systems in the sample")
    ap.add_argument("--requests", type=int, default=16, help="cfg5: number of requests in the sample")
    ap.add_argument("--rate", type=float, default=2.0, help="cfg5: mean arrival rate, requests/s")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="cfg4 / cfg5 / --launch-list precision")
    ap.add_argument("--launch-list", action="store_true",
                    help="only two launch-by-launch passes of the solver (--precision; for an ncu launch list: skip the "
                         "first pass's launches, capture the second's); prints no bench line")
    a = ap.parse_args()
    dflt = {"cfg3": (64, 512, 128)}.get(a.workload, (32, 256, 256))
    a.npl = a.npl if a.npl is not None else dflt[0]
    a.b = a.b if a.b is not None else dflt[1]
    a.ne = a.ne if a.ne is not None else dflt[2]
    return a


def shard_energies(ne_per_rank, world, rank, lo=-1.0, hi=1.0):
    """Weak scaling: the global grid has ne_per_rank * world energies uniform in
    [lo, hi]; rank r solves the contiguous slice r.  No energy is shared."""
    grid = np.linspace(lo, hi, ne_per_rank * world)
    return grid[rank * ne_per_rank:(rank + 1) * ne_per_rank]


class _DevicePtr:
    """A device address seen as a flat float64 array (CUDA array interface)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}


def _device_doubles(ptr, n):
    import torch
    return torch.as_tensor(_DevicePtr(ptr, n), device="cuda")


def max_over_ranks(value, dist=None, device=None):
    """Max of a float over all ranks (the job time is the slowest rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def canonical_flops(npl, b):
    """Algorithmic real flops per energy point: the reference's call sequence
    for RKD plus the G^R downward pass sharing its upward pass, and the
    G^R_{1N} chain of the transmission (zgemm 8mnk, zgetrf 8/3 n^3, zgetrs
    8 n^2 nrhs)."""
    N = npl
    rkd = (8.0 / 3.0) * N + 72 * (N - 1) + 48 * (N - 2) + 16 * N + 16
    gr = 8 + 32 * (N - 1)
    trans = 8 * (N - 1) + 16
    return (rkd + gr + trans) * float(b) ** 3


# ---------------------------------------------------------------------------
# clocks sampling (nvidia-smi) during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thr = threading.Thread(target=self._read, daemon=True)
            self.thr.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = []
        mx = None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(name)
        under_load = [x for x in sm if mx and x > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(under_load) if under_load else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (the reference's algorithm restated in numpy/scipy)

def _cpu_solve_one(args):
    npl, b, E, seed, threads = args
    from threadpoolctl import threadpool_limits
    from oracle import physics
    with threadpool_limits(limits=threads):
        sysm = physics.physics_system(npl, b, seed=seed)
        t0 = time.perf_counter()
        physics.solve_energy(sysm, E)
        return time.perf_counter() - t0


def cpu_baseline(npl, b, energies, budget_s, seed=0):
    """Best of (i) one energy at a time with all BLAS threads (the reference's
    RGF/RKD benchmarks: one Julia thread, k BLAS threads,
    benchmrk/runbenchmrks.sh:44-47) and (ii) one energy per core with one BLAS
    thread each (its DDRGF model: Julia threads x 1 BLAS thread).  Each mode
    runs a bounded sample."""
    import multiprocessing as mp
    from threadpoolctl import threadpool_limits
    from oracle import physics
    cores = os.cpu_count() or 1
    sysm = physics.physics_system(npl, b, seed=seed)
    # (i) serial energies, all threads
    done, t0 = 0, time.perf_counter()
    with threadpool_limits(limits=cores):
        physics.solve_energy(sysm, energies[0])  # warm-up (excluded)
        t0 = time.perf_counter()
        while done < len(energies) and time.perf_counter() - t0 < budget_s:
            physics.solve_energy(sysm, energies[done])
            done += 1
    mode_i = done / (time.perf_counter() - t0)
    # (ii) one energy per process, one thread each
    ctx = mp.get_context("spawn")
    nproc = cores
    with ctx.Pool(nproc) as pool:
        pool.map(_cpu_solve_one, [(npl, b, energies[0], seed, 1)] * nproc)  # warm-up (import, first call)
        per = pool.map(_cpu_solve_one, [(npl, b, energies[k % len(energies)], seed, 1) for k in range(nproc)])
    mode_ii = nproc / max(per)
    best = max(mode_i, mode_ii)
    return {"value": best, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d energies serially with %d BLAS threads (%.2f pts/s) and %d energies in parallel, one BLAS "
                      "thread each (%.2f pts/s); full-size N=%d, b=%d; numpy/scipy OpenBLAS" %
                      (done, cores, mode_i, nproc, mode_ii, npl, b),
            "modes": {"serial_all_threads": mode_i, "parallel_1_thread": mode_ii}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    energies = np.linspace(-1.0, 1.0, args.ne)
    vals, walls = [], []
    cb = None
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        r = cpu_baseline(args.npl, args.b, energies, budget_s=args.cpu_budget_s / 2)
        if step >= args.warmup:
            vals.append(r["value"])
            walls.append(time.perf_counter() - t0)
            cb = r
    v = float(np.median(vals))
    # a step is one bounded sample of the workload (both threading modes); its
    # wall time is ms_per_step, its energies per second the value
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * float(np.median(walls)), "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded numpy, the generator of the config)",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "npl": args.npl, "b": args.b, "energies": args.ne, "precision": "fp64",
                       "note": "LibNEGF.jl is Julia and no Julia toolchain exists here: the reference arm times the "
                               "oracle, a numpy/scipy restatement of its LAPACK/BLAS call sequence; each step is a "
                               "bounded sample of the workload's energies (ms_per_step is that sample's wall time, "
                               "value its energy points per second)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cb["cores"], "kind": "port", "sample": cb["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm

def measured_hbm_gbs():
    """Measured HBM copy bandwidth of the GPU (MEASURED_PEAKS.json at the
    repository root), else an earlier measurement of 6.65 TB/s."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback (6.65 TB/s)"


def _host_outputs(outs, ne, per, idx):
    """Host copies of the G^R / G^< diagonal blocks (flat complex128) and T of
    the energies idx from a solver's device outputs."""
    import torch
    res = []
    for w in range(2):
        v = _device_doubles(outs[w], 2 * ne * per).view(ne, 2 * per)[idx].cpu().numpy()
        res.append(v.view(np.complex128))
    res.append(_device_doubles(outs[2], 2 * ne)[0::2][torch.tensor(idx, device="cuda")].cpu().numpy())
    return res


def accuracy_vs_oracle(sysm, energies, idx, sizes, paths):
    """Per-block relative Frobenius error of each path's G^R / G^< diagonal
    blocks and |dT| / max(1, |T|) against the oracle (the reference's LAPACK
    call sequence restated on the host) at the energies idx."""
    from oracle import physics
    out = {k: {"max_block_rel_err_GR": 0.0, "max_block_rel_err_GL": 0.0, "max_T_err": 0.0} for k in paths}
    for j, e in enumerate(idx):
        r = physics.solve_energy(sysm, energies[e])
        o = 0
        for i, b in enumerate(sizes):
            gr_ref, gl_ref = r["GR"].M[(i, i)], 1j * r["Gn"].M[(i, i)]
            for k, (gr, gl, t) in paths.items():
                a = gr[j][o:o + b * b].reshape(b, b, order="F")
                c = gl[j][o:o + b * b].reshape(b, b, order="F")
                d = out[k]
                d["max_block_rel_err_GR"] = max(d["max_block_rel_err_GR"],
                                                float(np.linalg.norm(a - gr_ref) / np.linalg.norm(gr_ref)))
                d["max_block_rel_err_GL"] = max(d["max_block_rel_err_GL"],
                                                float(np.linalg.norm(c - gl_ref) / np.linalg.norm(gl_ref)))
            o += b * b
        for k, (gr, gl, t) in paths.items():
            out[k]["max_T_err"] = max(out[k]["max_T_err"], float(abs(t[j] - r["T"]) / max(1.0, abs(r["T"]))))
    for k in out:
        out[k]["energies"] = [float(energies[e]) for e in idx]
        out[k]["bar"] = 1e-10 if k == "mixed" else 1e-12
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    import libnegf_b200 as negf
    from oracle import physics  # input generator only (seeded synthetic H, Sigma)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev_index = torch.cuda.current_device()
    negf.load()
    # CPU baseline first (spawned pool, before heavy GPU work)
    cpu = None
    my_E = shard_energies(args.ne, world, rank)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.npl, args.b, my_E, args.cpu_budget_s)

    sysm = physics.physics_system(args.npl, args.b, seed=0)
    dev = negf.Device(sysm.Hd, sysm.Hu, sysm.sigL, sysm.sigR)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    per = sum(b * b for b in dev.sizes)
    if args.launch_list:
        solver = negf.Solver(dev, args.ne, eta=sysm.eta, precision=args.precision)
        solver.set_energies(my_E, sh)
        for _ in range(2):
            solver.run_profiled(sh)
        stream.synchronize()
        solver.check()
        print("launch list: %d launches per pass" % solver.stats()["launches"], flush=True)
        solver.close()
        dev.close()
        return
    import ctypes
    # roofline denominators of this GPU, measured in-run
    d1, d2, d3 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    negf._lib.check(negf.load().negf_probe_fp64_peak(ctypes.byref(d1), ctypes.byref(d2)))
    fp64_peak = max(d1.value, d2.value)
    negf._lib.check(negf.load().negf_probe_int8_peak(ctypes.byref(d3)))
    int8_peak = d3.value
    # FP64 arithmetic beside INT8 MMAs on one SM (cycles): the product kernel's
    # FP64 drains cannot hide under its MMAs when beside ~ alone + mma
    o1, o2, o3 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    negf._lib.check(negf.load().negf_probe_fp64_int8_overlap(ctypes.byref(o1), ctypes.byref(o2), ctypes.byref(o3)))
    overlap = {"fp64_alone_cycles": o1.value, "fp64_beside_int8_mma_cycles": o2.value, "int8_mma_cycles": o3.value}
    step_flops = canonical_flops(args.npl, args.b) * args.ne
    total_pts = args.ne * args.steps * world
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)

    def timed(solver, clk=None):
        """Warm-up, then K graph replays bracketed by barrier + sync; max over ranks."""
        solver.set_energies(my_E, sh)
        for _ in range(args.warmup):
            solver.run(sh)
        stream.synchronize()
        solver.check()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            solver.run(sh)
        ev1.record(stream)
        ev1.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        solver.check()
        return max_over_ranks(ev0.elapsed_time(ev1), dist if world > 1 else None, "cuda")

    def profiled(solver):
        """Per-kernel device time of one launch-by-launch pass."""
        solver.profile_read(reset=True)
        solver.run_profiled(sh)
        stream.synchronize()
        return solver.profile_read(reset=True)

    hbm_peak, hbm_src = measured_hbm_gbs()

    def breakdown_of(prof):
        tot = sum(v[0] for v in prof.values()) or 1.0
        out = {}
        for k, v in prof.items():
            if not v[2]:
                continue
            e = {"ms": v[0], "launches": v[2], "share": v[0] / tot}
            if k == "oz_split":  # HBM-bound: the library reports its algorithmic bytes
                gbs = v[1] / (v[0] / 1000.0) / 1e9 if v[0] > 0 else None
                e.update({"bytes_per_launch": v[1] / v[2], "gbs": gbs, "hbm_peak_gbs": hbm_peak,
                          "hbm_frac": gbs / hbm_peak if gbs else None, "hbm_peak_source": hbm_src})
            elif k == "oz_mma":  # INT8 operations (3 real products x digit pairs x 2mnk)
                e["int8_tops"] = (v[1] / (v[0] / 1000.0) / 1e12) if v[0] > 0 and v[1] > 0 else None
            else:
                e["tflops"] = (v[1] / (v[0] / 1000.0) / 1e12) if v[0] > 0 and v[1] > 0 else None
            out[k] = e
        return out

    # ---- FP64 path (reference precision): timing, breakdown, reference outputs
    solver = negf.Solver(dev, args.ne, eta=sysm.eta)
    fstats = solver.stats()
    fms = timed(solver)
    fprof = profiled(solver)
    k_ms, k_fl, k_n = fprof["gemm"]
    f_ach = (k_fl / k_n) / ((k_ms / k_n) / 1000.0) / 1e12 if k_n else 0.0
    fvalue = total_pts / (fms / 1000.0)
    fp64 = {"value": fvalue, "unit": UNIT, "ms_per_step": fms / args.steps,
            "algorithmic_tflops": step_flops / ((fms / args.steps) / 1000.0) / 1e12,
            "gpu_launches": int(fstats["launches"]) * args.steps,
            "kernels": breakdown_of(fprof),
            "roofline": {"kernel": "zgemm3m_batched_kernel (DMMA m16n8k4 f64)", "bound": "tensor",
                         "achieved": f_ach, "peak": fp64_peak, "unit": "TFLOP/s",
                         "frac": f_ach / fp64_peak if fp64_peak else None,
                         "peak_source": "FP64 mma.sync throughput measured in-run (negf_probe_fp64_peak)"}}
    checked = list(range(0, args.ne, max(1, args.ne // 32)))
    solver.run(sh)
    stream.synchronize()
    outs = solver.outputs()
    refs = [_device_doubles(outs[w], 2 * args.ne * per).view(args.ne, 2 * per)[checked].clone() for w in range(2)]
    t_ref = _device_doubles(outs[2], 2 * args.ne)[0::2].clone()
    # four energies checked against the oracle (host copies of both paths' blocks)
    oidx = sorted({min(args.ne - 1, args.ne * k // 4 + args.ne // 8) for k in range(4)})
    host_f64 = _host_outputs(outs, args.ne, per, oidx)
    solver.close()

    # ---- mixed path (the headline): INT8 tensor-core Schur products
    solver = negf.Solver(dev, args.ne, eta=sysm.eta, precision="mixed")
    stats = solver.stats()
    with ClockSampler(dev_index) as clk:
        ms = timed(solver)
    prof = profiled(solver)
    value = total_pts / (ms / 1000.0)
    outs = solver.outputs()
    errs = [0.0, 0.0]
    for w in range(2):
        got = _device_doubles(outs[w], 2 * args.ne * per).view(args.ne, 2 * per)[checked]
        o = 0
        for bsz in dev.sizes:
            sl_ = slice(2 * o, 2 * (o + bsz * bsz))
            num = torch.linalg.vector_norm(got[:, sl_] - refs[w][:, sl_], dim=1)
            den = torch.linalg.vector_norm(refs[w][:, sl_], dim=1)
            errs[w] = max(errs[w], float((num / den).max()))
            o += bsz * bsz
    t_mix = _device_doubles(outs[2], 2 * args.ne)[0::2]
    t_err = float(((t_mix - t_ref).abs() / t_ref.abs().clamp(min=1.0)).max())
    del refs, t_ref
    host_mix = _host_outputs(outs, args.ne, per, oidx)
    acc_oracle = None
    if rank == 0:
        acc_oracle = accuracy_vs_oracle(sysm, my_E, oidx, dev.sizes, {"mixed": host_mix, "fp64": host_f64})

    # dominant kernel: the INT8 product kernel; the library reports its
    # algorithmic work as INT8 operations, 3 real products x digit pairs x
    # 2mnk per complex product (28 pairs for the Schur products, 34 for the
    # Gauss-Jordan updates)
    kind = max(prof, key=lambda k: prof[k][0])
    k_ms, k_fl, k_n = prof[kind]
    if kind == "oz_mma":
        achieved = (k_fl / k_n) / ((k_ms / k_n) / 1000.0) / 1e12
        roof = {"kernel": "ozaki_mma_kernel (tcgen05.mma kind::i8, TMEM accumulators)", "bound": "tensor",
                "achieved": achieved, "peak": int8_peak, "unit": "TOP/s (int8)",
                "frac": achieved / int8_peak if int8_peak else None,
                "peak_source": "dense kind::i8 tcgen05 throughput measured in-run (negf_probe_int8_peak)",
                "int8_ops_per_launch": k_fl / k_n}
    else:
        achieved = (k_fl / k_n) / ((k_ms / k_n) / 1000.0) / 1e12 if k_n else 0.0
        roof = {"kernel": kind, "bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak if fp64_peak else None}
    # DRAM bytes of the dominant kernel are an ncu measurement; this run is not
    # under ncu, so the per-launch traffic is not reported here
    roof["traffic"] = None
    roof["fp64_beside_int8"] = overlap
    roof["share"] = k_ms / sum(v[0] for v in prof.values())
    roof["launch_ms"] = k_ms / max(1, k_n)
    whole = {"algorithmic_tflops": step_flops / ((ms / args.steps) / 1000.0) / 1e12,
             "executed_complex_tflops": stats["flops"] / ((ms / args.steps) / 1000.0) / 1e12,
             "speedup_vs_fp64_path": value / fvalue}

    # ---- end to end through the public API with host buffers (pinned), mixed path
    e2e = None
    if not args.no_e2e:
        nbytes = args.ne * per * 16
        gr_h = torch.empty(args.ne * per * 2, dtype=torch.float64, pin_memory=True)
        gl_h = torch.empty(args.ne * per * 2, dtype=torch.float64, pin_memory=True)
        t_h = torch.empty(2 * args.ne, dtype=torch.float64, pin_memory=True)
        hd = [torch.from_numpy(np.asfortranarray(h).T.copy()).pin_memory() for h in sysm.Hd]
        hu = [torch.from_numpy(np.asfortranarray(h).T.copy()).pin_memory() for h in sysm.Hu]
        sl = torch.from_numpy(np.asfortranarray(sysm.sigL).T.copy()).pin_memory()
        sr = torch.from_numpy(np.asfortranarray(sysm.sigR).T.copy()).pin_memory()
        hd_np = [x.numpy().T for x in hd]
        hu_np = [x.numpy().T for x in hu]

        def e2e_step():
            # upload, energies, one pass with the G^R / G^< layers downloaded as
            # they become final (negf_solver_run_download), T
            dev.upload(hd_np, hu_np, sl.numpy().T, sr.numpy().T)
            solver.set_energies(my_E, sh)
            solver.run_download(gr_h.data_ptr(), gl_h.data_ptr(), t_h.data_ptr(), sh)

        for _ in range(max(1, args.warmup)):
            e2e_step()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        el = max_over_ranks(time.perf_counter() - t0, dist if world > 1 else None, "cuda")
        h2d = sum(h.nbytes for h in sysm.Hd) + sum(h.nbytes for h in sysm.Hu) + 2 * sysm.sigL.nbytes + my_E.nbytes
        e2e = {"value": total_pts / el, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(2 * nbytes + 16 * args.ne), "ms_per_step": 1000 * el / args.steps}

    # p50 / p99 solve latency of a short Poisson request stream through the
    # library's request server (mixed precision, continuous batching)
    serving = None
    if rank == 0 and world == 1 and not args.no_serving:
        reqs, gaps = request_stream(args.serve_requests, args.serve_rate, 6, (16, 64), [64, 128, 192, 256], (16, 64))
        serving = serve_stream(reqs, gaps, "mixed")
        serving["workload"] = ("%d requests, N in {16..64}, b in {64..256}, 16..64 energies each, Poisson arrivals "
                               "at %.1f/s" % (args.serve_requests, args.serve_rate))

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int8 products / f64",
                "data": "synthetic (seeded numpy generator of the config)",
                "config": {"workload": WORKLOAD, "npl": args.npl, "b": args.b, "energies_per_gpu": args.ne,
                           "eta": 1e-6, "mu_l": 0.1, "mu_r": -0.1, "kT": 0.025, "precision": "mixed",
                           "parallelism": "energies sharded across ranks, no collective" if world > 1 else "1 GPU",
                           "l2": "inputs larger than L2: %.1f GB device working set per pass" %
                                 (stats["workspace_bytes"] / 1e9)},
                "accuracy_vs_fp64": {"max_block_rel_err_GR": errs[0], "max_block_rel_err_GL": errs[1],
                                     "max_T_err": t_err, "energies_checked": len(checked), "bar": 1e-10},
                "accuracy_vs_oracle": acc_oracle,
                "p50_s": serving["p50_s"] if serving else None, "p99_s": serving["p99_s"] if serving else None,
                "serving": serving,
                "roofline": roof, "kernels": breakdown_of(prof), "whole_step": whole, "clocks": clk.summary(),
                "gpu_launches": int(stats["launches"]) * args.steps,
                "e2e": e2e, "cpu_baseline": cpu, "fp64_path": fp64,
                "method": "3M complex products of 7-digit base-256 int8 splits of 54-bit fixed-point rows (28 digit "
                          "pairs per real product) on tcgen05.mma kind::i8 with exact int32 TMEM accumulation; "
                          "FP64 Gauss-Jordan inversions"}
        print(json.dumps(line), flush=True)
    solver.close()
    dev.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_cfg3(args):
    """Selected inverse of M(E) for many energies: N = 64 layers of b = 512
    (--npl / --b), 128 energies (--ne) uniform in [-1, 1], the same H / Sigma
    generator (seed 0), by DDRGF with four partitions (interior size 15:
    separators at layers 0, 16, 32, 48), by the block selected inverse
    (Block_factorization! + Block_inverse!, lu(NoPivot()) diagonal blocks) and
    by sequential RGF, each in FP64 and in the mixed precision mode.  A step is
    one pass over all energies through negf_device_selected_inverse with
    device outputs, in chunks of --chunk energies (planning and workspace
    allocation inside the timed region); accuracy: the mixed outputs against
    the FP64 GPU outputs on the first chunk and against the oracle's sequential
    RGF on one energy."""
    import ctypes
    import torch
    import libnegf_b200 as negf
    from libnegf_b200 import _lib
    from oracle import physics, rgf as o_rgf
    npl, b, ne, chunk = args.npl, args.b, args.ne, args.chunk
    sysm = physics.physics_system(npl, b, seed=0)
    dev = negf.Device(sysm.Hd, sysm.Hu, sysm.sigL, sysm.sigR)
    E = np.linspace(-1.0, 1.0, ne)
    sd, su = npl * b * b, (npl - 1) * b * b
    gd = torch.empty(2 * chunk * sd, dtype=torch.float64, device="cuda")
    gu = torch.empty(2 * chunk * su, dtype=torch.float64, device="cuda")
    gl = torch.empty(2 * chunk * su, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    lib = negf.load()
    d1 = max(1, (npl - 4) // 4)  # four partitions: 4 (d1 + 1) = npl
    methods = {"ddrgf": (_lib.NEGF_METHOD_DDRGF, [d1]), "selinv": (_lib.NEGF_METHOD_SELINV, []),
               "rgf": (_lib.NEGF_METHOD_RGF, [])}

    def one_chunk(method, precision, e0):
        m, lv = methods[method]
        cnt = min(chunk, ne - e0)
        o = negf.make_opts(sysm.eta, max_chunk=cnt, precision=precision)
        Ec = np.ascontiguousarray(E[e0:e0 + cnt])
        _lib.check(lib.negf_device_selected_inverse(
            dev.handle, cnt, Ec.ctypes.data_as(_lib.c_double_p), ctypes.byref(o), m, len(lv),
            _lib.int_array(lv) if lv else None, gd.data_ptr(), gu.data_ptr(), gl.data_ptr(), 1,
            ctypes.c_void_p(stream.cuda_stream)))

    def host_blocks(t, n_blocks, e):
        z = t.view(-1, 2)[e * n_blocks * b * b:(e + 1) * n_blocks * b * b].cpu().numpy()
        z = z[:, 0] + 1j * z[:, 1]
        return [z[i * b * b:(i + 1) * b * b].reshape(b, b, order="F") for i in range(n_blocks)]

    res = {}
    ref_chunk = {}
    clk = ClockSampler(torch.cuda.current_device())
    with clk:
        for method in [x for x in args.methods.split(",") if x]:
            for precision in ("fp64", "mixed"):
                one_chunk(method, precision, 0)  # warm-up (kernel attributes, first allocations)
                times = []
                for _ in range(args.steps):
                    t0 = time.perf_counter()
                    for e0 in range(0, ne, chunk):
                        one_chunk(method, precision, e0)
                    times.append(time.perf_counter() - t0)
                t = float(np.median(times))
                # accuracy on the first chunk: mixed vs the FP64 GPU path, both vs the oracle on energy 0
                one_chunk(method, precision, 0)
                outs = [host_blocks(gd, npl, 0), host_blocks(gu, npl - 1, 0), host_blocks(gl, npl - 1, 0)]
                ref_chunk[(method, precision)] = outs
                res[(method, precision)] = {"pts_per_s": ne / t, "s_per_step": t}
    # the oracle's sequential RGF on energy 0 (the CPU restatement of bndiag_of_inv_rgf_local!)
    G = o_rgf.bndiag_of_inv_rgf_local(sysm.M_of_E(E[0]))
    ref = [[G.M[(i, i)] for i in range(npl)], [G.M[(i, i + 1)] for i in range(npl - 1)],
           [G.M[(i + 1, i)] for i in range(npl - 1)]]

    def err(a, r):
        return max(max(np.linalg.norm(x - y) / np.linalg.norm(y) for x, y in zip(pa, pr)) for pa, pr in zip(a, r))

    lines = {}
    for (method, precision), v in res.items():
        acc = {"vs_oracle_rgf_energy0": err(ref_chunk[(method, precision)], ref)}
        if precision == "mixed" and (method, "fp64") in ref_chunk:
            acc["vs_fp64_gpu_energy0"] = err(ref_chunk[(method, precision)], ref_chunk[(method, "fp64")])
        v["accuracy"] = acc
        lines.setdefault(method, {})[precision] = v
    for method, d in lines.items():
        if "fp64" in d and "mixed" in d:
            d["speedup_mixed_vs_fp64"] = d["mixed"]["pts_per_s"] / d["fp64"]["pts_per_s"]
    head = lines.get("ddrgf", next(iter(lines.values())))
    print(json.dumps({"metric": "energy pts/s (selected inverse of M(E): DDRGF, block selected inverse, RGF)",
                      "value": head["mixed"]["pts_per_s"] if "mixed" in head else None, "unit": UNIT,
                      "n_gpus": 1, "steps": args.steps, "dtype": "int8 products / f64",
                      "data": "synthetic (seeded numpy generator of the config)",
                      "config": {"workload": "batched selected inverse + DDRGF, N=%d layers x b=%d, %d energies, "
                                             "four partitions (interior size %d)" % (npl, b, ne, d1),
                                 "chunk": chunk, "headline": "ddrgf, mixed"},
                      "methods": lines, "clocks": clk.summary()}), flush=True)
    dev.close()


def run_cfg4(args):
    """Uneven batch: seeded systems with N ~ U{8..96}, b in {32,64,128,192,256,384}
    (first = last block for T), 16 energies each, through the budget-packed
    scheduler with autotuned knobs; device time of the solves only."""
    import torch
    import libnegf_b200 as negf
    from libnegf_b200.batch import solve_uneven
    from oracle import physics
    rng = np.random.default_rng(4)
    specs = [(int(rng.integers(8, 97)), int(rng.choice([32, 64, 128, 192, 256, 384]))) for _ in range(args.systems)]
    devs = []
    for k, (n, b) in enumerate(specs):
        s = physics.physics_system(n, b, seed=1000 + k)
        devs.append(negf.Device(s.Hd, s.Hu, s.sigL, s.sigR))
    energies = [np.linspace(-0.9, 0.9, 16) + 1e-3 * k for k in range(len(devs))]
    flops = sum(canonical_flops(n, b) * 16 for n, b in specs)
    clk = ClockSampler(torch.cuda.current_device())
    with clk:
        st = solve_uneven(devs, energies, precision=args.precision, eta=1e-6)
    print(json.dumps({"metric": "energy pts/s (uneven batch)", "value": st["pts_per_s_device"], "unit": UNIT,
                      "wall_pts_per_s": st["pts_per_s_wall"], "n_gpus": 1, "dtype": args.precision,
                      "data": "synthetic (seeded)",
                      "config": {"workload": "uneven batch, %s%d systems (N in U{8..96}, b in "
                                             "{32,64,128,192,256,384}), 16 energies each" %
                                             ("" if len(devs) >= 512 else "bounded sample of ", len(devs)),
                                 "groups": st["groups"], "budget_gb": st["budget_bytes"] / 1e9,
                                 "knobs": st["knobs"]},
                      "energy_points": st["energy_points"], "device_ms": st["device_ms"],
                      "algorithmic_tflops": flops / (st["device_ms"] / 1000.0) / 1e12,
                      "tuning_ms_per_pass": [(c, t) for c, t in (st["tuning"] or [])],
                      "clocks": clk.summary()}), flush=True)
    for d in devs:
        d.close()


def request_stream(n_req, rate, seed, npl_range, b_choices, ne_range, ne_div=1):
    """Seeded requests (N uniform in npl_range, b from b_choices, energy lists
    of ne_range // ne_div points, the H / Sigma generator with a per-request
    seed) and their Poisson inter-arrival gaps at `rate` requests/s."""
    from oracle import physics
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n_req):
        n = int(rng.integers(npl_range[0], npl_range[1] + 1))
        b = int(rng.choice(b_choices))
        ne = max(1, int(rng.integers(ne_range[0], ne_range[1] + 1)) // ne_div)
        s = physics.physics_system(n, b, seed=seed * 1000 + k)
        reqs.append((s, np.linspace(-0.9, 0.9, ne)))
    return reqs, rng.exponential(1.0 / rate, size=n_req)


def serve_stream(reqs, gaps, precision, lanes=4, receive="pinned"):
    """Submit the requests at their arrival times to the library's request
    server (negf_server_*, continuous batching over `lanes` streams) and wait
    for all; latency = entry into submit to completion.  receive="pinned": the
    client's receive buffers (G^R, G^< diagonal blocks and T of every request)
    are pinned host memory allocated before the stream starts, so results
    arrive at DMA speed; "fresh": new pageable arrays per request (their pages
    are first touched by the copy)."""
    from libnegf_b200.server import NativeServer
    outs, keep = [None] * len(reqs), []
    if receive == "pinned":
        import torch
        for k, (s, E) in enumerate(reqs):
            n = len(E) * sum(int(h.shape[0]) ** 2 for h in s.Hd)
            gr = torch.empty(n, dtype=torch.complex128, pin_memory=True)
            gl = torch.empty(n, dtype=torch.complex128, pin_memory=True)
            keep += [gr, gl]
            outs[k] = (gr.numpy(), gl.numpy(), np.empty(len(E)))
    srv = NativeServer(lanes=lanes, precision=precision, eta=1e-6)
    try:
        tickets = []
        t0 = time.perf_counter()
        for (s, E), gap, out in zip(reqs, gaps, outs):
            time.sleep(gap)
            tickets.append(srv.submit(s.Hd, s.Hu, s.sigL, s.sigR, E, want_blocks=True, out=out))
        for tk in tickets:
            tk.wait(timeout=1800)
        wall = time.perf_counter() - t0
        st = srv.stats()
    finally:
        srv.close()
    pts = sum(len(E) for _, E in reqs)
    return {"pts_per_s": pts / wall, "p50_s": st["p50_s"], "p99_s": st["p99_s"], "requests": st["requests"],
            "energy_points": pts, "wall_s": wall, "groups": st["groups"],
            "peak_inflight_groups": st["peak_inflight_groups"], "lanes": lanes, "precision": precision,
            "receive_buffers": {"pinned": "pinned host memory allocated before the stream",
                                "fresh": "new pageable arrays per request"}[receive]}


def run_cfg5(args):
    """Request stream: seeded requests (N in {16..128}, b in {64..512}, energy
    lists of 32..1024 scaled to a bounded sample) arriving as a Poisson process
    at --rate, served by the library's request server (four lanes, continuous
    batching) in FP64 and in the mixed precision mode; latency = entry into
    submit to completion."""
    import torch
    reqs, gaps = request_stream(args.requests, args.rate, 5, (16, 128), [64, 128, 192, 256, 384, 512], (32, 1024),
                                ne_div=8)
    clk = ClockSampler(torch.cuda.current_device())
    res = {}
    with clk:
        for precision in ("fp64", "mixed"):
            res[precision] = serve_stream(reqs, gaps, precision, receive="fresh")  # up to ~140 GB per request
    print(json.dumps({"metric": "energy pts/s and p50/p99 solve latency (request stream)",
                      "value": res["mixed"]["pts_per_s"], "unit": UNIT, "p50_s": res["mixed"]["p50_s"],
                      "p99_s": res["mixed"]["p99_s"], "n_gpus": 1, "dtype": "int8 products / f64",
                      "data": "synthetic (seeded)",
                      "config": {"workload": "bounded sample of the request stream: %d requests, N in {16..128}, "
                                             "b in {64..512}, energy lists of 4..128 (1/8 of 32..1024), Poisson "
                                             "arrivals at %.2f/s" % (len(reqs), args.rate)},
                      "by_precision": res, "clocks": clk.summary()}), flush=True)


def spawn_ranks(args):
    """--gpus N without a launcher: start N ranks (one per GPU) through
    torch.distributed.run on this node and return the launcher's exit code."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args))
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "cfg3":
        run_cfg3(args)
    elif args.workload == "cfg4":
        run_cfg4(args)
    elif args.workload == "cfg5":
        run_cfg5(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
