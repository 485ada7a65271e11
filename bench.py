"""Benchmark of the fiber3d hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload stresslet_sphere|oseen_fibers]

Default workload ``stresslet_sphere`` (the double-layer sum on a spherical
periphery): 12000 Fibonacci-sphere nodes of radius 10 (outward normals, equal
weights 4 pi R^2/N, density N(0,1) times the weight) summed onto the 12000
nodes themselves (pair j == i skipped, as in
stresslet_kernel_times_normal_times_density_numba) and onto 4096 points
uniform in a ball of radius 9 (stresslet_kernel_source_target_numba): one
step = 12000*11999 + 12000*4096 = 193,140,000 pair interactions, FP64.

Metric: Stokes pair interactions per second (whole job; N GPUs run N
replicas — the workload does not shard on one node in this tier).
``value`` is measured with inputs resident in HBM, one CUDA-event pair per
step on the launching stream, L2 flushed (256 MiB write) between steps
outside the event pairs.  ``e2e`` is the same metric through the drop-in
Python API (fiber3d_b200.kernels) from pinned host buffers, host<->device
copies inside the timed region.  ``--impl reference`` times fiber3d's CPU
algorithm for the same workload (the C/OpenMP restatement in oracle/) on
the host cores, on a bounded sample of targets.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FLOP_PER_PAIR = {"stresslet": 29, "oseen": 28, "rotlet": 25}
L2_FLUSH_BYTES = 256 << 20


# ------------------------------------------------------------------ setup --
def dist_info():
    from fiber3d_b200 import replicas
    return replicas.rank_info()


def make_workload(name: str):
    from fiber3d_b200 import geometry
    if name == "stresslet_sphere":
        nodes, normals, w, mu, vol = geometry.stresslet_sphere_workload(seed=2)
        q = mu * w[:, None]
        n = nodes.shape[0]
        targets = np.concatenate([nodes, vol])
        grp_t = np.concatenate([np.arange(n), -np.ones(vol.shape[0])]).astype(np.int32)
        grp_s = np.arange(n, dtype=np.int32)
        pairs = n * (n - 1) + n * vol.shape[0]
        return dict(kind="stresslet", src=nodes, trg=targets, dens=q, nrm=normals, gs=grp_s,
                    gt=grp_t, pairs=pairs, nodes=nodes, vol=vol, w=w,
                    desc="stresslet double layer, 12000-node sphere R=10 -> 12000 nodes "
                         "(j==i skipped, then the O(N) singularity subtraction of the periphery "
                         "operator) + 4096 ball points R=9, FP64")
    if name == "oseen_fibers":
        x, f = geometry.oseen_fiber_workload(seed=1)
        n = x.shape[0]
        grp = np.arange(n, dtype=np.int32)
        return dict(kind="oseen", src=x, trg=x, dens=f, nrm=None, gs=grp, gt=grp,
                    pairs=n * (n - 1), nodes=x, vol=None,
                    desc="Oseen sum, 32 straight fibers x 32 Chebyshev-Lobatto nodes, "
                         "j==i skipped, FP64")
    raise SystemExit(f"unknown workload {name}")


def workload_config(name: str, wl) -> dict:
    """The `config` of a pair-sum line; identical in both arms."""
    return {"workload": name, "description": wl["desc"], "pairs_per_step": wl["pairs"],
            "l2": "flushed between steps (256 MiB write, outside the event pairs)"}


def host_cores() -> dict:
    """Threads the CPU legs use and the host's physical cores."""
    from oracle import pairs_c
    try:
        import psutil
        phys = psutil.cpu_count(logical=False)
    except Exception:  # noqa: BLE001
        phys = None
    return {"threads": pairs_c.max_threads(), "physical_cores": phys, "logical_cpus": os.cpu_count()}


class ClockSampler:
    """Samples SM clock, power and throttle reasons through NVML every 10 ms
    in a background thread while the timed region runs (reads only)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self.max_mhz = None
        self._stop = None
        self._thread = None
        self.error = None

    def __enter__(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nvml = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # noqa: BLE001 - report, never fail the bench
            self.error = f"nvml unavailable: {e}"
            return self
        self._stop = threading.Event()

        def run():
            nv = self._nvml
            while not self._stop.is_set():
                try:
                    sm = nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                    self.samples.append((sm, rs))
                except Exception:  # noqa: BLE001
                    pass
                self._stop.wait(0.01)

        self._sample()
        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        return self

    def _sample(self):
        try:
            nv = self._nvml
            self.samples.append((nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM),
                                 nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)))
        except Exception:  # noqa: BLE001
            pass

    def __exit__(self, *exc):
        if self._thread is not None:
            self._sample()
            self._stop.set()
            self._thread.join(timeout=2)

    def summary(self):
        if self.error:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.error]}
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["no samples"]}
        sm = [s for s, _ in self.samples]
        reasons = sorted({k for _, r in self.samples for k, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sm), "source": "NVML every 10 ms during the timed region"}


# -------------------------------------------------------------- GPU arm ---
def measured_peak(L, precision: str, torch, gpu_index: int = 0):
    """FMA throughput (FLOP/s) of this GPU from the library's probe kernel,
    with the SM clock sampled while it runs."""
    import ctypes
    sink = torch.zeros(1, dtype=torch.float64, device="cuda")
    flops = ctypes.c_double(0)
    st = L.stream_handle()
    prec = {"fp64": 0, "fp32c": 1, "fp64_mma": 2}[precision]
    for _ in range(2):
        L.call("f3d_probe_fma", prec, 2000, L.ptr(sink), ctypes.byref(flops), st)
    torch.cuda.synchronize()
    best = 0.0
    with ClockSampler(gpu_index) as clk:
        for _ in range(8):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            L.call("f3d_probe_fma", prec, 2000, L.ptr(sink), ctypes.byref(flops), st)
            e1.record()
            e1.synchronize()
            best = max(best, flops.value / (e0.elapsed_time(e1) * 1e-3))
    return best, clk.summary()


def gpu_arm(args, rank, world, local):
    import torch
    from fiber3d_b200 import _lib as L
    from fiber3d_b200 import replicas
    from fiber3d_b200 import kernels as K

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    wl = make_workload(args.workload)
    kind = wl["kind"]
    to = lambda a, dt=torch.float64: torch.as_tensor(a, dtype=dt, device=dev).contiguous()
    src, trg, dens = to(wl["src"]), to(wl["trg"]), to(wl["dens"])
    nrm = to(wl["nrm"]) if wl["nrm"] is not None else None
    gs, gt = to(wl["gs"], torch.int32), to(wl["gt"], torch.int32)
    out = torch.empty(trg.numel(), dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    # one launch over one array: targets = [nodes; ball points], sources =
    # its first n points (the nodes), the pair j == i skipped; the autotuner
    # chooses among the regular launch shapes and (FP64) the symmetric form,
    # which evaluates each node pair once and the ball points one-sided
    from fiber3d_b200 import autotune
    src = trg[:dens.shape[0]]
    shapes = {p: autotune.tune(kind, src, trg, dens, nrm, self_mode="skip_index", precision=p)
              for p in ("fp64", "fp32c")}
    launches_per_step = 1

    def pair_sums(precision):
        K.pair_sum(kind, src, trg, dens, nrm, self_mode="skip_index", precision=precision, out=out,
                   shape=shapes[precision])

    subtract = None
    if kind == "stresslet":
        # the periphery operator's rows on the node targets (tstep.py:1097-1104):
        # res = v - E mu - mu + n sum(n.q), E the singularity-subtraction vectors
        from fiber3d_b200.hydro import singularity_vectors
        n_nodes = wl["nodes"].shape[0]
        wts = to(wl["w"])
        E = singularity_vectors(src, nrm, wts, 1.0, 5e-3, 1e-5)
        res = torch.empty(3 * n_nodes, dtype=torch.float64, device=dev)
        scratch = torch.zeros(1, dtype=torch.float64, device=dev)
        launches_per_step += 1

        def subtract():
            L.call("f3d_shell_residual", L.ptr(out), L.ptr(E), L.ptr(wts), L.ptr(nrm), L.ptr(dens), L.ptr(res),
                   n_nodes, L.ptr(scratch), L.stream_handle(dev))

    def step(precision="fp64"):
        pair_sums(precision)
        if subtract is not None:
            subtract()

    def timed(precision, steps, warmup, kernel_times=None):
        """Per-step device times (ms); with kernel_times, also the pair
        kernel's own time in each step (an event between the two launches)."""
        for _ in range(warmup):
            step(precision)
        torch.cuda.synchronize()
        replicas.barrier()
        torch.cuda.synchronize()
        evs = []
        for _ in range(steps):
            flush.fill_(1)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            torch.cuda.nvtx.range_push(f"timed_pairs_{precision}")
            e0.record()
            pair_sums(precision)
            e1.record()
            if subtract is not None:
                subtract()
            e2.record()
            torch.cuda.nvtx.range_pop()
            evs.append((e0, e1, e2))
        torch.cuda.synchronize()
        replicas.barrier()
        if kernel_times is not None:
            kernel_times.extend(a.elapsed_time(b) for a, b, _ in evs)
        return [a.elapsed_time(c) for a, _, c in evs]

    peak64, peak64_clocks = measured_peak(L, "fp64", torch, local)
    peak32, _ = measured_peak(L, "fp32c", torch, local)
    kern_ms = []
    with ClockSampler(local) as clk:
        t_ms = timed("fp64", args.steps, args.warmup, kernel_times=kern_ms)
    clocks = clk.summary()
    total_ms, = replicas.max_over_ranks([sum(t_ms)], dev)
    ms_step = total_ms / args.steps
    pairs = wl["pairs"]
    value = replicas.aggregate_rate(pairs, args.steps, world, total_ms)

    # the timed launches' output against the library-default launch shape
    timed_out = out.clone()
    K.pair_sum(kind, src, trg, dens, nrm, self_mode="skip_group", src_group=gs, trg_group=gt,
               precision="fp64", out=out)
    ref64 = out.clone()
    check64 = float((timed_out - ref64).abs().max() / ref64.abs().max())
    # FP32-compensated variant of the same step and its error vs FP64
    t32 = timed("fp32c", args.steps, args.warmup)
    err32 = float((out - ref64).abs().max() / ref64.abs().max())
    ms32 = sum(t32) / len(t32)

    # e2e through the drop-in API from pinned host buffers
    host = {k: torch.as_tensor(wl[k]).pin_memory() for k in ("nodes", "dens", "nrm", "vol") if wl[k] is not None}
    nbytes = lambda *ks: sum(host[k].numel() * host[k].element_size() for k in ks)
    # what the calls below copy to the device: each call its own inputs
    h2d = (nbytes("nodes", "nrm", "dens") + nbytes("nodes", "vol", "nrm", "dens") if kind == "stresslet"
           else nbytes("nodes", "dens"))

    def e2e_step():
        if kind == "stresslet":
            a = K.stresslet_kernel_times_normal_times_density_numba(host["nodes"], host["nrm"], host["dens"])
            b = K.stresslet_kernel_source_target_numba(host["nodes"], host["vol"], host["nrm"], host["dens"])
            return a.nbytes + b.nbytes
        a = K.oseen_kernel_times_density_numba(host["nodes"], host["dens"])
        return a.nbytes

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    d2h = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        d2h = e2e_step()
    e1.record()
    e1.synchronize()
    e2e_ms, = replicas.max_over_ranks([e0.elapsed_time(e1)], dev)
    e2e_value = replicas.aggregate_rate(pairs, args.steps, world, e2e_ms)

    flop_pair = FLOP_PER_PAIR[kind]
    kern_avg = sum(kern_ms) / len(kern_ms)
    achieved = flop_pair * pairs / (kern_avg * 1e-3)
    line = {
        "metric": "Stokes pair interactions per second (FP64)",
        "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": workload_config(args.workload, wl),
        "parallelism": f"replicas x{world}",
        "launch_shape": {p: [v.tpt, v.sl, v.nsplit, v.use_tma] for p, v in shapes.items()},
        "roofline": {"bound": "fp64", "achieved": achieved / 1e12, "peak": peak64 / 1e12,
                     "unit": "TFLOP/s", "frac": achieved / peak64,
                     "kernel_ms_avg": kern_avg,
                     # DRAM bytes per launch of this kernel on this workload, from an ncu capture
                     # of it: symmetric form read 997.9 KB + write 29.2 KB (its tile partials stay
                     # in L2); one-sided form read 1.391 MB, write 0
                     "traffic": (None if args.workload != "stresslet_sphere"
                                 else 1027072 if shapes["fp64"].sl == -1 else 1391104),
                     "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                     "note": f"{flop_pair} algorithmic flop per ordered pair (rsqrt not counted; the "
                             "symmetric form evaluates each unordered pair once for both directions); peak = "
                             "measured FP64 FMA rate of this GPU (f3d_probe_fma), with the SM clock seen "
                             "while it ran",
                     "peak_clocks": peak64_clocks,
                     "kernel": (f"pair_sym_kernel<{kind}, skip_index>" if shapes["fp64"].sl == -1
                                else f"pair_kernel<{kind}, skip_index, fp64>")},
        "timed_output_vs_default_shape_max_rel": check64,
        "fp32c": {"value": pairs / (ms32 * 1e-3) * world, "ms_per_step": ms32,
                  "max_rel_err_vs_fp64": err32, "peak_fp32_tflops": peak32 / 1e12},
        "e2e": {"value": e2e_value, "unit": "pairs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "path": "fiber3d_b200.kernels drop-in calls from pinned host tensors"},
        "clocks": clocks,
        "gpu_launches": args.steps * launches_per_step,
    }
    if rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline(wl, seconds=args.cpu_seconds)
    summary = {"cfg2_pairs_fp64": {"ms_per_step": ms_step, "kernel_ms": kern_avg, "gpairs_per_s": value / 1e9,
                                   "e2e_gpairs_per_s": e2e_value / 1e9, "roofline_frac": achieved / peak64,
                                   "fp32c_max_rel_err": err32}}
    if args.workload == "stresslet_sphere" and not args.no_step:
        # the other half of the headline: full time step (512 fibers x 32
        # points, 4 spheres, 12000-node periphery, GMRES rel. residual 1e-8),
        # learned warm start + mixed precision against plain FP64
        st = hydro_arm(args, rank, world, local, warmup=args.step_warmup, steps=args.step_steps,
                       emit=False)["step"]
        line["step"] = {
            "config": "512 fibers x 32 points (L=2, E=0.0025, dt=1e-3), 4 rigid spheres x 400 nodes, "
                      "12000-node periphery R=10, GMRES restart 100, rel. residual 1e-8",
            "steps": args.step_steps, "warmup": args.step_warmup,
            "plain_fp64_ms": st["fp64"]["ms_per_step"],
            "learned_mixed_ms": st["learned_mixed"]["ms_per_step"],
            "speedup_learned_mixed_vs_plain_fp64": st["learned_mixed"]["speedup_vs_fp64"],
            "modes": {m: {k: v[k] for k in ("ms_per_step", "ms_per_step_last_half", "iterations", "long_solves",
                                            "true_rel_residual", "tol", "fiber_pc_rebuilt", "fp64_residuals",
                                            "first_residual_bound_max", "oracle",
                                            "rel_err_vs_fp64_1e-12_solve", "speedup_vs_fp64", "phases_ms")
                          if k in v}
                      for m, v in st.items() if m not in ("training", "grid_velocity")},
            "training": st["training"],
            "grid_velocity": st.get("grid_velocity"),
        }
        s3 = {"fp64_ms": st["fp64"]["ms_per_step"]}
        for m in ("learned_mixed", "learned_mixed_tol1e-9", "extrapolate_mixed", "flownet_mixed"):
            if m not in st:
                continue
            s3[f"{m}_ms"] = st[m]["ms_per_step"]
            s3[f"{m}_iterations_total"] = int(sum(st[m]["iterations"]))
            s3[f"{m}_speedup"] = st[m]["speedup_vs_fp64"]
            s3[f"{m}_err_vs_fp64_solve"] = st[m]["rel_err_vs_fp64_1e-12_solve"]
        for m in ORACLE_MODES:
            o = st[m].get("oracle")
            if o:
                s3[f"{m}_oracle_true_residual"] = o["true_rel_residual"]
        cpu = st["fp64"].get("oracle", {}).get("cpu_step")
        if cpu:
            s3["cpu_step_s"] = cpu["value_s"]
            s3["cpu_threads"] = cpu["threads"]
        s3["learned_correction_scale"] = st["training"]["scale"]
        fn = st["training"].get("flownet")
        if fn:
            s3["flownet_heldout_rel_err"] = fn["heldout_rel_err"]
            s3["flownet_true_map_residual_median"] = float(np.median(fn["true_map_initial_rel_residual"]))
        summary["cfg3_step"] = s3
        # config 4: the batched block-diagonal preconditioner
        bp = block_pc_measure(args, dev, 10, 3, args.cpu_seconds)
        line["block_pc"] = {"config": f"{args.nblocks} fibers, N uniform in {{16,24,32,48,64}}, 4N x 4N blocks, "
                                      "factor + solve in one CUDA graph", **bp}
        summary["cfg4_block_pc"] = {k: bp[k] for k in ("ms", "gflops", "max_rel_err_vs_scipy", "cpu_ms", "cpu_cores")}
        # config 1: the 1024-point Oseen sum
        of = oseen_fibers_measure(args, dev, 50, 5, args.cpu_seconds)
        line["oseen_fibers"] = {"config": "32 fibers x 32 Chebyshev-Lobatto nodes, Oseen j != i, FP64", **of}
        summary["cfg1_oseen_1024"] = {k: of[k] for k in ("us_per_call", "hbm_gbs", "e2e_us_per_call",
                                                         "cpu_pairs_per_s")}
    # last, so that a tail of the line carries it
    line["summary"] = summary
    if rank == 0:
        print(json.dumps(line), flush=True)


# -------------------------------------------------------------- CPU arm ---
def cpu_sample_rate(wl, nthreads: int, seconds: float):
    """Pairs/s of the C/OpenMP restatement of fiber3d's kernel on a prefix of
    the targets, grown until one sample takes >= 1 s, repeated for ~seconds."""
    from oracle import pairs_c
    kind, src, trg, dens, nrm = wl["kind"], wl["src"], wl["trg"], wl["dens"], wl["nrm"]
    nt = 64
    while True:
        t0 = time.perf_counter()
        pairs_c.pair_sum(kind, src, trg[:nt], dens, nrm, nthreads=nthreads)
        dt = time.perf_counter() - t0
        if dt >= 1.0 or nt >= trg.shape[0]:
            break
        nt = min(trg.shape[0], nt * 2)
    reps, best = 0, float("inf")
    t_start = time.perf_counter()
    while time.perf_counter() - t_start < seconds or reps == 0:
        t0 = time.perf_counter()
        pairs_c.pair_sum(kind, src, trg[:nt], dens, nrm, nthreads=nthreads)
        best = min(best, time.perf_counter() - t0)
        reps += 1
    return nt * src.shape[0] / best, nt, reps


def cpu_baseline(wl, seconds: float):
    hc = host_cores()
    rate, nt, reps = cpu_sample_rate(wl, hc["threads"], seconds)
    return {"value": rate, "unit": "pairs/s", "cores": hc["threads"], **hc, "kind": "port",
            "sample": f"{nt} of {wl['trg'].shape[0]} targets x {wl['src'].shape[0]} sources, "
                      f"best of {reps}; C/OpenMP restatement of fiber3d's numba loop "
                      "(cores = OpenMP threads used)"}


def fmm_reference_arm(args, world):
    """The FMM workload's reference: fiber3d's direct numba sums (what its
    STKFMM path is checked against; STKFMM itself is not available), restated
    in C/OpenMP, on all host threads, over a target sample per step."""
    from oracle import pairs_c
    n = args.fmm_n
    w = fmm_workload(n, seed=0)
    hc = host_cores()
    nt = max(16, min(n, int(2e9 / (2 * n))))  # about 1 s of CPU work per step
    rates = []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        pairs_c.pair_sum("oseen", w["sl"], w["trg"][:nt], w["f"], epsilon_distance=0.0, reg=0.0)
        pairs_c.pair_sum("stresslet", w["dl"], w["trg"][:nt], w["dens"], w["nrm"], epsilon_distance=0.0, reg=0.0)
        if step >= args.warmup:
            rates.append(2 * n * nt / (time.perf_counter() - t0))
    value = statistics.median(rates)
    line = {
        "impl": "reference",
        "metric": f"FMM equivalent Stokes pair interactions per second (FP64, order {args.fmm_order})",
        "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 2 * n * n / value * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded): fiber3d's STKFMM check shape (kernels/test_stkfmm.py)",
        "config": {"workload": "fmm", "n_single_layer": n, "n_double_layer": n, "n_targets": n,
                   "cube_side": w["side"], "order": args.fmm_order, "max_pts": args.fmm_max_pts,
                   "l2": "flushed between steps (256 MiB write, outside the event pairs)"},
        "parallelism": f"host cores (rank 0 of {world})",
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": hc["threads"], **hc, "kind": "port",
                         "sample": f"direct sums onto {nt} of {n} targets per step (C/OpenMP restatement of "
                                   "fiber3d's numba loops; STKFMM, fiber3d's CPU FMM, is not installed)"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def dense_inverse_reference_arm(args, world):
    """The dense_inverse workload's reference: fiber3d's scipy.linalg.lu_factor
    of the dense shell operator (tstep.py:348) on the host cores, the operator
    built by the oracle's restatement (tstep.py:327-347) for a sphere of
    args.dense_cpu_nodes nodes and the time scaled by the cube of the size."""
    import scipy.linalg as sla
    from fiber3d_b200 import geometry
    from oracle import kernels_np as KN, system as S
    ns = max(200, min(args.nshell, int(args.dense_cpu_nodes)))
    nodes, normals = geometry.fibonacci_sphere(ns, args.shell_radius)
    w = np.full(ns, 4.0 * np.pi * args.shell_radius ** 2 / ns)
    E = S.singularity_vectors(nodes, normals, w, 1.0)
    M = KN.stresslet_kernel_times_normal_dense(nodes, normals, eta=1.0)
    for i in range(ns):
        M[3 * i:3 * i + 3, 3 * i:3 * i + 3] -= E[i] / w[i] + np.eye(3) / w[i]
    M += KN.complementary_kernel(None, normals)
    times = []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        sla.lu_factor(M)
        if step >= args.warmup:
            times.append(time.perf_counter() - t0)
    m, ms_ = 3 * args.nshell, 3 * ns
    value = statistics.median(times) * (m / ms_) ** 3 * 1e3
    hc = host_cores()
    line = {"impl": "reference", "metric": "periphery preconditioner set-up: dense inverse (ms)", "value": value,
            "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": value,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (Fibonacci sphere)",
            "config": {"workload": "dense_inverse", "nodes": int(args.nshell), "matrix": int(m),
                       "radius": args.shell_radius},
            "parallelism": f"host cores (rank 0 of {world})",
            "cpu_baseline": {"value": value, "unit": "ms", "cores": hc["threads"], **hc, "kind": "reference",
                             "sample": f"scipy.linalg.lu_factor of the {ms_} x {ms_} operator of a {ns}-node "
                                       f"sphere, scaled by ({m}/{ms_})^3"},
            "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def reference_arm(args, rank, world):
    if rank != 0:
        return
    if args.workload == "dense_inverse":
        dense_inverse_reference_arm(args, world)
        return
    if args.workload == "surface_quadrature":
        quadrature_reference_arm(args, world)
        return
    if args.workload == "fmm":
        fmm_reference_arm(args, world)
        return
    wl = make_workload(args.workload)
    hc = host_cores()
    threads = hc["threads"]
    per_step = max(1.0, args.cpu_seconds / max(args.steps, 1))
    rates = []
    for _ in range(args.warmup):
        cpu_sample_rate(wl, threads, 0.0)
    for _ in range(args.steps):
        r, nt, _ = cpu_sample_rate(wl, threads, per_step)
        rates.append(r)
    value = statistics.median(rates)
    line = {
        "impl": "reference",
        "metric": "Stokes pair interactions per second (FP64)", "value": value, "unit": "pairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wl["pairs"] / value * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": workload_config(args.workload, wl),
        "parallelism": f"host cores (rank 0 of {world})",
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, **hc, "kind": "port",
                         "sample": f"{nt} targets x {wl['src'].shape[0]} sources per step sample; "
                                   "C/OpenMP restatement of fiber3d's numba loop (oracle/)"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# modes whose first timed step is checked against the CPU oracle
ORACLE_MODES = ("fp64", "learned_mixed", "learned_mixed_tol1e-9")


def step_oracle(P, snap, cpu_time=False, iterations=None):
    """The CPU oracle's matrix-free restatement of fiber3d's step
    (oracle/system.py) at a marched step's geometry: the true relative
    residual ||b - A x|| / ||b|| of the device solution x with the ORACLE's
    A and b, the device right-hand side against the oracle's, and the device
    solution against the device FP64 solve to 1e-12.  With cpu_time, fiber3d's
    method timed on the host (the step's CPU baseline): building the system
    (explicit flows, right-hand side, fiber operators and their LU, the
    singularity vectors), one matvec, one fiber+body preconditioner apply,
    and the periphery LU apply estimated from a dense 12000^2 matvec scaled to
    (3 Nshell)^2 (memory bound, like the two triangular solves of lu_solve);
    total = build + (iterations + 1) x (matvec + preconditioner)."""
    from oracle import system as S
    from fiber3d_b200.hydro import quaternion_rotation
    n_f = [np.asarray(f).reshape(-1, 3).shape[0] for f in P.fibers]
    offs = np.concatenate([[0], np.cumsum(n_f)])
    xf = snap["x_fib"].reshape(-1, 3)
    fibers = [xf[offs[k]:offs[k + 1]] for k in range(len(n_f))]
    rots = [quaternion_rotation(q) for q in snap["quats"]]
    t0 = time.perf_counter()
    op = S.system_at(P, fibers, snap["locs"], rots)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    res = op.true_residual(snap["sol"])
    t_mv = time.perf_counter() - t0
    out = {"true_rel_residual": res,
           "rhs_rel_err_vs_oracle": float(np.max(np.abs(snap["rhs"] - op.rhs)) / np.max(np.abs(op.rhs))),
           "fp64_1e-12_solve_true_rel_residual": op.true_residual(snap["ref"]),
           "geometry": "first timed step (marched)"}
    if cpu_time:
        x = snap["sol"]
        t0 = time.perf_counter()
        op.pc(x)
        t_pc = time.perf_counter() - t0
        m = 12000
        A = np.random.default_rng(0).random((m, m))
        v = np.ones(m)
        A @ v
        t0 = time.perf_counter()
        for _ in range(3):
            A @ v
        t_small = (time.perf_counter() - t0) / 3
        del A
        t_shell = t_small * (3 * op.nshell / m) ** 2
        its = iterations if iterations is not None else 4
        total = t_build + (its + 1) * (t_mv + t_pc + t_shell)
        out["cpu_step"] = {"value_s": total, "build_s": t_build, "matvec_s": t_mv, "pc_fibers_bodies_s": t_pc,
                           "pc_shell_est_s": t_shell, "iterations": its, **host_cores(),
                           "kind": "port", "how": "oracle/system.py (C/OpenMP pair sums + numpy/scipy) on the "
                                                 "host; build + (iterations+1) x (matvec + PC), shell PC "
                                                 "apply scaled from a 12000^2 dense matvec"}
    return out


def hydro_arm(args, rank, world, local, warmup=None, steps=None, emit=True):
    """Time steps of the full problem (512 fibers x 32 points, 4 rigid
    spheres of 400 nodes, 12000-node periphery of radius 10; GMRES restart
    100 to relative residual 1e-8), marching in time: each timed step moves
    the geometry with the previous solution (fibers, bodies), rebuilds the
    explicit flows, right-hand side and fiber/body blocks, factors the block
    preconditioner and solves.  Plain FP64 and mixed precision run from the
    same initial state.  The periphery preconditioner (explicit inverse of
    the dense shell operator) is per-run set-up, as in fiber3d's
    tstep.__init__, and is excluded."""
    import torch
    from fiber3d_b200 import geometry, hydro as H, replicas
    warmup = args.warmup if warmup is None else warmup
    steps = args.steps if steps is None else steps
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    P = geometry.hydro_step_problem(seed=3, nshell=args.nshell, nfib=args.nfib, shell_radius=args.shell_radius,
        fiber_ball=args.fiber_ball, body_shell=args.body_shell)
    t0 = time.perf_counter()
    shell = H.ShellOperator(P.shell, P.eta, P.reg, P.eps_dist, dev, pc=args.shell_pc)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    out, xs = {}, {}
    # learned warm start: training pairs (history features -> correction of
    # the quadratic extrapolation) from the solver's own steps on seeds
    # disjoint from the benchmark trajectory; the network is trained on the
    # GPU by the library's kernels
    from fiber3d_b200 import warmstart as W
    t0 = time.perf_counter()
    feats, targs = [], []
    for seed in args.train_seeds:
        Pt = geometry.hydro_step_problem(seed=seed, nshell=args.nshell, nfib=args.nfib,
                                         shell_radius=args.shell_radius,
        fiber_ball=args.fiber_ball, body_shell=args.body_shell)
        st_ = H.HydroSystem(Pt, shell_op=shell, device=dev)
        _, Xf, Tf = W.march(st_, args.train_steps, guess="extrapolate", record=True,
                            record_from=args.train_skip)
        feats.append(Xf)
        targs.append(Tf)
        del st_
    X_train, T_train = torch.cat(feats), torch.cat(targs)
    net = W.LearnedWarmStart(seed=0, device=dev)
    hist = net.fit(X_train, T_train, epochs=args.train_epochs, batch=1024, lr=1e-3)
    # correction factors chosen by GMRES iterations on held-out trajectories
    val_seeds = [max(args.train_seeds) + 1, max(args.train_seeds) + 2]
    Pvs = [geometry.hydro_step_problem(seed=sd, nshell=args.nshell, nfib=args.nfib,
                                       shell_radius=args.shell_radius,
        fiber_ball=args.fiber_ball, body_shell=args.body_shell) for sd in val_seeds]
    sel = net.select_scale(lambda: [H.HydroSystem(Pv, shell_op=shell, device=dev) for Pv in Pvs],
                           args.train_steps, count_from=args.train_skip)
    torch.cuda.synchronize()
    train = {"samples": int(X_train.shape[0]), "seconds": time.perf_counter() - t0,
             "loss_first_last": [hist[0], hist[-1]], "gain": net.gain.tolist(), "scale": net.scale,
             "scale_selection": sel, "validation_seeds": val_seeds,
             "seeds": list(args.train_seeds), "steps_per_seed": args.train_steps,
             "skipped_steps": args.train_skip}
    # mode: (guess, mixed precision, preconditioner refresh interval, GMRES tolerance)
    modes = {"fp64": ("zero", False, 1, 1e-8), "mixed": ("zero", True, 1, 1e-8),
             "extrapolate_fp64": ("extrapolate", False, 1, 1e-8),
             "extrapolate_mixed": ("extrapolate", True, 1, 1e-8),
             "learned_fp64": ("learned", False, 1, 1e-8),
             "learned_mixed_pc1": ("learned", True, 1, 1e-8),
             "learned_mixed": ("learned", True, "auto", 1e-8),
             "learned_mixed_tol1e-9": ("learned", True, "auto", 1e-9),
             "learned_mixed_tol1e-10": ("learned", True, "auto", 1e-10)}
    flow = None
    if not args.no_flownet:
        # the network of the specification's form: (positions, background
        # velocity) -> (tensions, force densities) per fiber, mapped to
        # X^{n+1} through the slender-body mobility; trained on the plain
        # solver's steps of disjoint seeds
        from fiber3d_b200 import flowstart as FS
        t0 = time.perf_counter()
        fx, fy = [], []
        for seed in args.train_seeds[:args.flow_seeds]:
            Pt = geometry.hydro_step_problem(seed=seed, nshell=args.nshell, nfib=args.nfib,
                                             shell_radius=args.shell_radius, fiber_ball=args.fiber_ball,
                                             body_shell=args.body_shell)
            st_ = H.HydroSystem(Pt, shell_op=shell, device=dev)
            _, a, b = FS.march(st_, args.train_steps, guess="extrapolate", record=True, tol=1e-10)
            fx.append(a)
            fy.append(b)
            del st_
        flow = FS.FlowWarmStart(seed=0, device=dev)
        fhist, fval = flow.fit(torch.cat(fx), torch.cat(fy), epochs=args.train_epochs, batch=1024, lr=1e-3)
        # the map itself, with the step's true tensions and forces, on the
        # first steps of a validation trajectory (bounds any network of this form)
        Pv = geometry.hydro_step_problem(seed=max(args.train_seeds) + 1, nshell=args.nshell, nfib=args.nfib,
                                         shell_radius=args.shell_radius, fiber_ball=args.fiber_ball,
                                         body_shell=args.body_shell)
        ov = FS.march(H.HydroSystem(Pv, shell_op=shell, device=dev), 12, guess="extrapolate",
                      oracle_steps=8, record_from=2)
        torch.cuda.synchronize()
        train["flownet"] = {"samples": int(sum(a.shape[0] for a in fx)), "seconds": time.perf_counter() - t0,
                            "seeds": list(args.train_seeds[:args.flow_seeds]),
                            "loss_first_last": [fhist[0], fhist[-1]], "heldout_rel_err": fval,
                            "true_map_initial_rel_residual": [x.get("oracle_map_rel_residual") for x in ov
                                                              if "oracle_map_rel_residual" in x],
                            "extrapolation_initial_rel_residual": [x["initial_rel_residual"] for x in ov[2:10]]}
        modes["flownet_mixed"] = ("flow", True, "auto", 1e-8)
    snap = {}
    for mode, (guess, mixed, pc_refresh, tol) in modes.items():
        sysd = H.HydroSystem(P, shell_op=shell, device=dev, tune=True, pc_refresh=pc_refresh)
        torch.cuda.synchronize()
        replicas.barrier()
        history = []
        times, its, resid, phases, r0s, worst, finals, fresh, fp64r, fbounds = [], [], [], [], [], [], [], [], [], []
        for step in range(warmup + steps):
            torch.cuda.synchronize()
            sysd.timers.report()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            timed_step = step >= warmup
            if timed_step:
                torch.cuda.nvtx.range_push(f"timed_step_{mode}")
            e0.record()
            # the guess needs only the previous solutions: formed first, it is
            # handed to advance(), which sums its Oseen flow in the same pass
            # as the explicit flow
            sysd.timers.start("warm_start")
            x0 = None
            if guess == "extrapolate":
                x0 = W.extrapolate(history)
            elif guess == "learned":
                x0 = W.learned_guess(sysd, history, net)
            elif guess == "flow":
                x0 = flow.guess(sysd, history, u_bg if history else None)
            sysd.timers.stop("warm_start")
            if history:
                sysd.advance(history[-1], x0=x0)
            sysd.timers.start("GMRES")
            refreshed = sysd._pc_age == 0
            res = sysd.solve(tol=tol, restart=100, mixed=mixed, x0=x0)
            sysd.timers.stop("GMRES")
            if guess == "flow":
                # the network's next input: this solution's background velocity
                sysd.timers.start("background_flow")
                u_bg = FS.background_velocity(sysd, res["x"])
                sysd.timers.stop("background_flow")
            e1.record()
            e1.synchronize()
            if timed_step:
                torch.cuda.nvtx.range_pop()
            ph = sysd.timers.report()
            sol = res["x"]
            history = (history + [sol])[-W.HISTORY:]
            if step >= warmup:
                times.append(e0.elapsed_time(e1))
                its.append(res["iterations"])
                if res["iterations"] > 10:  # record the details of an unusually long solve
                    worst.append({"step": step, "iterations": res["iterations"],
                                  "refinements": res.get("refinements", 0),
                                  "fp64_residuals": res.get("fp64_residuals", 0),
                                  "history": [float(f"{h:.3g}") for h in res["history"]]})
                r0s.append(res["history"][0])
                finals.append(res["history"][-1])
                fp64r.append(res.get("fp64_residuals", 0))
                fbounds.append(res.get("first_residual_bound"))
                fresh.append(bool(refreshed))
                phases.append(ph)
                y = torch.empty_like(sol)
                sysd.matvec(sol, y)
                resid.append(float(torch.linalg.vector_norm(y - sysd.rhs) / torch.linalg.vector_norm(sysd.rhs)))
            if step == warmup:
                # accuracy: the same step solved in FP64 from zero to 1e-12
                # (outside the timed region) is the reference solution
                ref = sysd.solve(tol=1e-12, restart=100)["x"]
                xs[mode] = float(torch.linalg.vector_norm(sol - ref) / torch.linalg.vector_norm(ref))
                if mode in ORACLE_MODES and rank == 0 and world == 1 and not args.no_oracle:
                    # this step's geometry and solution, for the CPU oracle after the loop
                    locs, quats = sysd.body_state()
                    snap[mode] = dict(x_fib=sysd.x_fib.cpu().numpy().copy(), locs=locs, quats=quats,
                                      sol=sol.cpu().numpy(), rhs=sysd.rhs.cpu().numpy(),
                                      ref=ref.cpu().numpy())
        if mode in snap:
            # checked against the oracle's matrix-free step at this geometry
            # (and, for fiber3d's method, its CPU time): outside every timing
            out.setdefault(mode, {})["oracle"] = step_oracle(P, snap.pop(mode), cpu_time=(mode == "fp64"),
                                                             iterations=statistics.median(its))
        out[mode] = {**out.get(mode, {}), "ms_per_step": statistics.median(times), "iterations": its,
                     "ms_per_step_last_half": statistics.median(times[len(times) // 2:]),
                     "true_rel_residual": max(resid), "refinements": res.get("refinements", 0),
                     "initial_rel_residual": r0s, "final_rel_residual_bound": finals,
                     "fiber_pc_rebuilt": fresh, "tol": tol, "long_solves": worst,
                     "fp64_residuals": sum(fp64r),
                     "first_residual_bound_max": max((x for x in fbounds if x is not None), default=None),
                     "phases_ms": {k: statistics.median([p.get(k, 0.0) for p in phases]) for k in phases[0]}}
        if mode == "learned_mixed":
            # velocity field on fiber3d's own grid (tstep.py:1240-1270) for the
            # last step's solution, as the time step's optional output
            # evaluates it; outside the per-step timings
            grid = torch.as_tensor(geometry.ellipsoid_grid(), device=dev)
            for _ in range(2):
                sysd.grid_velocity(sol, grid, body0_radius=0.5)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(5):
                vg = sysd.grid_velocity(sol, grid, body0_radius=0.5)
            e1.record()
            e1.synchronize()
            out["grid_velocity"] = {"grid_points": int(grid.shape[0]), "ms": e0.elapsed_time(e1) / 5,
                                    "finite": bool(torch.isfinite(vg).all())}
        del sysd
    # each replica's median step; the job's is the slowest replica's
    slowest = replicas.max_over_ranks([out[m]["ms_per_step"] for m in modes], dev)
    for mode, ms in zip(modes, slowest):
        out[mode]["ms_per_step"] = ms
    for mode in modes:
        out[mode]["rel_err_vs_fp64_1e-12_solve"] = xs[mode]
        out[mode]["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out[mode]["ms_per_step"]
    out["training"] = train
    line = {"metric": "hydro time step (ms), GMRES rel. residual 1e-8", "value": out["fp64"]["ms_per_step"],
            "unit": "ms", "n_gpus": world, "steps": steps, "warmup": warmup,
            "higher_is_better": False, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": "hydro_step", "fibers": args.nfib, "points_per_fiber": 32,
                       "bodies": 4, "body_nodes": 400, "shell_nodes": args.nshell,
                       "shell_radius": args.shell_radius, "fiber_ball": args.fiber_ball,
                       "body_shell": args.body_shell,
                       "system_size": int(3 * args.nshell + 4 * 1206 + 4 * 32 * args.nfib),
                       "shell_pc": args.shell_pc, "shell_setup_s": setup_s}, "step": out}
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line


def _quadrature_problem(args):
    from scipy.spatial import ConvexHull
    from fiber3d_b200 import geometry
    nodes, _ = geometry.fibonacci_sphere(args.nshell, args.shell_radius)
    tri = ConvexHull(nodes).simplices.astype(np.int32)
    return nodes, tri, 2.0 * nodes  # gradh of |x|^2 - R^2 (shape_gallery's sphere)


def cpu_quadrature_rate(nodes, tri, grad, seconds: float):
    """Triangles/s of the CPU restatement (oracle/quadrature.py: the
    neighbour search, the local system and LAPACK's solve of each triangle)
    on consecutive triangles for about `seconds`."""
    from oracle import quadrature as OQ
    ts = np.sort(tri, axis=1)
    tn = OQ.triangle_normals(nodes, ts)
    en = OQ.edge_normals(ts, tn)
    mids = (nodes[ts[:, 0]] + nodes[ts[:, 1]] + nodes[ts[:, 2]]) / 3
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds or done == 0:
        s = done % len(ts)
        nni = OQ.nearest_neighbors(nodes, mids[s:s + 64])
        for k in range(len(nni)):
            M, r, d = OQ.triangle_system(nodes, grad, ts[s + k], tn[s + k], en[s + k], nni[k])
            np.linalg.solve(M, r)
        done += len(nni)
    return done / (time.perf_counter() - t0), done


def quadrature_reference_arm(args, world):
    """The CPU restatement of fiber3d's quadrature loop (one core), each step
    a bounded sample of triangles extrapolated to the whole surface."""
    nodes, tri, grad = _quadrature_problem(args)
    per_step = max(1.0, args.cpu_seconds / max(args.steps, 1))
    for _ in range(args.warmup):
        cpu_quadrature_rate(nodes, tri, grad, 0.0)
    samples = [cpu_quadrature_rate(nodes, tri, grad, per_step) for _ in range(args.steps)]
    ms = statistics.median(len(tri) / r * 1e3 for r, _ in samples)
    line = {"impl": "reference", "metric": "surface quadrature set-up (ms)", "value": ms, "unit": "ms",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (shape_gallery sphere)",
            "config": {"workload": "surface_quadrature", "nodes": int(args.nshell), "triangles": int(len(tri)),
                       "radius": args.shell_radius, "parallelism": "one host core"},
            "cpu_baseline": {"value": ms, "unit": "ms", "cores": 1, "kind": "port",
                             "sample": f"{samples[0][1]} triangles per step sample, extrapolated to {len(tri)}; "
                                       "numpy/LAPACK restatement of fiber3d's loop (oracle/quadrature.py)"},
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def quadrature_arm(args, rank, world, local):
    """RBF surface quadrature of the periphery (fiber3d's set-up step,
    quadratures/Smooth_Closed_Surface_Quadrature_RBF.py with the exact
    gradient, tstep/tstep.py:285-300): args.nshell nodes of shape_gallery's
    sphere of radius args.shell_radius, triangles from scipy's ConvexHull.  A
    step is one full call: triangle preparation, edge normals, the 80-nearest
    search, the 116 x 116 local solves and the per-node sums."""
    import torch
    from fiber3d_b200 import quadrature as Qd, replicas
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    nodes, tri, grad = _quadrature_problem(args)
    X = torch.as_tensor(nodes, device=dev)
    T = torch.as_tensor(tri, device=dev)
    G = torch.as_tensor(grad, device=dev)
    for _ in range(args.warmup):
        Qd.surface_quadrature_weights(X, T, G)
    times = []
    with ClockSampler(local) as clk:
        replicas.barrier()
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            w = Qd.surface_quadrature_weights(X, T, G)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        replicas.barrier()
    ms = replicas.max_over_ranks([statistics.median(times)], dev)[0]
    # end to end from host arrays, as fiber3d calls it
    e2e = []
    for _ in range(max(3, args.steps // 2)):
        t0 = time.perf_counter()
        wh = Qd.surface_quadrature_weights(nodes, tri, grad, device=dev).cpu().numpy()
        e2e.append((time.perf_counter() - t0) * 1e3)
    ntri = len(tri)
    # LU of the 116 x 116 system with the right-hand side appended:
    # sum_{m<116} m (m + 1) multiply-adds per triangle
    flops = 2.0 * sum(m * (m + 1) for m in range(116)) * ntri
    R = args.shell_radius
    line = {"metric": "surface quadrature set-up (ms)", "value": ms, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (shape_gallery sphere)",
            "config": {"workload": "surface_quadrature", "nodes": int(args.nshell), "triangles": int(ntri),
                       "radius": R, "neighbors": 80, "poly_order": 7, "l2": "inputs 0.9 MB, L2-resident"},
            "roofline": {"bound": "fp64", "achieved": flops / (ms * 1e-3) / 1e12, "peak": 33.5,
                         "unit": "TFLOP/s", "frac": flops / (ms * 1e-3) / 1e12 / 33.5, "traffic": None,
                         "note": "algorithmic LU flops over the whole call (all eight kernels); "
                                 "peak = measured FP64 FMA rate"},
            "e2e": {"value": statistics.median(e2e), "unit": "ms",
                    "h2d_bytes_per_step": int(nodes.nbytes + grad.nbytes + tri.nbytes),
                    "d2h_bytes_per_step": int(wh.nbytes)},
            "gpu_launches": 8 * args.steps,
            "clocks": clk.summary(),
            "checks": {"area_rel_err": float(wh.sum() / (4 * np.pi * R * R) - 1),
                       "x2_rel_err": float((wh * nodes[:, 0] ** 2).sum() / (4 * np.pi * R ** 4 / 3) - 1),
                       "bitwise_repeatable": bool(torch.equal(w, Qd.surface_quadrature_weights(X, T, G)))}}
    if rank == 0 and world == 1:
        rate, done = cpu_quadrature_rate(nodes, tri, grad, args.cpu_seconds)
        line["cpu_baseline"] = {"value": ntri / rate * 1e3, "unit": "ms", "cores": 1, "kind": "port",
                                "sample": f"{done} of {ntri} triangles, extrapolated; numpy/LAPACK "
                                          "restatement (fiber3d's own loop ran 4.8 ms per triangle here)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return line


def dense_inverse_arm(args, rank, world, local):
    """The periphery preconditioner's set-up: the dense shell operator of an
    args.nshell-node sphere (Fibonacci nodes, equal-area weights, radius
    args.shell_radius; tstep.py:327-347) inverted in place by
    f3d_dense_inverse (blocked Gauss-Jordan, FP64 tensor-core updates).  A
    step is one inversion of the 3N x 3N matrix (a fresh copy each time).
    fiber3d factors this matrix with scipy.linalg.lu_factor (tstep.py:348):
    that call on the host cores, timed on a smaller sphere and scaled by the
    cube of the size, is the CPU baseline; cuSOLVER's inverse
    (torch.linalg.inv) of the same matrix is reported beside it."""
    import ctypes
    import torch
    from fiber3d_b200 import _lib as L, geometry, hydro as H, replicas
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    steps, warmup = max(1, min(args.steps, 3)), min(args.warmup, 1)

    def operator(n):
        nodes, normals = geometry.fibonacci_sphere(n, args.shell_radius)
        w = np.full(n, 4.0 * np.pi * args.shell_radius ** 2 / n)
        sh = H.ShellOperator(H.Shell(nodes, normals, w), 1.0, 5e-3, 1e-5, dev, build_inverse=False)
        m = 3 * n
        ld = H.dense_inverse_ld(m)
        M = torch.zeros((ld, ld), dtype=torch.float64, device=dev)
        L.call("f3d_surface_dense", 0, L.ptr(sh.nodes), L.ptr(sh.normals), L.ptr(sh.E), L.ptr(sh.weights), None,
               L.ptr(M), n, ld, 1.0, 5e-3, 1e-5, L.stream_handle(dev))
        return (nodes, normals, w), M, m

    host, M0, m = operator(args.nshell)
    ld = M0.shape[0]
    A = torch.empty_like(M0)
    nb = ctypes.c_size_t(0)
    L.call("f3d_dense_inverse_workspace_bytes", m, ld, ctypes.byref(nb))
    ws = torch.empty(nb.value, dtype=torch.uint8, device=dev)

    def invert():
        L.call("f3d_dense_inverse", L.ptr(A), m, ld, L.ptr(ws), ws.numel(), L.stream_handle(dev))

    for _ in range(warmup):
        A.copy_(M0)
        invert()
    times = []
    with ClockSampler(local) as clk:
        replicas.barrier()
        for _ in range(steps):
            A.copy_(M0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            invert()
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        replicas.barrier()
    ms = replicas.max_over_ranks([statistics.median(times)], dev)[0]
    # accuracy: residual of the inverse on a random vector, and cuSOLVER's inverse
    g = torch.Generator(device=dev).manual_seed(1)
    x = torch.randn(m, generator=g, device=dev, dtype=torch.float64)
    Mm = M0[:m, :m]
    res = float(torch.linalg.vector_norm(Mm @ (A[:m, :m] @ x) - x) / torch.linalg.vector_norm(x))
    X = A[:m, :m].clone()
    del A
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ref = torch.linalg.inv(Mm)
    torch.cuda.synchronize()
    lib_s = time.perf_counter() - t0
    diff = float(torch.linalg.matrix_norm(X - ref) / torch.linalg.matrix_norm(ref))
    del ref, X
    # end to end: the ShellOperator set-up from host arrays (singularity
    # vectors, dense operator, inverse, FP32 and row-scaled FP16 copies)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sh = H.ShellOperator(H.Shell(*host), 1.0, 5e-3, 1e-5, dev)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    del sh
    torch.cuda.empty_cache()
    peak, peak_clk = measured_peak(L, "fp64_mma", torch, local)
    npad = ld
    flops = 2.0 * float(npad) ** 3
    achieved = flops / (ms * 1e-3)
    line = {"metric": "periphery preconditioner set-up: dense inverse (ms)", "value": ms, "unit": "ms",
            "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (Fibonacci sphere)",
            "config": {"workload": "dense_inverse", "nodes": int(args.nshell), "matrix": int(m),
                       "padded": int(npad), "radius": args.shell_radius,
                       "l2": f"matrix {m * m * 8 / 1e9:.1f} GB, far above L2"},
            "roofline": {"bound": "fp64-tensor", "achieved": achieved / 1e12, "peak": peak / 1e12,
                         "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                         "kernel": "gj_update_kernel (with the per-step pivot-block inverse and panel)",
                         "note": "2 np^3 flops of the whole call (np = matrix size padded to 128); peak = "
                                 "measured FP64 tensor-core MMA rate (f3d_probe_fma precision 2)",
                         "peak_clocks": peak_clk},
            "checks": {"residual_M_Xv_minus_v": res, "rel_diff_vs_cusolver_inverse": diff},
            "library_baseline": {"torch_linalg_inv_ms": lib_s * 1e3,
                                 "note": "cuSOLVER getrf + getri through torch on the same matrix"},
            "e2e": {"value": e2e_s * 1e3, "unit": "ms",
                    "h2d_bytes_per_step": int(sum(a.nbytes for a in host)), "d2h_bytes_per_step": 0,
                    "path": "ShellOperator(Shell(nodes, normals, weights)) from host arrays"},
            "gpu_launches": int(steps * (3 * (npad // 128) + 1)),
            "clocks": clk.summary()}
    if rank == 0 and world == 1:
        import scipy.linalg as sla
        ns = max(200, min(args.nshell, int(args.dense_cpu_nodes)))
        _, Ms, ms_ = operator(ns)
        Mh = Ms[:ms_, :ms_].cpu().numpy()
        del Ms
        reps, t_cpu = 0, 0.0
        while reps < 1 or (t_cpu < args.cpu_seconds and reps < 5):
            t0 = time.perf_counter()
            sla.lu_factor(Mh)
            t_cpu += time.perf_counter() - t0
            reps += 1
        per = t_cpu / reps
        line["cpu_baseline"] = {"value": per * (m / ms_) ** 3 * 1e3, "unit": "ms", "cores": os.cpu_count(),
                                "kind": "reference",
                                "sample": f"scipy.linalg.lu_factor (fiber3d's call) of the {ms_} x {ms_} operator "
                                          f"of a {ns}-node sphere, {per:.2f} s, scaled by ({m}/{ms_})^3; "
                                          "LU only (2/3 n^3), threads as the host LAPACK uses them"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return line


def block_pc_measure(args, dev, steps, warmup, cpu_seconds):
    """Batched block-diagonal preconditioner (config 4): 2000 fibers with
    point counts uniform in {16, 24, 32, 48, 64} (geometry of the step
    workload), their 4N x 4N systems assembled on the device (fiber3d's
    fiber operator with BC rows), then factor + solve of all blocks captured
    in one CUDA graph (two persistent launches plus a copy), panel width from
    the autotuner.  Baseline: scipy.linalg.lu_factor / lu_solve per block,
    the calls fiber3d makes (tstep_utils.py:1405-1419, tstep.py:985-988)."""
    import torch
    import scipy.linalg as sla
    from fiber3d_b200 import geometry, hydro as H, replicas
    rng = np.random.default_rng(4)
    npts = rng.choice([16, 24, 32, 48, 64], size=args.nblocks)
    fibers = geometry.perturbed_fibers(rng, args.nblocks, npts, 2.0, 10.0, min_sep=0.05)
    ff = np.concatenate([np.tile(rng.normal(scale=0.1, size=3), (n, 1)) for n in npts])
    P = H.Problem(fibers, [2.0] * args.nblocks, 0.0025, 1e-3, 1.0, [], None, ff)
    sysd = H.HydroSystem(P, device=dev)
    lu = sysd.lu
    A0 = lu.A.clone()
    rhs = torch.as_tensor(rng.normal(size=lu.nvec), device=dev)
    x = torch.empty_like(rhs)
    panel = lu.tune_panel()
    flop_factor = float(sum(2.0 / 3.0 * (4 * n) ** 3 for n in npts))
    flop = flop_factor + float(sum(2.0 * (4 * n) ** 2 for n in npts))
    bytes_blocks = float(sum(8 * (4 * n) ** 2 for n in npts))

    def work():
        lu.A.copy_(A0)
        lu.factor()
        x.copy_(rhs)
        lu.solve(x)
    for _ in range(warmup):
        work()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s2 = torch.cuda.Stream(dev)
    s2.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(s2):
        work()
    torch.cuda.current_stream(dev).wait_stream(s2)
    with torch.cuda.graph(g):
        work()
    for _ in range(warmup):
        g.replay()
    torch.cuda.synchronize()
    replicas.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        g.replay()
    e1.record()
    e1.synchronize()
    replicas.barrier()
    ms, = replicas.max_over_ranks([e0.elapsed_time(e1) / steps], dev)
    # parity and CPU baseline on the same blocks
    A_h = A0.cpu().numpy()
    rhs_h = rhs.cpu().numpy()
    xg = x.cpu().numpy()
    blocks = [A_h[lu.moff_h[b]:lu.moff_h[b] + lu.sizes_h[b] ** 2].reshape(lu.sizes_h[b], lu.sizes_h[b])
              for b in range(lu.count)]
    t0 = time.perf_counter()
    nb_cpu = 0
    err = 0.0
    while True:
        for b, Ab in enumerate(blocks):
            o, n = int(lu.voff_h[b]), int(lu.sizes_h[b])
            xr = sla.lu_solve(sla.lu_factor(Ab, check_finite=False), rhs_h[o:o + n])
            if nb_cpu == 0:
                err = max(err, float(np.max(np.abs(xr - xg[o:o + n])) / np.max(np.abs(xr))))
        nb_cpu += 1
        if time.perf_counter() - t0 > min(10.0, cpu_seconds):
            break
    cpu_ms = (time.perf_counter() - t0) / nb_cpu * 1e3
    del g
    return {"ms": ms, "gflops": flop / (ms * 1e-3) / 1e9, "factor_gflop": flop_factor / 1e9,
            "block_bytes_gb": bytes_blocks / 1e9, "max_rel_err_vs_scipy": err, "panel": panel,
            "cpu_ms": cpu_ms, "cpu_cores": os.cpu_count(),
            "cpu_sample": f"scipy.linalg.lu_factor + lu_solve over all {args.nblocks} blocks, {nb_cpu} pass(es)"}


def fmm_workload(n: int, seed: int = 0):
    """fiber3d's own FMM check (kernels/test_stkfmm.py:39-53): n single-layer
    sources, n double-layer sources and n targets uniform in a cube of side
    (4 pi 2n / (3e-3))^(1/3) (volume fraction 1e-3), N(0, 1) densities and
    normals.  Seeded synthetic stand-in of the same shape."""
    rng = np.random.default_rng(seed)
    side = (4 * np.pi * 2 * n / (3 * 1e-3)) ** (1 / 3)
    return dict(sl=rng.random((n, 3)) * side, dl=rng.random((n, 3)) * side, trg=rng.random((n, 3)) * side,
                f=rng.normal(size=(n, 3)), nrm=rng.normal(size=(n, 3)), dens=rng.normal(size=(n, 3)), side=side)


def fmm_arm(args, rank, world, local):
    """The FMM (fiber3d's useFMM path, kernels.py:1298-1485): one step = one
    evaluation of the single + double layer at the targets on a built tree.
    value: equivalent pair interactions per second, (n_SL + n_DL) n_trg / time.
    Reported beside it: the tree build, the direct GPU sum of the same
    velocities and the FMM's error against it, the far-field roofline."""
    import torch
    from fiber3d_b200 import fmm as F, kernels as K, replicas, stkfmm
    from fiber3d_b200 import _lib as L
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.fmm_n
    w = fmm_workload(n, seed=rank)
    t = {k: torch.as_tensor(v, device=dev) for k, v in w.items() if k != "side"}
    m = F.FMM(order=args.fmm_order, max_pts=args.fmm_max_pts, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    m.set_points(t["sl"], t["dl"], t["trg"])
    torch.cuda.synchronize()
    setup_ms = (time.perf_counter() - t0) * 1e3
    out = torch.empty(3 * n, dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    evaluate = lambda: m.evaluate(sl_density=t["f"], dl_normal=t["nrm"], dl_density=t["dens"], out=out)
    for _ in range(args.warmup):
        evaluate()
    torch.cuda.synchronize()
    replicas.barrier()
    evs = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            evaluate()
            e1.record()
            evs.append((e0, e1))
        torch.cuda.synchronize()
    replicas.barrier()
    ms = [a.elapsed_time(b) for a, b in evs]
    total_ms, = replicas.max_over_ranks([sum(ms)], dev)
    pairs = 2 * n * n
    value = replicas.aggregate_rate(pairs, args.steps, world, total_ms)
    # the direct sum of the same velocities (exact FP64, coincident pairs excluded)
    # (one untimed pass first: the workspace is allocated there; then the
    # median of three timed passes)
    ref = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    kw = dict(self_mode="skip_close", epsilon_distance=1e-150, reg=0.0, out=ref, accumulate=False)

    def direct():
        K.pair_sum("oseen", t["sl"], t["trg"], t["f"], **kw)
        K.pair_sum("stresslet", t["dl"], t["trg"], t["dens"], t["nrm"], **dict(kw, accumulate=True))

    direct()
    torch.cuda.synchronize()
    dts = []
    for _ in range(3 if n <= 300000 else 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        direct()
        e1.record()
        e1.synchronize()
        dts.append(e0.elapsed_time(e1))
    direct_ms = statistics.median(dts)
    err_l2 = float(torch.linalg.vector_norm(out - ref) / torch.linalg.vector_norm(ref))
    err_inf = float((out - ref).abs().max() / ref.abs().max())
    peak64, _ = measured_peak(L, "fp64", torch, local)
    flops = m.far_field_flops()
    info = m.tree_info()
    # e2e: fiber3d's combined call on host arrays with an stkfmm handle (the
    # tree is built on the first call and kept while the points are the same)
    h = stkfmm.STKFMM(args.fmm_order, args.fmm_max_pts, stkfmm.PAXIS.NONE, stkfmm.KERNEL(stkfmm.KERNEL.PVel))
    call = lambda: K.single_double_layer_kernel_source_target_stkfmm(w["sl"], w["dl"], w["trg"], w["nrm"], w["f"],
                                                                     w["dens"], fmm_PVel=h)
    for _ in range(2):
        call()
    te = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        call()
        te.append(time.perf_counter() - t0)
    e2e_s = statistics.median(te)
    # CPU: the C/OpenMP restatement of the direct sums on a target sample
    from oracle import pairs_c
    hc = host_cores()
    nt_cpu = min(n, 256)
    t0 = time.perf_counter()
    pairs_c.pair_sum("oseen", w["sl"], w["trg"][:nt_cpu], w["f"], epsilon_distance=0.0, reg=0.0)
    pairs_c.pair_sum("stresslet", w["dl"], w["trg"][:nt_cpu], w["dens"], w["nrm"], epsilon_distance=0.0, reg=0.0)
    cpu_rate = 2 * n * nt_cpu / (time.perf_counter() - t0)
    line = {
        "metric": f"FMM equivalent Stokes pair interactions per second (FP64, order {args.fmm_order})",
        "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded): fiber3d's STKFMM check shape (kernels/test_stkfmm.py)",
        "config": {"workload": "fmm", "n_single_layer": n, "n_double_layer": n, "n_targets": n,
                   "cube_side": w["side"], "order": args.fmm_order, "max_pts": args.fmm_max_pts,
                   "l2": "flushed between steps (256 MiB write, outside the event pairs)"},
        "parallelism": f"replicas x{world}",
        "tree": {**info, "setup_ms": setup_ms},
        "accuracy_vs_direct": {"rel_l2": err_l2, "rel_linf": err_inf},
        "direct_gpu_ms": direct_ms, "speedup_vs_direct_gpu": direct_ms / (total_ms / args.steps),
        "roofline": {"bound": "fp64", "kernel": "fmm_gemm_kernel (interaction lists)",
                     "achieved": flops / (total_ms / args.steps * 1e-3) / 1e12, "peak": peak64 / 1e12,
                     "unit": "TFLOP/s", "frac": flops / (total_ms / args.steps * 1e-3) / peak64,
                     "note": "far-field flops per evaluation (2 (3n)(4n) per interaction-list entry) over the "
                             "whole evaluation's time: a lower bound of the GEMM kernel's own rate"},
        "cpu_baseline": {"value": cpu_rate, "unit": "pairs/s", "cores": hc["threads"], **hc, "kind": "port",
                         "sample": f"direct sums onto {nt_cpu} targets (C/OpenMP restatement of fiber3d's numba "
                                   "loops, the sums fiber3d checks STKFMM against)"},
        "e2e": {"value": pairs / e2e_s, "unit": "pairs/s", "h2d_bytes_per_step": 18 * n * 8,
                "d2h_bytes_per_step": 3 * n * 8,
                "path": "fiber3d_b200.kernels.single_double_layer_kernel_source_target_stkfmm, numpy in/out, "
                        "stkfmm handle"},
        "clocks": clk.summary(),
        "gpu_launches": m.last_launches() * args.steps,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def block_pc_arm(args, rank, world, local):
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    r = block_pc_measure(args, dev, args.steps, args.warmup, args.cpu_seconds)
    line = {"metric": "block-diagonal preconditioner factor+solve time (ms)", "value": r["ms"], "unit": "ms",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": "block_pc", "blocks": args.nblocks, "block_sizes": "4N, N in {16,24,32,48,64}",
                       "panel": r["panel"], "graph": "copy + factor + copy + solve, one CUDA graph"},
            "gflops": r["gflops"], "max_rel_err_vs_scipy": r["max_rel_err_vs_scipy"],
            "cpu_baseline": {"value": r["cpu_ms"], "unit": "ms", "cores": r["cpu_cores"], "kind": "reference",
                             "sample": r["cpu_sample"]}}
    if rank == 0:
        print(json.dumps(line), flush=True)


def oseen_fibers_measure(args, dev, steps, warmup, cpu_seconds):
    """Config 1: the Oseen sum of 32 fibers x 32 Chebyshev-Lobatto nodes
    (1024 points, j == i skipped; kernels.py:214-287), FP64.  Latency bound:
    device time per call, the HBM rate of its 73.7 KB of algorithmic I/O,
    the drop-in call from pinned host buffers, and the C/OpenMP port."""
    import torch
    from fiber3d_b200 import autotune, kernels as K
    wl = make_workload("oseen_fibers")
    x = torch.as_tensor(wl["src"], device=dev)
    f = torch.as_tensor(wl["dens"], device=dev)
    shape = autotune.tune("oseen", x, x, f, self_mode="skip_index")
    out = torch.empty(x.numel(), dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(warmup):
        K.pair_sum("oseen", x, x, f, self_mode="skip_index", shape=shape, out=out)
    torch.cuda.synchronize()
    evs = []
    for _ in range(steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        K.pair_sum("oseen", x, x, f, self_mode="skip_index", shape=shape, out=out)
        e1.record()
        evs.append((e0, e1))
    torch.cuda.synchronize()
    us = statistics.median(a.elapsed_time(b) for a, b in evs) * 1e3
    io_bytes = 3 * x.numel() * 8  # x, f in; u out
    xh, fh = torch.as_tensor(wl["src"]).pin_memory(), torch.as_tensor(wl["dens"]).pin_memory()
    for _ in range(warmup):
        K.oseen_kernel_times_density_numba(xh, fh)
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        K.oseen_kernel_times_density_numba(xh, fh)
        ts.append(time.perf_counter() - t0)
    e2e_us = statistics.median(ts) * 1e6
    cpu_rate, _, _ = cpu_sample_rate(wl, host_cores()["threads"], min(2.0, cpu_seconds))
    return {"us_per_call": us, "pairs_per_s": wl["pairs"] / (us * 1e-6), "io_bytes": io_bytes,
            "hbm_gbs": io_bytes / (us * 1e-6) / 1e9, "e2e_us_per_call": e2e_us,
            "e2e_pairs_per_s": wl["pairs"] / (e2e_us * 1e-6), "cpu_pairs_per_s": cpu_rate,
            "launch_shape": [shape.tpt, shape.sl, shape.nsplit, shape.use_tma]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="stresslet_sphere",
                    choices=["stresslet_sphere", "oseen_fibers", "hydro_step", "block_pc",
                             "surface_quadrature", "fmm", "dense_inverse"])
    ap.add_argument("--dense-cpu-nodes", type=int, default=3000,
                    help="sphere of the CPU lu_factor sample of the dense_inverse workload")
    ap.add_argument("--fmm-n", type=int, default=1000000, help="points of each kind of the FMM workload")
    ap.add_argument("--fmm-order", type=int, default=8)
    ap.add_argument("--fmm-max-pts", type=int, default=1000)
    ap.add_argument("--nblocks", type=int, default=2000)
    ap.add_argument("--train-seeds", type=int, nargs="*", default=list(range(11, 19)))
    ap.add_argument("--train-steps", type=int, default=40)
    ap.add_argument("--train-epochs", type=int, default=40)
    ap.add_argument("--train-skip", type=int, default=8,
                    help="steps at the start of each trajectory left out of training and selection")
    ap.add_argument("--nshell", type=int, default=12000)
    ap.add_argument("--nfib", type=int, default=512)
    ap.add_argument("--shell-radius", type=float, default=10.0)
    ap.add_argument("--fiber-ball", type=float, default=5.0, help="radius of the ball holding the fiber centres")
    ap.add_argument("--body-shell", type=float, default=7.5, help="distance of the body centres from the origin")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--shell-pc", default="dense", choices=["dense", "block"],
                    help="periphery preconditioner of the time step: the dense inverse (fiber3d's LU) or "
                         "the block-Jacobi one")
    ap.add_argument("--no-step", action="store_true",
                    help="pair throughput only (skip the embedded time-step comparison)")
    ap.add_argument("--no-flownet", action="store_true",
                    help="skip the (positions, background velocity) network and its mode")
    ap.add_argument("--flow-seeds", type=int, default=4, help="training trajectories of that network")
    ap.add_argument("--no-oracle", action="store_true",
                    help="skip the CPU-oracle check (and CPU time) of the step's solutions")
    ap.add_argument("--step-warmup", type=int, default=8)
    ap.add_argument("--step-steps", type=int, default=40)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local = dist_info()
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    # launch shapes are tuned on this run's own sums: a shape file left by
    # other programs holds shapes tuned on other sizes of the same
    # power-of-two size bucket
    if "FIBER3D_B200_TUNE" not in os.environ:
        import tempfile
        os.environ["FIBER3D_B200_TUNE"] = os.path.join(tempfile.mkdtemp(prefix="f3d_bench_"), "pair_shapes.json")
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.workload == "hydro_step":
            hydro_arm(args, rank, world, local)
        elif args.workload == "block_pc":
            block_pc_arm(args, rank, world, local)
        elif args.workload == "surface_quadrature":
            quadrature_arm(args, rank, world, local)
        elif args.workload == "fmm":
            fmm_arm(args, rank, world, local)
        elif args.workload == "dense_inverse":
            dense_inverse_arm(args, rank, world, local)
        else:
            gpu_arm(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
