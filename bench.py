"""Benchmark of the FMM hot path on B200 (one JSON line on rank 0).

Workload (the headline configuration): 1,000,000 particles uniform in [0,1)^3 (seeded), charges uniform in
[-1,1], Laplace 1/r, Chebyshev order 7, octree height 6, MIXED precision (FP32 compensated P2P, split-FP16
tcgen05 M2L with FP32 accumulation).  One step = one FMM evaluation from particles: GPU tree build
(Morton keys, radix sort, lists) + P2M, M2M, M2L, L2L, L2P, P2P.

  value  particles/s with the particles resident in HBM (device-pointer b200fmm_set_particles + execute),
         device time from CUDA events on the library's stream, summed over the K timed steps, max over ranks;
  e2e    the same through host buffers: pinned x, y, z, q copied in by b200fmm_set_particles, results
         (phi, fx, fy, fz) copied back by b200fmm_get_results, every step;
L2 is flushed (a 512 MiB write) between timed steps, outside the timed intervals.

Multi-GPU (torchrun): replicas only -- every rank evaluates its own copy of the workload, no collective in
the data path ("scaling": "weak"); NCCL is used only for the barrier and the max-over-ranks reduction.

--impl reference times the reference's own CPU implementation (ScalFMM FFmmAlgorithmThread +
FChebSymKernel, compiled from its sources into oracle/_ref) on the host cores: one step = one evaluation
of the same workload (tree insertion and kernel construction untimed, as the reference's own drivers time
algo.execute()).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))  # the seeded distributions of the workloads
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

METRIC = "particles/s per FMM eval (1M uniform, Chebyshev p=7, height 6, mixed precision)"
N_PART, ORDER, HEIGHT, SEED = 1_000_000, 7, 6, 42
FLOPS_PER_P2P_PAIR = 20  # 3 sub, 5 for r^2, rsqrt as 1, 3 for 1/r^3 and q scaling, 2 potential, 6 force


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=N_PART)
    ap.add_argument("--height", type=int, default=HEIGHT, help="octree height (profiling of small cases only)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="form of the timed steps (the headline is mixed; fp64 times the plain form, for profiles)")
    ap.add_argument("--nrhs", type=int, default=1, help="charge vectors per step (profiles of the multi-RHS path)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batch-of-problems measurement")
    ap.add_argument("--no-pins", action="store_true",
                    help="skip the CPU reference runs that pin the FP64 GPU FMM at the full workload sizes")
    return ap.parse_args()


def particles(n, seed=SEED):
    rng = np.random.default_rng(seed)
    pos = rng.random((3, n))
    q = rng.uniform(-1.0, 1.0, n)
    return pos[0].copy(), pos[1].copy(), pos[2].copy(), q


def plummer(n, rng, scale=0.1):
    """Plummer sphere (scale radius 0.1) centred in the unit cube, points outside the cube rejected."""
    out, have = [], 0
    while have < n:
        m = 2 * n
        r = scale / np.sqrt(rng.random(m) ** (-2.0 / 3.0) - 1.0)
        d = rng.standard_normal((3, m))
        d /= np.linalg.norm(d, axis=0)
        pnt = d * r + 0.5
        keep = np.all((pnt >= 0.0) & (pnt < 1.0), axis=0)
        out.append(pnt[:, keep])
        have += int(keep.sum())
    pnt = np.concatenate(out, axis=1)[:, :n]
    return pnt[0].copy(), pnt[1].copy(), pnt[2].copy()


def leaf_height(x, y, z, target=30.0, lo=4, hi=7):
    """Smallest height in [lo, hi] whose leaves hold about `target` particles as a particle sees them (the
    particle-weighted mean occupancy, sum n_leaf^2 / N, at most 2 x target); the Plummer core is far denser
    than the average, so the plain mean N / leaves would leave thousands of particles in the core leaves."""
    for h in range(lo, hi + 1):
        side = 1 << (h - 1)
        c = np.minimum((np.stack([x, y, z]) * side).astype(np.int64), side - 1)
        _, cnt = np.unique((c[0] * side + c[1]) * side + c[2], return_counts=True)
        if (cnt.astype(float) ** 2).sum() / x.size <= 2.0 * target:
            return h
    return hi


def batch_workload(seed=5):
    """64 independent problems, sizes log-uniform in 10,000..500,000, Plummer positions, charges U[-1,1],
    Chebyshev order 5..7 per problem, height in 4..7 chosen for about 30 particles per leaf."""
    rng = np.random.default_rng(seed)
    problems = []
    for k in range(64):
        n = int(np.exp(rng.uniform(np.log(1e4), np.log(5e5))))
        x, y, z = plummer(n, rng)
        problems.append(dict(x=x, y=y, z=z, q=rng.uniform(-1.0, 1.0, n), order=5 + k % 3,
                             height=leaf_height(x, y, z)))
    return problems


def batch_measure(S, device):
    problems = batch_workload()
    total = sum(p["x"].size for p in problems)
    b = S.Batch("cheb_sym", "mixed", nstreams=4, device=device)
    b.run(problems)  # handles, operators and buffers of every (order, height)
    dev, wall = [], []
    for _ in range(5):
        b.run(problems)
        dev.append(b.last_device_ms())
        wall.append(b.last_time_ms())
    b.close()
    med = statistics.median(dev)
    return {"problems": len(problems), "particles": total, "ms": med, "particles_per_s": total / (med * 1e-3),
            "device_ms_runs": dev, "wall_ms_runs": wall,
            "workload": "64 problems, n log-uniform in [1e4, 5e5], Plummer (a = 0.1) truncated to the unit cube, "
                        "Chebyshev order 5..7, height 4..7 for ~30 particles per leaf as a particle sees it, MIXED, "
                        "4 worker streams",
            "timing": "device time of b200fmm_batch_execute (CUDA events: start to the last worker stream's end; "
                      "host arrays in and out, tree builds included), median of 5 after one untimed run"}


def workload_config(n, height=HEIGHT, precision="mixed", nrhs=1):
    cfg = {"workload": f"{n} particles uniform in [0,1)^3, q~U[-1,1] (seed {SEED}), Laplace 1/r, Chebyshev order "
                       f"{ORDER}, height {height}", "particles": n, "order": ORDER, "height": height,
           "precision": "mixed: FP32 compensated P2P, split-FP16 x3 tcgen05 M2L, FP64 P2M/M2M/L2L/L2P",
           "l2": "flushed between timed steps (512 MiB write)", "parallelism": "replicas"}
    if precision != "mixed":
        cfg["precision"] = "fp64: every operator in FP64 (the plain form)"
    if nrhs > 1:
        cfg["nrhs"] = nrhs
    return cfg


# ------------------------------------------------------------------------------------------------------
# clocks
# ------------------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm", "clocks.max.sm", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index, period_ms=20):
        self.index = index
        self.period_ms = period_ms
        self.samples = []
        self.proc = None
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        # one long-lived nvidia-smi streaming a line every period_ms
        try:
            for line in self.proc.stdout:
                vals = [v.strip() for v in line.strip().split(",")]
                if len(vals) == len(self.FIELDS):
                    self.samples.append(vals)
        except Exception:
            pass

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + ",".join(self.FIELDS),
                                          "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t.start()
            time.sleep(0.3)  # let the first samples arrive before the timed region starts
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=10)
            except Exception:
                self.proc.kill()
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops_sustained", 1400.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1400.0, 1590.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the tensor-core M2L kernel, from the committed ncu summary (None if absent)."""
    f = ROOT / "profiles" / "m2l_tc_kernel_traffic.txt"
    if f.exists():
        for line in f.read_text().splitlines():
            if line.startswith("bytes_per_launch_scaled_to_bench_workload"):
                return float(line.split("=")[1].strip())
    return None


# ------------------------------------------------------------------------------------------------------
# CPU baseline: the reference itself (oracle/_ref), else the CPU restatement
# ------------------------------------------------------------------------------------------------------
class _StdoutToStderr:
    """The reference library prints progress lines on stdout; keep stdout for the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def cpu_eval(x, y, z, q, steps=1):
    with _StdoutToStderr():
        return _cpu_eval(x, y, z, q, steps)


def _cpu_eval(x, y, z, q, steps=1):
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    if O.ref_available():
        times = []
        for _ in range(steps):
            r = O.ref_fmm(O.CHEB_SYM, ORDER, HEIGHT, 1.0, (0.5, 0.5, 0.5), x, y, z, q, nthreads=threads)
            times.append(r["times"]["execute"])
        return times, "reference", threads, "ScalFMM FFmmAlgorithmThread + FChebSymKernel (order 7, height 6) built from " \
                                            "its sources, algo.execute() of the full workload"
    from oracle import precompute as PC

    ranks, uv = PC.pack_reference_layout(PC.sym_operators(ORDER), ORDER)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        O.fmm(O.CHEB_SYM, ORDER, HEIGHT, 1.0, (0.5, 0.5, 0.5), x, y, z, q, sym_ranks=ranks, sym_uv=uv, nthreads=threads)
        times.append(time.perf_counter() - t0)
    return times, "port", threads, "CPU restatement (oracle/fmm_oracle.c) of the full workload"


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = args.n
    x, y, z, q = particles(n)
    from oracle import oracle as O

    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libscalfmm_ref.so was not built"}))
        return 0
    cpu_eval(x, y, z, q, steps=args.warmup)
    times, kind, cores, sample = cpu_eval(x, y, z, q, steps=args.steps)
    total = sum(times)
    value = n * args.steps / total
    line = {"metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(n), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "particles/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------------------
def run_gpu(args):
    import torch
    import torch.distributed as dist

    import scalfmm_b200 as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    # a dedicated (non-default) stream: the library launches on it and the CUDA events are recorded on it
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    n = args.n
    x, y, z, q = particles(n)
    qt = q  # charges of the timed steps: the headline's vector, or nrhs vectors (profiles of the multi-RHS path)
    if args.nrhs > 1:
        qt = np.random.default_rng(SEED + 1).uniform(-1.0, 1.0, (args.nrhs, n)).ravel()
    dx, dy, dz, dq = (torch.from_numpy(a).to(dev) for a in (x, y, z, qt))
    hx, hy, hz, hq = (torch.from_numpy(a).pin_memory() for a in (x, y, z, qt))
    out_h = [torch.empty(n * args.nrhs, dtype=torch.float64).pin_memory() for _ in range(4)]
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    f = S.FMM("cheb_sym", ORDER, args.height, nrhs=args.nrhs, precision=args.precision, device=local,
              stream=stream.cuda_stream)

    def step_device():
        f.set_particles(dx, dy, dz, dq)
        f.execute()

    def step_e2e():
        f.set_particles(hx, hy, hz, hq)
        f.execute()
        f.results_into(*out_h)

    step_device()
    f.autotune()  # M2L work split and near-field work items for this tree shape, kept by the handle
    tuned = f.tuning()
    for _ in range(args.warmup):
        step_device()
        step_e2e()
    torch.cuda.synchronize()
    m2l_pairs, p2p_pairs = f.tree_stats()
    m2l_flops = f.m2l_flops()  # the two products of the low-rank (compressed-operator) tensor-core M2L

    phases = []  # e2e steps: (set_particles from host, execute, get_results to host) in ms

    def step_e2e_phased():
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        f.set_particles(hx, hy, hz, hq)
        ev[1].record(stream)
        f.execute()
        ev[2].record(stream)
        f.results_into(*out_h)
        ev[3].record(stream)
        phases.append(ev)

    def timed(fn, idle_start=False):
        ms = []
        kernel = []
        launches = 0
        for _ in range(args.steps):
            flush.fill_(1.0)
            if idle_start:
                # the library's host-input copies run on a stream of their own: none may begin before the start
                # event, so the stream is idle when it is recorded
                stream.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            e.synchronize()
            ms.append(s.elapsed_time(e))
            kernel.append(f.kernel_times())
            launches += f.launch_count()
        return ms, kernel, launches

    def timed_pipelined():
        # K end-to-end steps in one timed region: each step uploads its inputs from pinned host memory, builds
        # the tree, evaluates and queues its results' copy to pinned host memory on the library's copy stream
        # (get_results_async), which overlaps the next step's upload and tree build; the L2 flush between
        # steps and the last step's copy are inside the region
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches = 0
        stream.synchronize()
        s.record(stream)
        for _ in range(args.steps):
            flush.fill_(1.0)
            f.set_particles(hx, hy, hz, hq)
            f.execute()
            f.results_into_async(*out_h)
            launches += f.launch_count()
        f.join_results()
        e.record(stream)
        e.synchronize()
        return s.elapsed_time(e), launches

    for _ in range(2):  # warm-up of the asynchronous copy path
        step_device()
        f.set_particles(hx, hy, hz, hq)
        f.execute()
        f.results_into_async(*out_h)
    f.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms_dev, ktimes, launches = timed(step_device)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms_e2e, _, launches_e2e = timed(step_e2e_phased, idle_start=True)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t_pipe, launches_pipe = timed_pipelined()
    torch.cuda.synchronize()
    t_dev = sum(ms_dev)
    t_e2e = sum(ms_e2e)
    if world > 1:
        t = torch.tensor([t_dev, t_e2e, t_pipe], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_dev, t_e2e, t_pipe = t.tolist()

    hbm, bf16_sus, bf16_burst, peak_src = measured_peaks()
    m2l_ms = statistics.mean(k["m2l"] for k in ktimes)
    p2p_ms = statistics.mean(k["p2p"] for k in ktimes)
    achieved = m2l_flops / (m2l_ms * 1e-3) / 1e12  # split products counted once
    # the kernel runs about 1.4 ms inside a 3 ms step and the timed region lasts well under a second: the burst
    # figure applies; three FP16 products per logical product
    peak = bf16_burst / 3.0
    traffic = profile_traffic()
    p2p_tflops = p2p_pairs * FLOPS_PER_P2P_PAIR / (p2p_ms * 1e-3) / 1e12
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12

    line = {
        "metric": METRIC, "value": world * n * args.steps / (t_dev * 1e-3), "unit": "particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/f16x3 (mixed), f64 far-field bookkeeping",
        "data": "synthetic", "config": workload_config(n, args.height, args.precision, args.nrhs),
        "e2e": {"value": world * n * args.steps / (t_pipe * 1e-3), "unit": "particles/s",
                "h2d_bytes_per_step": 4 * 8 * n, "d2h_bytes_per_step": 4 * 8 * n,
                "ms_per_step": t_pipe / args.steps,
                "mode": "time-stepping loop through the public API: per step set_particles from pinned host arrays "
                        "(H2D + tree build), execute, get_results_async into pinned host arrays; the results' "
                        "copy of step k overlaps the upload and tree build of step k+1; one timed region over "
                        "all K steps (CUDA events, L2 flushes between steps included, ends after the last copy)",
                "blocking_value": world * n * args.steps / (t_e2e * 1e-3),
                "blocking_ms_per_step": t_e2e / args.steps,
                "blocking_mode": "each step timed alone with the blocking get_results (set_particles, execute, "
                                 "get_results; CUDA events around the step, L2 flushed before it)"},
        "gpu_launches": launches + launches_e2e + launches_pipe,
        "roofline": {"bound": "tensor", "kernel": "lr_y_kernel + m2l_tc_kernel (tcgen05 split-FP16 low-rank M2L)",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "note": f"algorithmic M2L flops per launch = {m2l_flops:.4e}: Y = V^T M per source cell "
                             f"(2 p^3 x the ranks of the slots it feeds) + U Y per pair (2 p^3 r) over {m2l_pairs} "
                             f"pairs, split products counted once; peak = {peak_src} "
                             f"burst bf16 {bf16_burst} TFLOP/s / 3 (three FP16 products per logical product); "
                             f"kernel time {m2l_ms:.3f} ms (CUDA events on the launching stream)"},
        "p2p": {"pairs": p2p_pairs, "kernel_ms": p2p_ms, "gpairs_per_s": p2p_pairs / (p2p_ms * 1e-3) / 1e9,
                "tflops_at_20_per_pair": p2p_tflops, "frac_fp32_peak": p2p_tflops / fp32_peak,
                "fp32_peak_note": "148 SMs x 128 FP32 lanes x 2 x 1965 MHz (nominal)"},
        "pass_ms": f.timings(),
        "e2e_phases_ms": {
            "set_particles_host": statistics.mean(a[0].elapsed_time(a[1]) for a in phases),
            "execute": statistics.mean(a[1].elapsed_time(a[2]) for a in phases),
            "get_results_host": statistics.mean(a[2].elapsed_time(a[3]) for a in phases),
            "note": "set_particles_host = H2D of x, y, z, q (32 MB, pinned) + GPU tree build; get_results_host = "
                    "un-permutation + D2H of phi, fx, fy, fz (32 MB, pinned); tree build alone (device arrays): "
                    "pass_ms.tree"},
        "autotuned": {"m2l_splits": tuned[0], "p2p_whole_leaf": tuned[1], "p2p_item_targets": tuned[2]},
        "clocks": clk.summary(),
    }
    f.close()

    ref_times = None
    if rank == 0 and not args.no_accuracy:
        line["accuracy"], ref_times = accuracy(S, torch, dev, stream, x, y, z, q, pins=not args.no_pins)
        line["multi_rhs"] = multi_rhs_measure(S, torch, dev, stream, x, y, z, pins=not args.no_pins)
        line["ellipsoid"] = ellipsoid_measure(S, torch, dev, stream, pins=not args.no_pins)
    if rank == 0 and not args.no_batch:
        line["batch"] = batch_measure(S, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            if ref_times is None:
                ref_times, kind, cores, sample = cpu_eval(x, y, z, q, steps=1)
            else:
                kind, cores, sample = "reference", os.cpu_count() or 1, REF_SAMPLE
            line["cpu_baseline"] = {"value": n / ref_times[0], "unit": "particles/s", "cores": cores, "kind": kind,
                                    "cpu_model": cpu_model(), "sample": sample}
        except Exception as exc:  # the baseline is reported, never the target
            line["cpu_baseline"] = {"value": None, "unit": "particles/s", "cores": os.cpu_count(), "kind": "reference",
                                    "cpu_model": cpu_model(), "sample": f"failed: {exc}"}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


REF_SAMPLE = ("ScalFMM FFmmAlgorithmThread + FChebSymKernel (order 7, height 6) built from its sources, algo.execute() "
              "of the full workload (the run whose outputs pin the FP64 GPU FMM in accuracy)")
FIELDS = ("phi", "fx", "fy", "fz")


def cpu_model():
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def device_eval(S, torch, f, stream, arrays, reps=3):
    """Best device time (ms) of set_particles (device arrays) + execute over `reps` runs after one untimed run,
    and the results of the last run."""
    f.set_particles(*arrays)
    f.execute()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        f.set_particles(*arrays)
        f.execute()
        e.record(stream)
        e.synchronize()
        ms.append(s.elapsed_time(e))
    return min(ms), f.results()


def timed_create(S, *a, **k):
    t0 = time.perf_counter()
    f = S.FMM(*a, **k)
    return f, 1e3 * (time.perf_counter() - t0)


def accuracy(S, torch, dev, stream, x, y, z, q, pins=True):
    """The headline workload (1M uniform, Chebyshev order 7, height 6):
    * MIXED vs the plain FP64 GPU FMM (same tree, same operators) over all particles, and the time of both;
    * the FP64 GPU FMM loaded with the reference's own compressed operators against the reference's
      FFmmAlgorithmThread + FChebSymKernel on the same particles, all outputs (parity bar 1e-12), and MIXED
      against the same reference outputs;
    * both forms, at order 7 and order 8, against the FP64 direct sum on a seeded 10,000-target subsample;
    * the operator precompute (create()) time of each form.
    Returns the fields and the reference's algo.execute() time (None without the reference)."""
    from oracle import oracle as O

    n = x.size
    out = {}
    res = {}
    arrays = [torch.from_numpy(a).to(dev) for a in (x, y, z, q)]
    for prec in ("fp64", "mixed"):
        f, out[f"{prec}_create_ms"] = timed_create(S, "cheb_sym", ORDER, HEIGHT, precision=prec, device=dev.index,
                                                   stream=stream.cuda_stream)
        out[f"{prec}_ms_per_eval"], res[prec] = device_eval(S, torch, f, stream, arrays)
        out[f"{prec}_pass_ms"] = f.timings()
        if prec == "fp64":
            out["fp64_m2l_flops"] = f.m2l_flops()
            out["fp64_m2l_tflops"] = out["fp64_m2l_flops"] / (out["fp64_pass_ms"]["m2l"] * 1e-3) / 1e12
        f.close()
    out["fp64_particles_per_s"] = n / (out["fp64_ms_per_eval"] * 1e-3)
    out["mixed_over_fp64_speedup"] = out["fp64_ms_per_eval"] / out["mixed_ms_per_eval"]
    for k in FIELDS:
        out[f"mixed_vs_fp64_rel_l2_{k}"] = S.rel_l2(res["mixed"][k], res["fp64"][k])
    t = np.random.default_rng(7).choice(n, 10000, replace=False)
    d = S.direct(x, y, z, q, targets=t)
    for prec in ("fp64", "mixed"):
        for k in FIELDS:
            out[f"{prec}_vs_direct_rel_l2_{k}"] = S.rel_l2(res[prec][k][t], d[k])
    out["gate_mixed_vs_fp64_le_1e-6"] = bool(out["mixed_vs_fp64_rel_l2_phi"] <= 1e-6)
    # order 8: the order at which the FMM's own truncation error drops below 1e-6 against the direct sum
    for prec in ("fp64", "mixed"):
        try:
            f = S.FMM("cheb_sym", 8, HEIGHT, precision=prec, device=dev.index, stream=stream.cuda_stream)
        except S.B200FmmError as exc:  # a form not built for order 8 says so
            out[f"order8_{prec}"] = f"not built: {exc}"
            continue
        ms, r8 = device_eval(S, torch, f, stream, arrays, reps=2)
        f.close()
        out[f"order8_{prec}_ms_per_eval"] = ms
        for k in FIELDS:
            out[f"order8_{prec}_vs_direct_rel_l2_{k}"] = S.rel_l2(r8[k][t], d[k])
        out[f"gate_order8_{prec}_vs_direct_phi_le_1e-6"] = bool(out[f"order8_{prec}_vs_direct_rel_l2_phi"] <= 1e-6)
    ref_times = None
    if pins and O.ref_available():
        with _StdoutToStderr():
            ranks, uv, _, _ = O.ref_sym_operators(ORDER)
            ref = O.ref_fmm(O.CHEB_SYM, ORDER, HEIGHT, 1.0, (0.5, 0.5, 0.5), x, y, z, q, nthreads=os.cpu_count() or 1)
        ref_times = [ref["times"]["execute"]]
        f = S.FMM("cheb_sym", ORDER, HEIGHT, precision="fp64", device=dev.index, stream=stream.cuda_stream)
        f.set_sym_operators(ranks, uv)
        _, r64 = device_eval(S, torch, f, stream, arrays, reps=1)
        f.close()
        for k in FIELDS:
            out[f"pin_fp64_refops_vs_reference_rel_l2_{k}"] = S.rel_l2(r64[k], ref[k])
            out[f"pin_fp64_vs_reference_rel_l2_{k}"] = S.rel_l2(res["fp64"][k], ref[k])
            out[f"pin_mixed_vs_reference_rel_l2_{k}"] = S.rel_l2(res["mixed"][k], ref[k])
        out["pin_gate_fp64_refops_le_1e-12"] = bool(max(out[f"pin_fp64_refops_vs_reference_rel_l2_{k}"]
                                                        for k in FIELDS) <= 1e-12)
        out["pin_reference"] = ("ScalFMM FFmmAlgorithmThread + FChebSymKernel<order 7> (oracle/_ref, built from the "
                                "reference sources), same particles, all outputs; FP64 GPU loaded with the "
                                "reference's compressed operators (FChebSymM2LHandler export)")
        out["pin_reference_times_s"] = ref["times"]
    return out, ref_times


def multi_rhs_measure(S, torch, dev, stream, x, y, z, pins=True, nrhs=16):
    """Multi-RHS workload: the headline positions with 16 independent charge vectors U[-1,1] on one tree,
    Chebyshev order 7, height 6.  MIXED throughput (particles x RHS per second, device time of set_particles +
    execute), the M2L's algorithmic rate, MIXED vs the FP64 GPU FMM, and the FP64 GPU FMM (reference operators)
    against the reference's FFmmAlgorithmThread with NVALS = 16 on the same inputs."""
    from oracle import oracle as O

    n = x.size
    qm = np.random.default_rng(SEED + 1).uniform(-1.0, 1.0, (nrhs, n))
    arrays = [torch.from_numpy(a).to(dev) for a in (x, y, z, qm.ravel())]
    out = {"workload": f"{n} uniform particles (the headline positions) x {nrhs} charge vectors U[-1,1] (seed "
                       f"{SEED + 1}), Chebyshev order 7, height 6", "nrhs": nrhs}
    f = S.FMM("cheb_sym", ORDER, HEIGHT, nrhs=nrhs, precision="mixed", device=dev.index, stream=stream.cuda_stream)
    ms, rm = device_eval(S, torch, f, stream, arrays)
    f.set_particles(*arrays)
    f.execute()
    kt = f.kernel_times()
    flops = f.m2l_flops()
    _, bf16_sus, bf16_burst, src = measured_peaks()
    f.close()
    out["mixed_ms_per_eval"] = ms
    out["particle_rhs_per_s"] = n * nrhs / (ms * 1e-3)
    out["m2l"] = {"kernel_ms": kt["m2l"], "flops": flops, "achieved_tflops": flops / (kt["m2l"] * 1e-3) / 1e12,
                  "frac": flops / (kt["m2l"] * 1e-3) / 1e12 / (bf16_burst / 3.0),
                  "peak_note": f"{src} burst bf16 {bf16_burst} TFLOP/s / 3"}
    f = S.FMM("cheb_sym", ORDER, HEIGHT, nrhs=nrhs, precision="fp64", device=dev.index, stream=stream.cuda_stream)
    ranks = uv = None
    if pins and O.ref_available():
        with _StdoutToStderr():
            ranks, uv, _, _ = O.ref_sym_operators(ORDER)
        f.set_sym_operators(ranks, uv)
    ms64, r64 = device_eval(S, torch, f, stream, arrays, reps=1)
    f.close()
    out["fp64_ms_per_eval"] = ms64
    for k in FIELDS:
        out[f"mixed_vs_fp64_rel_l2_{k}"] = S.rel_l2(rm[k], r64[k])
    if ranks is not None:
        with _StdoutToStderr():
            ref = O.ref_fmm(O.CHEB_SYM, ORDER, HEIGHT, 1.0, (0.5, 0.5, 0.5), x, y, z, qm,
                            nthreads=os.cpu_count() or 1)
        for k in FIELDS:
            out[f"pin_fp64_refops_vs_reference_rel_l2_{k}"] = S.rel_l2(r64[k], ref[k])
        out["pin_gate_fp64_refops_le_1e-12"] = bool(max(out[f"pin_fp64_refops_vs_reference_rel_l2_{k}"]
                                                        for k in FIELDS) <= 1e-12)
        out["pin_reference"] = "ScalFMM FFmmAlgorithmThread + FChebSymKernel<order 7, NVALS 16> (oracle/_ref)"
        out["pin_reference_times_s"] = ref["times"]
    return out


def ellipsoid_measure(S, torch, dev, stream, pins=True, n=2_000_000):
    """Ellipsoid-surface workload: 2M area-uniform points on the surface of the ellipsoid with semi-axes
    (0.5, 0.3, 0.2) centred in the unit cube, charges U[0,1], Lagrange (uniform) interpolation order 6, height 7.
    MIXED throughput, MIXED vs the FP64 GPU FMM, the FP64 GPU FMM against the C restatement of the reference's
    FUnifKernel FMM (oracle/fmm_oracle.c) on all particles, and both against the direct sum on 10,000 targets."""
    from distributions import ellipsoid_surface
    from oracle import oracle as O

    x, y, z = ellipsoid_surface(n, 3)
    q = np.random.default_rng(4).random(n)
    arrays = [torch.from_numpy(a).to(dev) for a in (x, y, z, q)]
    out = {"workload": f"{n} area-uniform points on the ellipsoid (0.5, 0.3, 0.2) surface centred in the unit cube "
                       "(seed 3), q~U[0,1] (seed 4), Lagrange order 6, height 7"}
    res = {}
    for prec in ("mixed", "fp64"):
        f = S.FMM("lagrange", 6, 7, precision=prec, device=dev.index, stream=stream.cuda_stream)
        out[f"{prec}_ms_per_eval"], res[prec] = device_eval(S, torch, f, stream, arrays, reps=3 if prec == "mixed" else 1)
        out[f"{prec}_pass_ms"] = f.timings()
        if prec == "mixed":
            nc, _ = f.tree_info()
            out["cells_per_level"] = [int(v) for v in nc]
            out["m2l_pairs"], out["p2p_pairs"] = f.tree_stats()
        f.close()
    out["mixed_particles_per_s"] = n / (out["mixed_ms_per_eval"] * 1e-3)
    for k in FIELDS:
        out[f"mixed_vs_fp64_rel_l2_{k}"] = S.rel_l2(res["mixed"][k], res["fp64"][k])
    t = np.random.default_rng(7).choice(n, 10000, replace=False)
    d = S.direct(x, y, z, q, targets=t)
    for prec in ("fp64", "mixed"):
        for k in ("phi", "fx"):
            out[f"{prec}_vs_direct_rel_l2_{k}"] = S.rel_l2(res[prec][k][t], d[k])
    if pins:
        t0 = time.perf_counter()
        o = O.fmm(O.LAGRANGE, 6, 7, 1.0, (0.5, 0.5, 0.5), x, y, z, q)
        out["pin_oracle_s"] = time.perf_counter() - t0
        for k in FIELDS:
            out[f"pin_fp64_vs_oracle_rel_l2_{k}"] = S.rel_l2(res["fp64"][k], o[k])
        out["pin_gate_fp64_le_1e-12"] = bool(max(out[f"pin_fp64_vs_oracle_rel_l2_{k}"] for k in FIELDS) <= 1e-12)
        out["pin_reference"] = "C restatement of FUnifKernel's FMM (oracle/fmm_oracle.c, pinned against the reference)"
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
