"""Benchmark: PD iterations/s of the Cartesian ICTGV2 reconstruction on B200.

Workload (one step): one full reconstruction of the cine-like Cartesian
ICTGV2 problem, 192 x 192 pixels, 30 frames, 16 coils, complex64, 1000 PD
iterations, variable-density line mask at acceleration 12 (seeded synthetic
data of the benchmark's shapes; the reference's public data is not
available).  Parameters are the reference's default configuration file's
[ictgv2] section (timeSpaceWeight 4 / 0.5, alpha 0.5, alpha0 sqrt 2,
alpha1 1, lambda 6, sigma = tau = 0.3333), no gap evaluation (-g 0), the
reference's step-rule schedule.

  value  PD iterations/s, inputs resident in HBM, whole job over all ranks
  e2e    the same metric through the host-buffer C entry point
         (avx_reconstruct_host): host -> device copy of k-space, mask, coil
         maps and u0 and device -> host copy of the image inside the timed region
Multi-GPU: one independent reconstruction per rank (instances shard with no
collective); barrier + max-over-ranks device time.

--impl reference times the reference algorithm's CPU restatement (the
float64 oracle; the reference's own C++/CUDA and MATLAB code cannot run
here) on a bounded sample of the same workload.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PD iters/s, recons/s & p99 latency vs plain FP32 at <=1e-4 rel L2 err"
UNIT = "PD it/s"
ITERS = 1000
WORKLOAD = "config1 Cartesian ICTGV2 cine-like 192x192x30 frames x16 coils, R=12 line mask, 1000 PD iterations/recon"


def cfg_params(av):
    p = av.default_params(av.ICTGV2)
    p.maxIt = ITERS
    p.stopPDGap = 0.0
    p.sigma = p.tau = 0.3333
    p.sigmaTauRatio = 1.0
    p.timeSpaceWeight, p.timeSpaceWeight2 = 4.0, 0.5
    p.alpha, p.alpha0, p.alpha1 = 0.5, 1.41421356, 1.0
    p.lambda_ = 6.0
    p.adaptLambda = 0
    return p


def algorithmic_bytes(W, H, T, C, R):
    """Compulsory bytes per ICTGV2 iteration by stage (complex64 = 8 B).
    N = W*H*T pixels; S = C*R*W compact k-space values (R sampled rows over
    all frames)."""
    N = W * H * T
    S = C * R * W
    P, D = 8, 18
    return {
        # read xbar (P), read + write y (2D)
        "dual": 8 * N * (P + 2 * D),
        # read xbar1, b1; write the y-transformed rows
        "ydft": 8 * N + 8 * C * W * H + 8 * S,
        # read rows, z, d, mask; write z, Q'
        "rows": 8 * 5 * S + 4 * R * W,
        # read Q', b1; write K^H z
        "coladj": 8 * S + 8 * C * W * H + 8 * N,
        # read K^H z, x (P), y (D); write x, xbar (2P)
        "primal": 8 * N * (1 + 3 * P + D),
        # the whole iteration, the formula of the scope table: 8 [4PN + 2DN + 3CS] + 8 C W H + 4 S
        "iteration": 8 * (4 * P * N + 2 * D * N + 3 * S) + 8 * C * W * H + 4 * R * W,
    }


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """DRAM bytes per launch by kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "kernel_traffic.txt")
    out = {}
    if os.path.exists(path):
        for ln in open(path):
            f = ln.split()
            if len(f) >= 2 and not ln.startswith("#"):
                try:
                    out[f[0]] = float(f[1])
                except ValueError:
                    pass
    return out


def cpu_oracle_rate(prob, n_iter, workers):
    """PD it/s of the float64 oracle on the same problem (first n_iter
    iterations, step rule active at k < 10)."""
    from oracle import cartesian as ocart
    from oracle import solvers as so
    ocart.FFT_WORKERS = workers
    T, C, H, W = prob["kdata"].shape
    op = ocart.CartesianOperator(W, H, C, T, mask=prob["mask"], centered=False)
    p = so.init_params("ICTGV2")
    p.maxIt = n_iter
    p.sigma = p.tau = 0.3333
    p.timeSpaceWeight, p.timeSpaceWeight2 = 4.0, 0.5
    p.alpha, p.alpha0, p.alpha1 = 0.5, 1.41421356, 1.0
    p.lam = 6.0
    u0 = prob["u0"]
    x0 = np.repeat(u0[None].astype(complex), T, axis=0)
    d = prob["kdata"].astype(complex)
    b1 = prob["b1"].astype(complex)
    t0 = time.perf_counter()
    so.ictgv2(d, x0, b1, op, p)
    dt = time.perf_counter() - t0
    return n_iter / dt, dt


def make_problem(seed):
    from avionic_b200 import synth
    prob = synth.config1(seed)
    prob["u0"] = synth.time_average_u0(prob["kdata"], prob["mask"], prob["b1"])
    return prob


def run_reference(args, rank, world):
    """The reference arm: the oracle port on the host cores, rank 0 only."""
    if rank != 0:
        return
    workers = os.cpu_count() or 1
    prob = make_problem(1)
    n = max(1, args.ref_iters)
    for _ in range(args.warmup):
        cpu_oracle_rate(prob, 1, workers)
    rates, times = [], []
    for _ in range(args.steps):
        r, dt = cpu_oracle_rate(prob, n, workers)
        rates.append(r)
        times.append(dt)
    value = float(np.sum([n for _ in rates]) / np.sum(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": "%d PD iterations per step" % n},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port",
                         "sample": "%d steps x %d ICTGV2 iterations of the float64 oracle (scipy.fft workers=%d)"
                                   % (args.steps, n, workers)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-iters", type=int, default=2)
    ap.add_argument("--cpu-iters", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dft", default="split", choices=["split", "fp32"],
                    help="arithmetic of the y-transforms: split-BF16x3 tensor cores or fp32 CUDA cores")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import avionic_b200 as av

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    prob = make_problem(1 + rank)
    T, C, H, W = prob["kdata"].shape
    kd = av.to_device(prob["kdata"])
    md = av.to_device(prob["mask"])
    b1 = av.to_device(prob["b1"])
    x0 = av.to_device(np.repeat(prob["u0"][None], T, axis=0))
    x = torch.empty_like(x0)
    op = av.CartesianOperator(W, H, C, T, mask=md, centered=False)
    op.dft_mode = av.DFT_SPLIT_BF16X3 if args.dft == "split" else av.DFT_FP32
    solver = av.Solver(av.ICTGV2, op, cfg_params(av))
    solver.set_debug(False, 0)
    R = int(np.count_nonzero(prob["mask"].any(axis=2)))

    # warm-up: kernels, buffers and the CUDA graphs of the iteration shapes are set up here
    solver.set_timing(False)
    for _ in range(args.warmup):
        x.copy_(x0)
        solver.run(kd, x, b1)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    lat = []
    e0.record()
    for _ in range(args.steps):
        s0 = torch.cuda.Event(enable_timing=True)
        s0.record()
        x.copy_(x0)
        solver.run(kd, x, b1)
        s1 = torch.cuda.Event(enable_timing=True)
        s1.record()
        lat.append((s0, s1))
        launches += solver.stats().kernel_launches + 3  # + row gather and two set-up reductions
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    step_ms = [a.elapsed_time(b) for a, b in lat]
    if dist is not None:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * args.steps * ITERS / (ms / 1000.0)

    # the other arithmetic of the y-transforms, same problem and schedule (reported beside the headline)
    other = None
    if args.dft == "split" and op.dft_mode == av.DFT_SPLIT_BF16X3:
        op.dft_mode = av.DFT_FP32
        for _ in range(2):
            x.copy_(x0)
            solver.run(kd, x, b1)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        for _ in range(args.steps):
            x.copy_(x0)
            solver.run(kd, x, b1)
        g1.record()
        torch.cuda.synchronize()
        x_fp32 = x.clone()
        other = {"dft": "fp32 CUDA cores", "value": world * args.steps * ITERS / (g0.elapsed_time(g1) / 1000.0),
                 "unit": UNIT}
        op.dft_mode = av.DFT_SPLIT_BF16X3
        x.copy_(x0)
        solver.run(kd, x, b1)
        torch.cuda.synchronize()
        other["rel_l2_split_vs_fp32"] = float(torch.linalg.vector_norm(x - x_fp32) /
                                              torch.linalg.vector_norm(x_fp32))

    # per-stage durations: one more reconstruction with CUDA events between the
    # stages of every iteration (kernels launched directly, not from graphs)
    solver.set_timing(True)
    x.copy_(x0)
    solver.run(kd, x, b1)
    torch.cuda.synchronize()
    t_stage, n_timed = solver.kernel_times()
    solver.set_timing(False)
    kmean = np.array(t_stage)

    # roofline of the dominant kernel (largest mean duration per iteration)
    ab = algorithmic_bytes(W, H, T, C, R)
    names = ["dual", "ydft", "rows", "coladj", "primal"]
    dom = int(np.argmax(kmean))
    peak, peak_kind = load_peaks()
    achieved = ab[names[dom]] / (kmean[dom] / 1000.0) / 1e9
    traffic = load_traffic().get(names[dom])
    iter_ms = float(np.sum(kmean))
    kern = {"dual": "dual_kernel", "ydft": "ydft_kernel", "rows": "rows_kernel", "coladj": "coladj_kernel",
            "primal": "primal_kernel"}
    roof = {"bound": "hbm", "kernel": kern[names[dom]], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"
            if peak_kind == "measured" else "fallback 6650 GB/s", "traffic": traffic,
            "algorithmic_bytes_per_launch": ab[names[dom]],
            "kernel_ms": {n: float(kmean[i]) for i, n in enumerate(names)},
            "kernel_ms_source": "CUDA events around each stage, %d iterations of one extra reconstruction "
                                "after the timed region" % n_timed,
            "iteration_algorithmic_bytes": ab["iteration"],
            "iteration_frac": ab["iteration"] / (iter_ms / 1000.0) / 1e9 / peak}

    # end-to-end through the host-buffer entry point (pinned host buffers)
    pk = torch.from_numpy(prob["kdata"]).pin_memory()
    pm = torch.from_numpy(prob["mask"]).pin_memory()
    pb = torch.from_numpy(prob["b1"]).pin_memory()
    pu = torch.from_numpy(prob["u0"]).pin_memory()
    px = torch.empty((T, H, W), dtype=torch.complex64).pin_memory()
    import ctypes
    params = cfg_params(av)
    st = av.RunStats()

    def host_call():
        av.check(av.lib.avx_reconstruct_host(
            av.ICTGV2, W, H, C, T, ctypes.byref(params), 0, ctypes.c_void_p(pk.data_ptr()),
            ctypes.c_void_p(pm.data_ptr()), ctypes.c_void_p(pb.data_ptr()), ctypes.c_void_p(pu.data_ptr()),
            ctypes.c_void_p(px.data_ptr()), ctypes.byref(st)))

    host_call()
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(args.steps):
        host_call()
    f1.record()
    torch.cuda.synchronize()
    barrier()
    ems = f0.elapsed_time(f1)
    if dist is not None:
        tt = torch.tensor([ems], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ems = float(tt.item())
    e2e_value = world * args.steps * ITERS / (ems / 1000.0)
    av.lib.avx_reconstruct_host_release()
    h2d = pk.numel() * 8 + pm.numel() * 4 + pb.numel() * 8 + pu.numel() * 8
    d2h = px.numel() * 8

    # accuracy of this run against the float64 oracle is checked by the tests;
    # here: sanity that the image is finite
    assert torch.isfinite(torch.view_as_real(x)).all().item()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, dt = cpu_oracle_rate(prob, args.cpu_iters, 1)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "first %d ICTGV2 iterations of the float64 oracle on this problem (%.1f s, numpy, 1 thread;"
                         " step rule active at k<10)" % (args.cpu_iters, dt)}

    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": ("bf16x3-split y-DFTs on tensor cores (fp32 accumulate), f32 elsewhere" if args.dft == "split"
                  else "f32 (complex64)"),
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": "one independent reconstruction per GPU",
                   "l2": "inputs larger than L2 (working set ~0.4 GB per GPU)", "graphs": True,
                   "recons_per_s": value / ITERS,
                   "dft": args.dft, "other_dft_form": other,
                   "recon_latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                                        "p99": float(np.percentile(step_ms, 99))}},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": int(launches * world),
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
