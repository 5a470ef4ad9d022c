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
collective); barrier + max-over-ranks device time.  The batched
configuration's 64 instances are partitioned across ranks by device
footprint; its wall time is the slowest rank's.

--impl reference times the reference algorithm's CPU restatement (the
float64 oracle; the reference's own C++/CUDA and MATLAB code cannot run
here) on a bounded sample of the same workload: the step-rule iterations
k < 10 run as warm-up, every timed step runs --ref-iters iterations from k =
10 on (the reconstruction's common, fixed-step iteration), on all host cores.
That process never loads the library.

Accuracy: where a float64-oracle fixture of the same seeded problem exists
(tests/golden/oracle/, made by tests/golden/make_oracle_fixtures.py) the line
reports the relative L2 image error against it (rel_l2_vs_oracle).
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
WORKLOAD = "Cartesian ICTGV2 cine-like 192x192, 30 frames, 16 coils, R=12 line mask, 1000 PD iterations/recon"


# The line's config: the same dict in both arms (the reference arm's sample
# size and this arm's launch details are reported beside it, not in it).
CONFIG = {"workload": WORKLOAD, "iterations_per_recon": ITERS,
          "inputs": "seeded synthetic problem of the benchmark's shapes (synth.cine_192_problem, seed 1 + rank)",
          "l2": "inputs larger than L2 (working set ~0.4 GB per GPU)"}
FIXTURES = os.path.join(ROOT, "tests", "golden", "oracle")


def cfg_params(av):
    from avionic_b200 import synth
    p = av.default_params(av.ICTGV2)
    for k, v in synth.CINE_192_PARAMS.items():
        setattr(p, "lambda_" if k == "lambda" else k, v)
    p.adaptLambda = 0
    return p


def oracle_fixture(name):
    """The float64-oracle fixture `name` (a dict of arrays) or None."""
    path = os.path.join(FIXTURES, name + ".npz")
    if not os.path.exists(path):
        return None
    with np.load(path) as f:
        return {k: f[k] for k in f.files}


def rel_l2(x, ref):
    """||x - ref|| / ||ref|| in float64 (x a torch tensor or numpy array)."""
    a = x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)
    a = a.astype(np.complex128).ravel()
    b = np.asarray(ref).astype(np.complex128).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def vs_oracle(name, x):
    fx = oracle_fixture(name)
    return None if fx is None else rel_l2(x, fx["x"])


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
        # the whole iteration: fields read and written once, z and d at the
        # sampled values, b1 once, the kept rows' mask: 8 [4PN + 2DN + 3CS] + 8 C W H + 4 R W
        "iteration": 8 * (4 * P * N + 2 * D * N + 3 * S) + 8 * C * W * H + 4 * R * W,
        # the same with the reference's dense layout (z and d at all C N
        # k-space points, the mask as 4 N bytes), for comparison only
        "iteration_dense_layout": 8 * (4 * P * N + 2 * D * N + 3 * C * N) + 8 * C * W * H + 4 * N,
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


def tensor_roofline(mask, W, H, T, C, ydft_ms, coladj_ms):
    """Tensor-pipe roofline of the two split-BF16x3 kernels: the bf16 MMA FLOPs
    they issue per launch (six piece products; tiles as tc_dft.cu launches
    them: M = 128 (coil, column) pairs x N = 2 x rows per frame (padded to 16)
    x K = 2H for the y-transform, M = 128 image rows x N = 16 coils x 8
    columns x 2 x K = N' for the column adjoint) over the stage means, against
    the sustained bf16 figure of MEASURED_PEAKS.json (kernels timed inside a
    long reconstruction)."""
    rows = max(int(np.count_nonzero(np.any(mask[t] != 0, axis=1))) for t in range(T))
    npad = max(16, (2 * rows + 15) // 16 * 16)
    ceil = lambda a, b: -(-a // b)  # noqa: E731
    mma = lambda m, n, k: 2 * m * n * k  # noqa: E731
    ydft = T * ceil(C * W, 128) * ceil(2 * H, 32) * 2 * 6 * mma(128, npad, 16)
    coladj = T * ceil(H, 128) * ceil(W, 8) * sum(
        (npad // 16) * 6 * mma(128, ceil(2 * 8 * min(16, C - c0), 16) * 16, 16) for c0 in range(0, C, 16))
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, src = float(json.load(f)["bf16_tflops_sustained"]), "measured sustained"
    except Exception:
        peak, src = 1400.0, "fallback sustained"
    out = {"peak_tflops": peak, "peak_source": src + " (MEASURED_PEAKS.json bf16_tflops_sustained)",
           "n_per_mma_y_transform": npad}
    for name, fl, ms in (("ydft_tc", ydft, ydft_ms), ("coladj_tc", coladj, coladj_ms)):
        t = fl / (ms / 1000.0) / 1e12
        out[name] = {"bf16_mma_gflop_per_launch": fl / 1e9, "achieved_tflops": t, "frac": t / peak}
    return out


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


def cpu_oracle_seconds(method, prob, n_iter, workers, k0):
    """Seconds the float64 oracle takes for n_iter iterations of `method` on
    the problem, its iteration counter starting at k0 (k0 = 10 skips the
    step-rule start: iterations 10 .. 49 are fixed-step ones, the kind 971 of
    the benchmark's 1000 are).  scipy.fft runs the 2D transforms on `workers`
    threads."""
    from avionic_b200 import synth
    from oracle import cartesian as ocart
    from oracle import solvers as so
    ocart.FFT_WORKERS = workers
    T, C, H, W = prob["kdata"].shape
    op = ocart.CartesianOperator(W, H, C, T, mask=prob["mask"], centered=False)
    p = so.init_params(method)
    if method == "ICTGV2":
        for k, v in synth.CINE_192_PARAMS.items():
            setattr(p, "lam" if k == "lambda" else k, v)
    else:
        p.lam = op.adapt_lambda(*p.adapt_kd)
    p.maxIt = k0 + n_iter
    x0 = np.repeat(prob["u0"][None].astype(complex), T, axis=0)
    d = prob["kdata"].astype(complex)
    b1 = prob["b1"].astype(complex)
    t0 = time.perf_counter()
    so.run(method, d, x0, b1, op, p, None, k0)
    return time.perf_counter() - t0


def make_problem(seed):
    from avionic_b200 import synth
    return synth.cine_192_problem(seed)


def _batch_pass(av, torch, items, make_request, workers, dft, arrivals=None):
    """Runs one request per item through a BatchEngine with the given worker
    count and DFT form.  arrivals (seconds from the start, sorted) turns the
    submissions into an open-loop arrival stream; otherwise every request is
    submitted at once.  Returns the per-request completions, the outputs and
    the wall time from the first submission to the last completion."""
    outs = [it["x0"].clone() for it in items]
    torch.cuda.synchronize()
    eng = av.BatchEngine(0, hbm_budget=150 << 30, workers=workers)
    reqs = [make_request(it, out, dft, i) for i, (it, out) in enumerate(zip(items, outs))]
    done = {}
    t0 = time.perf_counter()
    for i, r in enumerate(reqs):
        if arrivals is not None:
            while True:
                lag = arrivals[i] - (time.perf_counter() - t0)
                if lag <= 0:
                    break
                got = eng.poll(wait_ms=max(1, int(lag * 1000)))
                for c in got:
                    done[c.tag] = (c, time.perf_counter() - t0)
                if not got:
                    time.sleep(min(lag, 0.002))  # nothing pending: poll returns at once
        eng.submit(r)
        for c in eng.poll(wait_ms=0):
            done[c.tag] = (c, time.perf_counter() - t0)
    while len(done) < len(reqs):
        for c in eng.poll(wait_ms=-1):
            done[c.tag] = (c, time.perf_counter() - t0)
    wall = max(t for _, t in done.values())
    eng.close()
    comps = [done[i][0] for i in range(len(reqs))]
    bad = [c.status for c in comps if c.status != 0]
    if bad:
        raise RuntimeError("batched requests failed with status %s" % bad[:4])
    return comps, outs, wall


def _rel_diff(torch, a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def run_batched(av, torch, workers, n=64, iters=800, rank=0, world=1, dist=None):
    """The batched configuration: n TGV2 reconstructions of uneven size
    (800 iterations each), submitted at once.  The plain form is FP32
    y-transforms with one reconstruction at a time (workers = 1); the batched
    form is split-BF16x3 with `workers` concurrent reconstructions.  With
    several ranks the instances are partitioned by device footprint (complex
    values: the TGV2 fields and the k-space) and every rank runs its share;
    the wall time is the slowest rank's."""
    from avionic_b200 import synth
    specs = synth.batched_specs(3, n)
    owner = shard_by_footprint([sp["W"] * sp["H"] * sp["T"] * (21 + sp["C"]) for sp in specs], world)
    with_fixture = set(synth.oracle_batched_indices(3, n)) if n == 64 else set()
    items, fixture_of = [], []
    for i, (sp, o) in enumerate(zip(specs, owner)):
        if o != rank:
            continue
        if i in with_fixture:  # generated on the host: the oracle fixture's exact inputs
            h = synth.cine_instance(sp)
            items.append(dict(kdata=av.to_device(h["kdata"]), mask=av.to_device(h["mask"]),
                              b1=av.to_device(h["b1"]), x0=av.to_device(np.repeat(h["u0"][None], sp["T"], axis=0))))
            fixture_of.append("batched_%d" % i)
        else:
            items.append(synth.cine_instance_gpu(sp))
            fixture_of.append(None)
    torch.cuda.synchronize()

    def make_request(it, out, dft, tag):
        p = av.default_params(av.TGV2)
        p.maxIt = iters
        return av.cartesian_request(av.TGV2, it["kdata"], out, it["b1"], mask=it["mask"], params=p,
                                    dft_mode=dft, tag=tag)

    _batch_pass(av, torch, items[:4], make_request, 2, av.DFT_SPLIT_BF16X3)  # warm-up: module loading
    forms = {}
    outs = {}
    for name, w, dft in (("plain_fp32_single", 1, av.DFT_FP32), ("split_single", 1, av.DFT_SPLIT_BF16X3),
                         ("fp32_batched", workers, av.DFT_FP32), ("split_batched", workers, av.DFT_SPLIT_BF16X3)):
        comps, o, wall = _batch_pass(av, torch, items, make_request, w, dft)
        wall = max_over_ranks(dist, wall, "cuda")
        its = sum_over_ranks(dist, sum(c.stats.iterations for c in comps), "cuda")
        lat = [c.queue_ms + c.run_ms for c in comps]  # this rank's requests
        forms[name] = {"workers": w, "recons_per_s": n / wall, "pd_it_per_s": its / wall, "wall_s": wall,
                       "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
                       "split_dft_instances": int(sum(c.dft_mode == av.DFT_SPLIT_BF16X3 for c in comps))}
        outs[name] = o
    ref = outs["plain_fp32_single"]
    fixtures = {f: oracle_fixture(f) for f in fixture_of if f}
    for name in forms:
        forms[name]["max_rel_l2_vs_plain_fp32"] = max_over_ranks(
            dist, max(_rel_diff(torch, a, b) for a, b in zip(outs[name], ref)), "cuda")
        errs = [rel_l2(o, fixtures[f]["x"]) for o, f in zip(outs[name], fixture_of) if f and fixtures[f] is not None]
        # every rank takes part in the reductions, with or without fixture instances
        e = max_over_ranks(dist, max(errs) if errs else -1.0, "cuda")
        forms[name]["max_rel_l2_vs_oracle"] = e if e >= 0 else None
        forms[name]["oracle_instances"] = int(sum_over_ranks(dist, len(errs), "cuda"))
    del items, outs
    torch.cuda.empty_cache()
    # the whole set's compulsory HBM traffic (each field read and written once per iteration, k-space at
    # its sampled rows) at the measured copy bandwidth: the time no form can beat
    peak, _ = load_peaks()
    ideal_bytes = 0
    for sp in specs:
        Ns = sp["W"] * sp["H"] * sp["T"]
        rows = sp["T"] * max(1, int(round(sp["H"] / sp["R"])))
        Ss = sp["C"] * rows * sp["W"]
        ideal_bytes += 8 * (4 * 4 * Ns + 2 * 9 * Ns + 3 * Ss) + 8 * sp["C"] * sp["W"] * sp["H"] + 4 * rows * sp["W"]
    ideal_s = ideal_bytes * iters / (peak * 1e9) / world
    for name in forms:
        forms[name]["frac_of_hbm_roofline"] = ideal_s / forms[name]["wall_s"]
    return {"workload": "%d TGV2 Cartesian reconstructions of uneven size (matrix 96-320, frames 8-48, coils 4-32, "
                        "acceleration 6-16), %d iterations each, submitted at once" % (n, iters),
            "hbm_roofline_s": ideal_s,
            "forms": forms,
            "speedup_split_batched_vs_plain_fp32_single": forms["split_batched"]["recons_per_s"] /
            forms["plain_fp32_single"]["recons_per_s"],
            "timing": "host wall clock from the first submission to the last completion (several streams)"
                      + ("; slowest of %d ranks, latencies of rank 0's share" % world if world > 1 else "")}


def run_serving(av, torch, workers, n, rates, max_it=1500, rel_gap=1e-4):
    """The serving configuration on a bounded sample: n requests (50/30/20 %
    TV/TGV2/ICTGV2, 70/30 % Cartesian/radial) arriving as a Poisson stream at
    each rate; every request stops at max_it iterations or once its
    normalised primal-dual gap (the gap over the pixel count, the reference's
    stop test, tgv2.cpp:317-330) falls below rel_gap, evaluated every 20
    iterations."""
    from avionic_b200 import synth
    specs = synth.serving_stream(4, n, 1.0)
    items = []
    for sp in specs:
        it = synth.cine_instance_gpu(sp) if sp["kind"] == "cartesian" else synth.radial_instance_gpu(sp)
        it["spec"] = sp
        items.append(it)
    torch.cuda.synchronize()

    def make_request(it, out, dft, tag):
        sp = it["spec"]
        p = av.default_params(av.METHODS[sp["method"]])
        p.maxIt = max_it
        p.stopPDGap = rel_gap
        if sp["kind"] == "cartesian":
            return av.cartesian_request(sp["method"], it["kdata"], out, it["b1"], mask=it["mask"], params=p,
                                        dft_mode=dft, tag=tag)
        return av.radial_request(sp["method"], it["kdata"], out, it["b1"], it["traj"], it["dens"], it["spokes"],
                                 it["n_fe"], params=p, kernel_width=it["kernel_width"],
                                 sector_width=it["sector_width"], osf=it["osf"], tag=tag)

    unit_arrivals = np.array([sp["arrival"] for sp in specs])
    res = {}
    outs = {}
    for name, w, dft in (("plain_fp32_single", 1, av.DFT_FP32), ("split_batched", workers, av.DFT_SPLIT_BF16X3)):
        per_rate = []
        for rate in rates:
            comps, o, wall = _batch_pass(av, torch, items, make_request, w, dft, arrivals=unit_arrivals / rate)
            lat = [c.queue_ms + c.run_ms for c in comps]
            gaps = [c.stats.last_gap for c in comps if c.stats.gap_count > 0]
            per_rate.append({"rate_req_per_s": rate, "recons_per_s": n / wall, "wall_s": wall,
                             "latency_ms": {q: float(np.percentile(lat, v)) for q, v in
                                            (("p50", 50), ("p95", 95), ("p99", 99))},
                             "iterations_mean": float(np.mean([c.stats.iterations for c in comps])),
                             "stopped_by_gap": int(sum(c.stats.stopped_by_gap for c in comps)),
                             "last_normalised_gap": {"min": float(np.min(gaps)), "p50": float(np.median(gaps))}
                             if gaps else None})
            outs[name] = o
        res[name] = {"workers": w, "per_rate": per_rate}
    res["max_rel_l2_split_batched_vs_plain_fp32"] = max(
        _rel_diff(torch, a, b) for a, b in zip(outs["split_batched"], outs["plain_fp32_single"]))
    del items, outs
    torch.cuda.empty_cache()
    return {"workload": "%d requests (sample of the 2000-request stream): 50/30/20%% TV/TGV2/ICTGV2, 70%% Cartesian "
                        "(matrix 96-320, frames 8-48, coils 4-32) / 30%% radial (128x128, 256 readout samples, 13-34 "
                        "spokes/frame, 20-60 frames, 12 coils), stop at normalised gap %g (gap / pixels) or %d "
                        "iterations, HBM budget 150 GB" % (n, rel_gap, max_it),
            "forms": res,
            "timing": "host wall clock; latency = submission (arrival) to completion"}


def run_radial(av, torch, steps=3):
    """The radial configuration: H1 coil-sensitivity estimation from the data,
    then a TGV2 reconstruction (500 iterations, the reference's default) with
    the Kaiser-Bessel gridding operator (width 3, grid oversampling 1.5,
    sector width 8), the CLI's flow for radial data without coil maps."""
    import ctypes
    from avionic_b200 import synth
    prob = synth.radial_128(2)  # generated on the host: the oracle fixture's exact inputs
    k, traj, dens = av.to_device(prob["kdata"]), av.to_device(prob["traj"]), av.to_device(prob["dens"])
    T, C, S = k.shape
    H, W = prob["truth"].shape[1:]
    q = av.coil_default_params()
    u = torch.empty((C, H, W), dtype=torch.complex64, device="cuda")
    b1 = torch.empty_like(u)

    def coils():
        av.check(av.lib.avx_coil_construction_radial(W, H, C, T, S, ctypes.byref(q), av._cptr(traj), av._cptr(dens),
                                                     av._cptr(k), av._cptr(u), av._cptr(b1)))

    coils()
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    coil_runs = []
    for _ in range(5):  # the median of five runs (the host-driven greedy steps vary run to run)
        c0.record()
        coils()
        c1.record()
        torch.cuda.synchronize()
        coil_runs.append(c0.elapsed_time(c1))
    coil_ms = float(np.median(coil_runs))
    x0 = (u[C - 1] / T)[None].repeat(T, 1, 1).contiguous()  # u0 of the radial coil construction (main.cpp:636-640)
    op = av.RadialOperator(W, H, C, T, traj, dens, prob["spokes"], 3.0, 8.0, 1.5)
    p = av.default_params(av.TGV2)
    p.maxIt = synth.RADIAL_ITERS
    solver = av.Solver(av.TGV2, op, p)
    p = solver.params  # lambda adapted at creation; every run starts from these sigma, tau
    x = torch.empty_like(x0)
    for _ in range(2):
        x.copy_(x0)
        solver.params = p
        solver.run(k, x, b1)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        x.copy_(x0)
        solver.params = p
        solver.run(k, x, b1)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    err = rel_l2(x, prob["truth"])
    err_oracle = vs_oracle("radial_128", x)
    solver.set_timing(True)
    x.copy_(x0)
    solver.params = p
    solver.run(k, x, b1)
    torch.cuda.synchronize()
    t_stage, n_timed = solver.kernel_times()
    solver.set_timing(False)
    fx = oracle_fixture("radial_128")
    err_b1 = rel_l2(b1, fx["b1"]) if fx is not None and "b1" in fx else None
    N = W * H * T
    peak, _ = load_peaks()
    stream = {"dual": 8 * N * (4 + 2 * 9), "primal": 8 * N * (1 + 3 * 4 + 9)}
    names = ["dual", "grid_fft", "interp_prox", "spread_ifft_crop", "primal"]
    kms = {n: float(t_stage[i]) for i, n in enumerate(names)}
    iters = synth.RADIAL_ITERS
    return {"workload": "radial golden-angle TGV2, 128x128, 40 frames, 12 coils, 256 readout samples x 21 spokes "
                        "per frame, KB width 3, osf 1.5, sector 8, %d iterations, H1 coil construction first" % iters,
            "coil_construction_ms": coil_ms, "recon_ms": ms, "pd_it_per_s": iters / (ms / 1000.0),
            "kernel_ms": kms,
            "stream_kernels_frac_of_hbm": {n: stream[n] / (kms[n] / 1000.0) / 1e9 / peak for n in stream},
            "rel_l2_vs_oracle": err_oracle, "coil_maps_rel_l2_vs_oracle": err_b1, "rel_l2_vs_phantom": err}


def run_tv128(av, torch, steps=5, cpu_iters=10):
    """The TV configuration: 128 x 128, 20 frames, 8 coils, central plus
    random lines at acceleration 8, 500 iterations with the reference's TV
    defaults (lambda from AdaptLambda), started from the time average.  Its
    working set (~55 MB) stays in L2 between launches."""
    from avionic_b200 import synth
    prob = synth.tv_ellipses_128_problem()
    T, C, H, W = prob["kdata"].shape
    kd, md, b1 = av.to_device(prob["kdata"]), av.to_device(prob["mask"]), av.to_device(prob["b1"])
    x0 = av.to_device(np.repeat(prob["u0"][None], T, axis=0))
    op = av.CartesianOperator(W, H, C, T, mask=md, centered=False)
    p = av.default_params(av.TV)
    p.maxIt = synth.TV_ELLIPSES_ITERS
    solver = av.Solver(av.TV, op, p)
    p = solver.params  # lambda adapted at creation; every run starts from these sigma, tau
    x = torch.empty_like(x0)
    for _ in range(3):
        x.copy_(x0)
        solver.params = p
        solver.run(kd, x, b1)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        x.copy_(x0)
        solver.params = p
        solver.run(kd, x, b1)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    err = vs_oracle("tv_ellipses_128", x)
    solver.set_timing(True)
    x.copy_(x0)
    solver.params = p
    solver.run(kd, x, b1)
    torch.cuda.synchronize()
    t_stage, _ = solver.kernel_times()
    solver.set_timing(False)
    names = ["dual", "ydft", "rows", "coladj", "primal"]
    kms = {n: float(t_stage[i]) for i, n in enumerate(names)}
    N = W * H * T
    peak, _ = load_peaks()
    dual_bytes = 8 * N * (1 + 2 * 3)
    iters = synth.TV_ELLIPSES_ITERS
    workers = os.cpu_count() or 1
    cpu_oracle_seconds("TV", prob, 1, workers, 10)
    dt = cpu_oracle_seconds("TV", prob, cpu_iters, workers, 10)
    fx = oracle_fixture("tv_ellipses_128")
    return {"workload": "Cartesian TV 128x128, 20 frames, 8 coils, 8 central + random lines at acceleration 8, "
                        "%d iterations (L2-resident working set)" % iters,
            "pd_it_per_s": iters / (ms / 1000.0), "recons_per_s": 1000.0 / ms, "recon_ms": ms,
            "rel_l2_vs_oracle": err, "kernel_ms": kms,
            "dual_roofline": {"achieved_gbs": dual_bytes / (kms["dual"] / 1000.0) / 1e9, "peak_gbs": peak,
                              "frac": dual_bytes / (kms["dual"] / 1000.0) / 1e9 / peak,
                              "algorithmic_bytes_per_launch": dual_bytes,
                              "note": "the fields stay in the 126 MB L2, so the fraction of HBM peak can exceed 1"},
            "cpu_baseline": {"pd_it_per_s": cpu_iters / dt, "cores": workers, "kind": "port",
                             "recons_per_s_extrapolated": cpu_iters / dt / iters,
                             "sample": "%d fixed-step TV iterations (k = 10..%d) of the float64 oracle" %
                                       (cpu_iters, 9 + cpu_iters),
                             "full_recon_s_fixture_host": float(fx["seconds"]) if fx is not None else None}}


def max_over_ranks(dist, value, device):
    """The job's time is its slowest rank's: the largest value over all ranks
    (the value itself without a process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, value, device):
    """The sum of value over all ranks (the value itself without a process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def shard_by_footprint(footprints, world):
    """Rank of every instance: the largest first, each to the rank with the
    least footprint so far (the lowest rank on ties).  Every rank computes the
    same assignment from the same list, so no exchange is needed."""
    load = [0.0] * world
    owner = [0] * len(footprints)
    for i in sorted(range(len(footprints)), key=lambda k: (-footprints[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += footprints[i]
    return owner


def job_rate(world, steps, ms):
    """PD iterations per second of the whole job: each of `world` ranks runs
    `steps` reconstructions of ITERS iterations; `ms` is the slowest rank's time."""
    return world * steps * ITERS / (ms / 1000.0)


def instance_seed(rank):
    """Each rank reconstructs its own instance (weak scaling, no collective on
    the data path)."""
    return 1 + rank


def run_reference(args, rank, world):
    """The reference arm: the oracle port on the host cores, rank 0 only.
    Warm-up runs the ten step-rule iterations of the start (k < 10) once;
    each timed step runs --ref-iters iterations with the counter at k >= 10,
    the fixed-step iterations that make up 971 of the 1000 (the 29 step-rule
    ones cost the CPU about 1.6 times as much, so this sample favours the CPU
    arm by about 2 %)."""
    if rank != 0:
        return
    workers = os.cpu_count() or 1
    prob = make_problem(1)
    n = max(1, args.ref_iters)
    warm = cpu_oracle_seconds("ICTGV2", prob, 10, workers, 0) if args.warmup > 0 else 0.0
    times = [cpu_oracle_seconds("ICTGV2", prob, n, workers, 10) for _ in range(args.steps)]
    value = float(n * len(times) / np.sum(times))
    sample = ("%d steps x %d fixed-step ICTGV2 iterations (counter k = 10..%d) of the float64 oracle on the "
              "benchmark problem, after the 10 step-rule iterations as warm-up (%.1f s); scipy.fft workers=%d, "
              "numpy elementwise work on one thread" % (args.steps, n, 9 + n, warm, workers))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": CONFIG,
        "sample": sample,
        "recons_per_s": value / ITERS,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port", "sample": sample},
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
    ap.add_argument("--cpu-iters", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dft", default="split", choices=["split", "fp32"],
                    help="arithmetic of the y-transforms: split-BF16x3 tensor cores or fp32 CUDA cores")
    ap.add_argument("--parts", default="headline,tv128,radial,batched,serving",
                    help="comma list: headline (the 192x192x30 cine ICTGV2 line), tv128, radial, batched, serving "
                         "(added to the line at N=1; batched at every N)")
    ap.add_argument("--batch-workers", type=int, default=8,
                    help="requests the engine advances together in the batched form")
    ap.add_argument("--serve-workers", type=int, default=4,
                    help="requests the engine advances together in the served form (fewer finish in arrival order "
                         "sooner; more overlap small requests)")
    ap.add_argument("--batch-size", type=int, default=64)
    ap.add_argument("--serve-requests", type=int, default=48,
                    help="requests per rate (bounded sample of the 2000-request stream)")
    ap.add_argument("--serve-rates", default="20,200",
                    help="comma list of arrival rates in requests/s (the configuration sweeps 20-200)")
    ap.add_argument("--serve-stop-gap", type=float, default=1e-4,
                    help="normalised primal-dual gap (gap / pixels) at which a served request stops")
    args = ap.parse_args()
    parts = set(args.parts.split(","))

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
    extra = {}
    if "batched" in parts:
        extra["batched"] = run_batched(av, torch, args.batch_workers, args.batch_size, rank=rank, world=world,
                                       dist=dist)
    if world == 1 and "tv128" in parts:
        extra["tv_ellipses_128"] = run_tv128(av, torch)
    if world == 1 and "radial" in parts:
        extra["radial"] = run_radial(av, torch)
    if world == 1 and "serving" in parts:
        extra["serving"] = run_serving(av, torch, args.serve_workers, args.serve_requests,
                                       [float(r) for r in args.serve_rates.split(",")],
                                       rel_gap=args.serve_stop_gap)
    if "headline" not in parts:
        if dist is not None:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps(extra), flush=True)
        return

    def barrier():
        if dist is not None:
            dist.barrier()

    prob = make_problem(instance_seed(rank))
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
    p0 = solver.params  # a run adapts sigma and tau; every reconstruction starts from the configured ones
    R = int(np.count_nonzero(prob["mask"].any(axis=2)))

    # warm-up: kernels, buffers, the autotuned launch shapes and the CUDA graphs
    # of the iteration shapes are set up here
    solver.set_timing(False)
    for _ in range(args.warmup):
        x.copy_(x0)
        solver.params = p0
        solver.run(kd, x, b1)
    torch.cuda.synchronize()
    tuning = solver.tuning()
    row_schedule = solver.kspace_schedule()

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
        solver.params = p0
        solver.run(kd, x, b1)
        s1 = torch.cuda.Event(enable_timing=True)
        s1.record()
        lat.append((s0, s1))
        launches += solver.stats().kernel_launches + 3  # + row gather and two set-up reductions
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(dist, e0.elapsed_time(e1), "cuda")
    step_ms = [a.elapsed_time(b) for a, b in lat]
    value = job_rate(world, args.steps, ms)
    # accuracy of the timed reconstruction against the float64 oracle's
    # fixture of the same problem (rank 0's instance, seed 1)
    assert torch.isfinite(torch.view_as_real(x)).all().item()
    err_oracle = vs_oracle("cine_192", x) if instance_seed(rank) == 1 else None

    # the other arithmetic of the y-transforms, same problem and schedule (reported beside the headline)
    other = None
    if args.dft == "split" and op.dft_mode == av.DFT_SPLIT_BF16X3:
        op.dft_mode = av.DFT_FP32
        for _ in range(2):
            x.copy_(x0)
            solver.params = p0
            solver.run(kd, x, b1)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        for _ in range(args.steps):
            x.copy_(x0)
            solver.params = p0
            solver.run(kd, x, b1)
        g1.record()
        torch.cuda.synchronize()
        x_fp32 = x.clone()
        other = {"dft": "fp32 CUDA cores", "value": job_rate(world, args.steps, max_over_ranks(dist, g0.elapsed_time(g1), "cuda")),
                 "unit": UNIT}
        op.dft_mode = av.DFT_SPLIT_BF16X3
        x.copy_(x0)
        solver.params = p0
        solver.run(kd, x, b1)
        torch.cuda.synchronize()
        other["rel_l2_split_vs_fp32"] = float(torch.linalg.vector_norm(x - x_fp32) /
                                              torch.linalg.vector_norm(x_fp32))
        if instance_seed(rank) == 1:
            other["rel_l2_vs_oracle"] = vs_oracle("cine_192", x_fp32)

    # per-stage durations: one more reconstruction with CUDA events between the
    # stages of every iteration (kernels launched directly, not from graphs)
    solver.set_timing(True)
    x.copy_(x0)
    solver.params = p0
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
            "iteration_frac": ab["iteration"] / (iter_ms / 1000.0) / 1e9 / peak,
            "iteration_bytes_dense_layout": ab["iteration_dense_layout"]}
    if args.dft == "split":
        roof["tensor_kernels"] = tensor_roofline(prob["mask"], W, H, T, C, kmean[1], kmean[3])

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
    ems = max_over_ranks(dist, f0.elapsed_time(f1), "cuda")
    e2e_value = job_rate(world, args.steps, ems)
    av.lib.avx_reconstruct_host_release()
    h2d = pk.numel() * 8 + pm.numel() * 4 + pb.numel() * 8 + pu.numel() * 8
    d2h = px.numel() * 8

    e2e_err = vs_oracle("cine_192", px) if instance_seed(rank) == 1 else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        workers = os.cpu_count() or 1
        cpu_oracle_seconds("ICTGV2", prob, 1, workers, 10)  # imports and first-touch
        dt = cpu_oracle_seconds("ICTGV2", prob, args.cpu_iters, workers, 10)
        cpu = {"value": args.cpu_iters / dt, "unit": UNIT, "cores": workers, "kind": "port",
               "sample": "%d fixed-step ICTGV2 iterations (counter k = 10..%d) of the float64 oracle on this problem "
                         "(%.1f s; scipy.fft workers=%d, numpy elementwise work on one thread)"
                         % (args.cpu_iters, 9 + args.cpu_iters, dt, workers)}

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
        "config": CONFIG,
        "recons_per_s": value / ITERS,
        "rel_l2_vs_oracle": err_oracle,
        "details": {"parallelism": "one independent reconstruction per GPU", "graphs": True,
                    "tuning": {"primal_tile": tuning[2], "dual_block_threads": tuning[3],
                               "dual_pixels_per_thread": 2 if tuning[1] >= 3 else 1,
                               "row_fft_rows_per_pass": row_schedule[0],
                               "row_fft_plan": "run-time" if row_schedule[1] else "compile-time"},
                    "dft": args.dft, "other_dft_form": other,
                    "recon_latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                                         "p99": float(np.percentile(step_ms, 99))}},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "rel_l2_vs_oracle": e2e_err},
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": int(launches * world),
    }
    line.update(extra)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
