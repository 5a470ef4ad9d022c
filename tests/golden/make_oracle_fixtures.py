"""Generates the float64-oracle fixtures of the benchmark problems at full size.

Each fixture is the final image of the oracle (oracle/solvers.py, a float64
restatement of the reference's TV / TGV2 / ICTGV2 loops) on a seeded
synthetic problem that ``avionic_b200.synth`` rebuilds bit for bit on any
machine (numpy only), stored as complex64 with the run's parameters:

  tv_ellipses_128  TV, 128 x 128, 20 frames, 8 coils, central plus random
                lines at acceleration 8, 500 iterations, the reference's TV
                defaults with lambda from AdaptLambda (tv.cpp:99-200)
  cine_192      ICTGV2, 192 x 192, 30 frames, 16 coils, variable-density lines
                at acceleration 12, 1000 iterations, the parameters of the
                reference's default configuration file's [ictgv2] section
                (ictgv2.cpp:294-492)
  batched_<i>   TGV2, instance i of the 64-instance batched set
                (synth.batched_specs(3, 64)), 800 iterations, the reference's
                TGV2 defaults with lambda from AdaptLambda (tgv2.cpp:180-338)
  radial_128    H1 coil-sensitivity construction from the radial data
                (coil_construction.cpp:447-556, main.cpp:210-248), then TGV2
                with the gridding operator, 500 iterations

Usage: python tests/golden/make_oracle_fixtures.py <case> [<case> ...]
       (cases: tv_ellipses_128, cine_192, batched, radial_128, or batched_<i>;
       ``manifest`` writes oracle/manifest.json, the SHA-256 of every case's
       regenerated inputs, which the tests check before comparing images).  A full run of
cine_192 takes about an hour on one core.  The GPU tests
(tests/test_oracle_fixtures.py) and bench.py compare the CUDA path with these
files.
"""

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from avionic_b200 import synth  # noqa: E402  (numpy generators; no library load)
from oracle import solvers as so  # noqa: E402
from oracle.cartesian import CartesianOperator  # noqa: E402

OUT = os.path.join(HERE, "oracle")


def _save(name, x, meta):
    os.makedirs(OUT, exist_ok=True)
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, x=np.asarray(x, dtype=np.complex64), **{k: np.asarray(v) for k, v in meta.items()})
    print("wrote %s (%.1f MB)" % (path, os.path.getsize(path) / 1e6), flush=True)


def tv_ellipses_128():
    prob = synth.tv_ellipses_128_problem()
    T, C, H, W = prob["kdata"].shape
    op = CartesianOperator(W, H, C, T, mask=prob["mask"], centered=False)
    p = so.init_params("TV")
    p.lam = op.adapt_lambda(*p.adapt_kd)
    p.maxIt = synth.TV_ELLIPSES_ITERS
    x0 = np.repeat(prob["u0"][None].astype(complex), T, axis=0)
    tr = {}
    t0 = time.time()
    x = so.tv(prob["kdata"].astype(complex), x0, prob["b1"].astype(complex), op, p, tr)
    sig, tau = tr["steps"][-1]
    _save("tv_ellipses_128", x, dict(method="TV", iterations=tr["iterations"], sigma=sig, tau=tau, lam=p.lam,
                                     seconds=time.time() - t0))


def cine_192():
    prob = synth.cine_192_problem()
    T, C, H, W = prob["kdata"].shape
    op = CartesianOperator(W, H, C, T, mask=prob["mask"], centered=False)
    p = so.init_params("ICTGV2")
    for k, v in synth.CINE_192_PARAMS.items():
        setattr(p, "lam" if k == "lambda" else k, v)
    x0 = np.repeat(prob["u0"][None].astype(complex), T, axis=0)
    tr = {}
    t0 = time.time()
    x = so.ictgv2(prob["kdata"].astype(complex), x0, prob["b1"].astype(complex), op, p, tr)
    sig, tau = tr["steps"][-1]
    _save("cine_192", x, dict(method="ICTGV2", iterations=tr["iterations"], sigma=sig, tau=tau,
                              seconds=time.time() - t0))


def batched(i):
    spec = synth.batched_specs(3, 64)[i]
    prob = synth.cine_instance(spec)
    T, C, H, W = prob["kdata"].shape
    op = CartesianOperator(W, H, C, T, mask=prob["mask"], centered=False)
    p = so.init_params("TGV2")
    p.lam = op.adapt_lambda(*p.adapt_kd)
    p.maxIt = synth.BATCHED_ITERS
    x0 = np.repeat(prob["u0"][None].astype(complex), T, axis=0)
    tr = {}
    t0 = time.time()
    x = so.tgv2(prob["kdata"].astype(complex), x0, prob["b1"].astype(complex), op, p, tr)
    sig, tau = tr["steps"][-1]
    _save("batched_%d" % i, x, dict(method="TGV2", index=i, W=W, H=H, T=T, C=C, iterations=tr["iterations"],
                                    sigma=sig, tau=tau, lam=p.lam, seconds=time.time() - t0))


def radial_128():
    from oracle import coils as oc
    from oracle import radial as rd
    prob = synth.radial_128(2)
    k, traj, dens = prob["kdata"], prob["traj"], prob["dens"]
    T, C, S = k.shape
    H, W = prob["truth"].shape[1:]
    kd = k.astype(complex)
    t0 = time.time()
    u0, crec = oc.time_averaged_radial(kd, traj.astype(float), dens.astype(float), W, H)
    u, b1 = oc.estimate_from(u0, crec)
    t1 = time.time()
    x0 = np.repeat((u[C - 1] / T)[None], T, axis=0)  # main.cpp:636-640
    op = rd.RadialOperator(W, H, C, T, traj.astype(float), dens.astype(float), 3.0, 8.0, 1.5)
    p = so.init_params("TGV2")
    p.lam = op.adapt_lambda(p.adapt_kd[0], p.adapt_kd[1], prob["spokes"])
    p.maxIt = synth.RADIAL_ITERS
    tr = {}
    x = so.tgv2(kd, x0, b1, op, p, tr)
    sig, tau = tr["steps"][-1]
    _save("radial_128", x, dict(method="TGV2", iterations=tr["iterations"], sigma=sig, tau=tau, lam=p.lam,
                                b1=b1.astype(np.complex64), coil_seconds=t1 - t0, seconds=time.time() - t0))


def case_inputs(case):
    """The arrays a case's reconstruction starts from (the hashed inputs)."""
    if case == "tv_ellipses_128":
        p = synth.tv_ellipses_128_problem()
        return [p["kdata"], p["mask"], p["b1"], p["u0"]]
    if case == "cine_192":
        p = synth.cine_192_problem()
        return [p["kdata"], p["mask"], p["b1"], p["u0"]]
    if case == "radial_128":
        p = synth.radial_128(2)
        return [p["kdata"], p["traj"], p["dens"]]
    if case.startswith("batched_"):
        p = synth.cine_instance(synth.batched_specs(3, 64)[int(case.split("_")[1])])
        return [p["kdata"], p["mask"], p["b1"], p["u0"]]
    raise KeyError(case)


def inputs_sha256(case):
    import hashlib
    h = hashlib.sha256()
    for a in case_inputs(case):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def all_cases():
    return ["tv_ellipses_128", "cine_192", "radial_128"] + ["batched_%d" % i for i in synth.oracle_batched_indices()]


def manifest():
    import json
    out = {c: inputs_sha256(c) for c in all_cases()}
    os.makedirs(OUT, exist_ok=True)
    with open(os.path.join(OUT, "manifest.json"), "w") as f:
        json.dump({"inputs_sha256": out}, f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote manifest of %d cases" % len(out))


def main(argv):
    for case in argv or ["tv_ellipses_128", "cine_192", "batched", "radial_128"]:
        if case == "manifest":
            manifest()
        elif case == "tv_ellipses_128":
            tv_ellipses_128()
        elif case == "cine_192":
            cine_192()
        elif case == "radial_128":
            radial_128()
        elif case == "batched":
            for i in synth.oracle_batched_indices():
                batched(i)
        elif case.startswith("batched_"):
            batched(int(case.split("_")[1]))
        else:
            raise SystemExit("unknown case %r" % case)


if __name__ == "__main__":
    main(sys.argv[1:])
