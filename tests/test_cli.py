"""The avionic executable: flags, configuration, .bin formats, exports.

CPU tests cover the paths that end before any device work (usage, invalid
method, unknown configuration keys, dimension mismatch, truncated files);
the GPU test runs a full reconstruction through the executable and compares
the written image with the float64 oracle.
"""

import os
import struct
import subprocess

import numpy as np
import pytest

from oracle import binfmt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "avionic_b200", "avionic")

needs_exe = pytest.mark.skipif(not os.path.exists(EXE), reason="avionic executable not built")


def run(args, **kw):
    return subprocess.run([EXE] + args, capture_output=True, text=True, timeout=600, **kw)


def write_problem(tmp, prob, with_u0=True):
    T, C, H, W = prob["kdata"].shape
    paths = {k: str(tmp / (k + ".bin")) for k in ("kdata", "mask", "b1", "u0")}
    binfmt.write_bin(paths["kdata"], prob["kdata"].astype(np.complex128))
    binfmt.write_bin(paths["mask"], prob["mask"].astype(np.float64))
    binfmt.write_bin(paths["b1"], prob["b1"].astype(np.complex128))
    if with_u0:
        binfmt.write_bin(paths["u0"], np.zeros((H, W), np.complex128))
    return paths, "%d:%d:1:%d:%d:1:%d:%d" % (W, H, W, H, C, T)


@needs_exe
def test_usage_and_errors(tmp_path):
    r = run(["-h"])
    assert r.returncode == 255 and "Usage: avionic" in r.stdout
    assert "--opnormSteps" in r.stdout
    r = run([])
    assert r.returncode == 255
    rng = np.random.default_rng(0)
    prob = {"kdata": (rng.standard_normal((2, 2, 4, 5)) + 0j).astype(np.complex64),
            "mask": np.ones((2, 4, 5), np.float32), "b1": np.ones((2, 4, 5), np.complex64)}
    paths, dims = write_problem(tmp_path, prob)
    out = str(tmp_path / "x.bin")
    r = run(["-m", "NOPE", "-d", dims, "-s", paths["b1"], paths["kdata"], paths["mask"], out])
    assert r.returncode == 255 and "invalid method" in r.stderr
    r = run(["-m", "TGV2_3D", "-d", dims, "-s", paths["b1"], paths["kdata"], paths["mask"], out])
    assert r.returncode == 255 and "not provided" in r.stderr
    r = run(["--opnormSteps", "many", "-m", "TV", "-d", dims, "-s", paths["b1"], paths["kdata"], paths["mask"], out])
    assert r.returncode == 255 and "invalid value 'many' for option 'opnormSteps'" in r.stderr
    cfg = tmp_path / "bad.cfg"
    cfg.write_text("[tv]\nlambdaa = 3\n")
    r = run(["-p", str(cfg), "-m", "TV", "-d", dims, "-s", paths["b1"], paths["kdata"], paths["mask"], out])
    assert r.returncode == 255 and "unrecognised option 'tv.lambdaa'" in r.stderr
    bad_dims = dims.replace(":2:2", ":3:2")
    r = run(["-m", "TV", "-d", bad_dims, "-s", paths["b1"], paths["kdata"], paths["mask"], out])
    assert r.returncode == 255 and "dims require" in r.stderr
    trunc = tmp_path / "trunc.bin"
    with open(paths["kdata"], "rb") as f:
        trunc.write_bytes(f.read()[:40])
    r = run(["-m", "TV", "-d", dims, "-s", paths["b1"], str(trunc), paths["mask"], out])
    assert r.returncode == 255 and "truncated" in r.stderr


@needs_exe
def test_method_sections_declare_their_own_keys(tmp_path):
    """[tvtemp] declares dt, sigma, tau, sigmaTauRatio and lambda only; [ictv]
    has no alpha0 (options_parser.cpp:204-257)."""
    rng = np.random.default_rng(1)
    prob = {"kdata": (rng.standard_normal((2, 2, 4, 5)) + 0j).astype(np.complex64),
            "mask": np.ones((2, 4, 5), np.float32), "b1": np.ones((2, 4, 5), np.complex64)}
    paths, dims = write_problem(tmp_path, prob)
    out = str(tmp_path / "x.bin")
    for method, section, key in (("TVTEMP", "tvtemp", "dx"), ("TVTEMP", "tvtemp", "timeSpaceWeight"),
                                 ("ICTV", "ictv", "alpha0")):
        cfg = tmp_path / ("%s.cfg" % key)
        cfg.write_text("[%s]\n%s = 1.0\n" % (section, key))
        r = run(["-p", str(cfg), "-m", method, "-d", dims, "-s", paths["b1"], paths["kdata"], paths["mask"], out])
        assert r.returncode == 255 and "unrecognised option '%s.%s'" % (section, key) in r.stderr


def test_bin_format_roundtrip(tmp_path):
    """The .bin layout of matlab/writebin_vector.m:35-44."""
    v = np.arange(5) + 1j * np.arange(5, 10)
    p = tmp_path / "v.bin"
    binfmt.write_bin(str(p), v)
    raw = p.read_bytes()
    assert raw[0] == 1 and struct.unpack("<I", raw[1:5])[0] == 5 and len(raw) == 5 + 80
    assert np.array_equal(binfmt.read_bin(str(p)), v)
    binfmt.write_bin(str(p), np.arange(3.0))
    assert p.read_bytes()[0] == 0 and len(p.read_bytes()) == 5 + 24


@needs_exe
@pytest.mark.gpu
@pytest.mark.parametrize("method", ["TV", "TVTEMP", "TGV2", "ICTV", "ICTGV2"])
def test_cli_reconstruction_matches_oracle(tmp_path, method):
    from avionic_b200 import synth
    from oracle import solvers as so
    from oracle.cartesian import CartesianOperator
    prob = synth.small(21)
    T, C, H, W = prob["kdata"].shape
    paths, dims = write_problem(tmp_path, prob)
    out = str(tmp_path / "recon.bin")
    cfg = tmp_path / "run.cfg"
    common = "lambda = 2.5\nsigma = 0.3333\ntau = 0.3333\nsigmaTauRatio = 1.0\n"
    cfg.write_text("maxIt = 80\n[tv]\n" + common + "timeSpaceWeight = 3.0\n[tvtemp]\n" + common +
                   "dt = 1.0\n[tgv2]\n" + common +
                   "timeSpaceWeight = 1.4\nalpha0 = 1.41421356\nalpha1 = 1.0\n[ictv]\n" + common +
                   "timeSpaceWeight = 4.0\ntimeSpaceWeight2 = 0.5\nalpha = 0.5\nalpha1 = 1.0\n[ictgv2]\n" +
                   common + "timeSpaceWeight = 4.0\ntimeSpaceWeight2 = 0.5\nalpha = 0.5\nalpha0 = 1.41421356\n"
                   "alpha1 = 1.0\n")
    r = run(["-m", method, "-p", str(cfg), "-e", "-g", "10", "-d", dims, "-s", paths["b1"], "-u", paths["u0"],
             paths["kdata"], paths["mask"], out])
    assert r.returncode == 0, r.stderr + r.stdout
    x = binfmt.read_bin(out).reshape(T, H, W)

    op = CartesianOperator(W, H, C, T, mask=prob["mask"], centered=False)
    p = so.init_params(method)
    p.maxIt, p.lam, p.sigma, p.tau = 80, 2.5, 0.3333, 0.3333
    p.timeSpaceWeight = {"TV": 3.0, "TVTEMP": 5.0, "TGV2": 1.4, "ICTV": 4.0, "ICTGV2": 4.0}[method]
    p.timeSpaceWeight2, p.alpha, p.alpha1 = 0.5, 0.5, 1.0
    p.alpha0 = 1.41421356
    p.debug, p.debugstep = True, 10
    tr = {}
    xo = so.run(method, prob["kdata"].astype(complex), np.zeros((T, H, W), complex), prob["b1"].astype(complex),
                op, p, tr)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-4
    gaps = binfmt.read_bin(str(tmp_path / "PDGap"))
    # the gap is a difference of nearly equal large terms: FP32 iterates give
    # a relative error well above the image's
    assert np.allclose(gaps.real, tr["PDGap"], rtol=1e-3)
    if method == "ICTGV2":
        assert binfmt.read_bin(str(tmp_path / "x3_component")).size == T * H * W
        assert binfmt.read_bin(str(tmp_path / "ICTGVnorm")).size == len(tr["ICTGVnorm"])
    if method == "ICTV":
        assert binfmt.read_bin(str(tmp_path / "x3_component")).size == T * H * W
        assert np.allclose(binfmt.read_bin(str(tmp_path / "ictvnorm")).real, tr["ictvnorm"], rtol=1e-3)


@needs_exe
@pytest.mark.gpu
def test_cli_opnorm_steps(tmp_path):
    """--opnormSteps 10: the initial steps come from the power-iteration
    estimate l of ||K||^2 (sigma = tau = 1/sqrt(l) at sigmaTauRatio 1); the
    estimate lies below the largest eigenvalue of K^H K (the oracle's
    estimate after 300 iterations, from another start) and the image equals
    the oracle's reconstruction from the printed steps."""
    import re
    from avionic_b200 import synth
    from oracle import opnorm as on
    from oracle import solvers as so
    from oracle.cartesian import CartesianOperator
    prob = synth.small(22)
    T, C, H, W = prob["kdata"].shape
    paths, dims = write_problem(tmp_path, prob)
    out = str(tmp_path / "recon.bin")
    cfg = tmp_path / "run.cfg"
    cfg.write_text("maxIt = 100\n[tgv2]\nlambda = 2.5\nsigmaTauRatio = 1.0\ntimeSpaceWeight = 1.4\n"
                   "alpha0 = 1.41421356\nalpha1 = 1.0\n")
    r = run(["-m", "TGV2", "-p", str(cfg), "--opnormSteps", "10", "-d", dims, "-s", paths["b1"], "-u", paths["u0"],
             paths["kdata"], paths["mask"], out])
    assert r.returncode == 0, r.stderr + r.stdout
    m = re.search(r"Operator norm estimate \|\|K\|\|\^2: (\S+) -> sigma (\S+), tau (\S+)", r.stdout)
    assert m, r.stdout
    l, sig, tau = (float(v) for v in m.groups())
    assert abs(sig * tau * l - 1.0) < 1e-4 and abs(sig / tau - 1.0) < 1e-6
    op = CartesianOperator(W, H, C, T, mask=prob["mask"], centered=False)
    p = so.init_params("TGV2")
    p.maxIt, p.lam, p.timeSpaceWeight, p.alpha0, p.alpha1 = 100, 2.5, 1.4, 1.41421356, 1.0
    rng = np.random.default_rng(0)
    top = on.getopnorm(on.method_normal("TGV2", op, prob["b1"].astype(complex), p),
                       [rng.standard_normal((T, H, W)) + 1j * rng.standard_normal((T, H, W))] +
                       [np.zeros((T, H, W), complex)] * 3, 300)
    assert 0.5 * top < l <= top * (1 + 1e-4)
    p.sigma, p.tau = np.float32(sig), np.float32(tau)
    xo = so.run("TGV2", prob["kdata"].astype(complex), np.zeros((T, H, W), complex), prob["b1"].astype(complex),
                op, p)
    x = binfmt.read_bin(out).reshape(T, H, W)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-4


@needs_exe
@pytest.mark.gpu
def test_cli_normalisation(tmp_path):
    """-o: the data are scaled by 255 / median of the centred time average's
    top values before the run (main.cpp:573-579); datanorm_factor.bin holds
    the factor (main.cpp:793-796) and the image is the reconstruction of the
    scaled data."""
    from avionic_b200 import synth
    from oracle import solvers as so
    from oracle.cartesian import CartesianOperator
    from oracle.normalize import normalization_factor
    prob = synth.small(23)
    T, C, H, W = prob["kdata"].shape
    paths, dims = write_problem(tmp_path, prob)
    out = str(tmp_path / "recon.bin")
    cfg = tmp_path / "run.cfg"
    cfg.write_text("maxIt = 60\n[tv]\nlambda = 2.5\nsigma = 0.3333\ntau = 0.3333\ntimeSpaceWeight = 3.0\n")
    r = run(["-m", "TV", "-o", "-p", str(cfg), "-g", "0", "-d", dims, "-s", paths["b1"], "-u", paths["u0"],
             paths["kdata"], paths["mask"], out])
    assert r.returncode == 0, r.stderr + r.stdout
    f = binfmt.read_bin(str(tmp_path / "datanorm_factor.bin"))
    k64 = prob["kdata"].astype(complex) * prob["mask"][:, None]
    fo = normalization_factor(k64, prob["mask"])
    assert f.size == 1 and abs(f[0] - fo) / fo < 1e-5
    x = binfmt.read_bin(out).reshape(T, H, W)
    op = CartesianOperator(W, H, C, T, mask=prob["mask"], centered=False)
    p = so.init_params("TV")
    p.maxIt, p.lam, p.sigma, p.tau, p.timeSpaceWeight = 60, 2.5, 0.3333, 0.3333, 3.0
    ks = (prob["kdata"] * np.float32(f[0].real)).astype(complex) * prob["mask"][:, None]
    xo = so.run("TV", ks, np.zeros((T, H, W), complex), prob["b1"].astype(complex), op, p, {})
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-4


@needs_exe
@pytest.mark.gpu
def test_cli_radial_with_coil_construction(tmp_path):
    """-n radial data without -s: coil construction, u0/b1 exports, then TGV2."""
    from oracle import coils as co
    from oracle import radial as rd
    from oracle import solvers as so
    from tests.test_radial import _problem
    pr = _problem(13, W=20, H=20, C=3, T=3, nfe=40, spf=7)
    T, C, S = pr["k"].shape
    W, H = pr["W"], pr["H"]
    raw = pr["k"] / np.sqrt(pr["dens"])[:, None, :]  # the CLI weights by sqrt(w) itself
    paths = {"kdata": str(tmp_path / "k.bin"), "traj": str(tmp_path / "traj.bin"), "dens": str(tmp_path / "w.bin")}
    binfmt.write_bin(paths["kdata"], raw.astype(np.complex64).astype(np.complex128))
    binfmt.write_bin(paths["traj"], pr["traj"].astype(np.float32).astype(np.float64))
    binfmt.write_bin(paths["dens"], pr["dens"].astype(np.float32).astype(np.float64))
    cfg = tmp_path / "run.cfg"
    cfg.write_text("maxIt = 40\n[coil]\nuNrIt = 20\nb1NrIt = 30\nb1FinalNrIt = 40\n[tgv2]\nlambda = 4.0\n"
                   "sigma = 0.3333\ntau = 0.3333\ntimeSpaceWeight = 1.4\nalpha0 = 1.41421356\nalpha1 = 1.0\n"
                   "[gpunufft]\nkernelWidth = 3\nsectorWidth = 8\nosf = 1.5\n")
    out = str(tmp_path / "recon.bin")
    dims = "%d:%d:0:%d:%d:0:%d:%d" % (W, H, pr["nfe"], pr["spf"], C, T)
    r = run(["-n", "-m", "TGV2", "-p", str(cfg), "-g", "0", "-w", paths["dens"], "-d", dims, paths["kdata"],
             paths["traj"], out])
    assert r.returncode == 0, r.stderr + r.stdout
    b1 = binfmt.read_bin(str(tmp_path / "b1_reconstructed.bin")).reshape(C, H, W)
    u0 = binfmt.read_bin(str(tmp_path / "u0_reconstructed.bin")).reshape(H, W)
    x = binfmt.read_bin(out).reshape(T, H, W)
    # oracle: same pipeline
    k32 = (raw.astype(np.complex64) * np.sqrt(pr["dens"].astype(np.float32))[:, None, :]).astype(complex)
    tr, de = pr["traj"].astype(np.float32).astype(float), pr["dens"].astype(np.float32).astype(float)
    p = co.default_params()
    p["uNrIt"], p["b1NrIt"], p["b1FinalNrIt"] = 20, 30, 40
    ua, crec = co.time_averaged_radial(k32, tr, de, W, H)
    uo, bo = co.estimate_from(ua, crec, p)
    assert np.linalg.norm(b1 - bo) / np.linalg.norm(bo) < 1e-4
    u0o = uo[C - 1] / T
    assert np.linalg.norm(u0 - u0o) / np.linalg.norm(u0o) < 1e-4
    op = rd.RadialOperator(W, H, C, T, tr, de, 3.0, 8.0, 1.5)
    q = so.init_params("TGV2")
    q.maxIt, q.lam, q.sigma, q.tau, q.timeSpaceWeight, q.alpha0 = 40, 4.0, 0.3333, 0.3333, 1.4, 1.41421356
    xo = so.tgv2(k32, np.repeat(u0.astype(np.complex64).astype(complex)[None], T, axis=0),
                 b1.astype(np.complex64).astype(complex), op, q)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-4
