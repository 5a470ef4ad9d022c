"""ctypes binding of the AVIONIC B200 reconstruction core (libavionic_core.so).

The product is ``libavionic_core.so`` (CUDA, sm_100a) behind the C ABI in
``include/avionic.h``.  This module binds that ABI with ctypes and mirrors the
reference's interface for the reconstruction path (``CartesianOperator``,
``TV``/``TGV2``/``ICTGV2`` solvers, ``utils`` stencils), taking device buffers
as torch CUDA tensors.  There is no CPU fallback: importing this module (or
touching any of its names through the package) fails loudly when the library
is missing, and every call raises on a non-zero status.
"""

import ctypes
import os

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libavionic_core.so")

TV, TVTEMP, TGV2, TGV2_3D, ICTV, ICTGV2 = 0, 1, 2, 3, 4, 5
METHODS = {"TV": TV, "TVTEMP": TVTEMP, "TGV2": TGV2, "ICTV": ICTV, "ICTGV2": ICTGV2}
P_OF = {TV: 1, TGV2: 4, ICTGV2: 8}
D_OF = {TV: 3, TGV2: 9, ICTGV2: 18}


class AvionicError(RuntimeError):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libavionic_core.so is not built (expected at %s); run "
            "`python -c 'import __graft_entry__ as g; g.build()'` or `make -C avionic_b200/csrc`" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    _abi.declare(lib)
    return lib


lib = _load()


def check(status):
    if status != 0:
        msg = lib.avx_last_error().decode(errors="replace")
        raise AvionicError("avionic status %d: %s" % (status, msg))


PDParams = _abi.PDParams
RunStats = _abi.RunStats


def default_params(method):
    p = PDParams()
    check(lib.avx_default_params(method, ctypes.byref(p)))
    return p


# ---------------------------------------------------------------------------
# device-buffer helpers (torch is only the allocator here)
# ---------------------------------------------------------------------------

def _torch():
    import torch
    return torch


def _cptr(t):
    """ctypes void pointer of a contiguous CUDA tensor."""
    if not t.is_cuda:
        raise AvionicError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise AvionicError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def _ptr_array(tensors):
    arr = (ctypes.c_void_p * len(tensors))()
    for i, t in enumerate(tensors):
        arr[i] = _cptr(t).value
    return arr


def to_device(a, dtype=None):
    """numpy array -> contiguous CUDA tensor (complex64 / float32)."""
    import numpy as np
    torch = _torch()
    a = np.asarray(a)
    if dtype is None:
        dtype = np.complex64 if np.iscomplexobj(a) else np.float32
    return torch.from_numpy(np.ascontiguousarray(a.astype(dtype))).cuda()


DFT_FP32 = 0            # fp32 CUDA-core transform along y
DFT_SPLIT_BF16X3 = 1    # tcgen05 tensor-core transform, operands split into three bf16 pieces


class CartesianOperator:
    """``CartesianOperator`` (CUDA/src/cartesian_operator.cpp:3-168).

    ``mask`` is None (the reference's empty mask) or a float32 CUDA tensor of
    shape (T, H, W)."""

    def __init__(self, width, height, coils, frames, mask=None, centered=True):
        self.W, self.H, self.C, self.T = width, height, coils, frames
        self.handle = ctypes.c_void_p()
        mptr = _cptr(mask) if mask is not None else None
        check(lib.avx_cartesian_operator_create(width, height, coils, frames, mptr, int(centered),
                                                ctypes.byref(self.handle)))

    @property
    def dft_mode(self):
        """DFT_FP32 or DFT_SPLIT_BF16X3: arithmetic of the transform along y."""
        m = ctypes.c_int()
        check(lib.avx_operator_get_dft_mode(self.handle, ctypes.byref(m)))
        return m.value

    @dft_mode.setter
    def dft_mode(self, mode):
        check(lib.avx_operator_set_dft_mode(self.handle, int(mode)))

    def backward(self, x, b1, out=None):
        """image (T,H,W) -> k-space (T,C,H,W) (BackwardOperation)."""
        torch = _torch()
        if out is None:
            out = torch.empty((self.T, self.C, self.H, self.W), dtype=torch.complex64, device=x.device)
        check(lib.avx_operator_backward(self.handle, _cptr(x), _cptr(out), _cptr(b1)))
        return out

    def forward(self, k, b1, out=None):
        """k-space (T,C,H,W) -> image (T,H,W) (ForwardOperation; masks k in place)."""
        torch = _torch()
        if out is None:
            out = torch.empty((self.T, self.H, self.W), dtype=torch.complex64, device=k.device)
        check(lib.avx_operator_forward(self.handle, _cptr(k), _cptr(out), _cptr(b1)))
        return out

    def opnorm(self, x0, b1, iters=10, history=False):
        """getopnorm (matlab/getopnorm.m:1-17): power-iteration estimate of
        ||K||^2 for this encoding operator, started from the image x0
        (T,H,W).  With history=True also returns |y^H x| after each of the
        iters + 1 applications of K^H K."""
        v = ctypes.c_double()
        h = (ctypes.c_double * (iters + 1))()
        check(lib.avx_operator_opnorm(self.handle, _cptr(x0), _cptr(b1), int(iters), ctypes.byref(v), h))
        return (v.value, list(h)) if history else v.value

    def adapt_lambda(self, k, d):
        lam = ctypes.c_float()
        check(lib.avx_operator_adapt_lambda(self.handle, ctypes.c_float(k), ctypes.c_float(d), ctypes.byref(lam)))
        return lam.value

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and h.value and lib is not None:  # lib is None once the interpreter is shutting down
            lib.avx_operator_destroy(h)
            self.handle = ctypes.c_void_p()


class RadialOperator(CartesianOperator):
    """``NoncartesianOperator`` (CUDA/src/noncartesian_operator.cpp:3-195):
    radial gridding operator.  ``traj`` float32 CUDA tensor (T, 2, S) of
    cycles/pixel, ``dens`` float32 (T, S); k-space tensors are (T, C, S)."""

    def __init__(self, width, height, coils, frames, traj, dens, spokes_per_frame, kernel_width=3.0,
                 sector_width=8.0, osf=2.0):
        self.W, self.H, self.C, self.T = width, height, coils, frames
        self.S = traj.shape[-1]
        self.handle = ctypes.c_void_p()
        nfe = self.S // spokes_per_frame
        check(lib.avx_radial_operator_create(width, height, coils, frames, spokes_per_frame * frames, nfe,
                                             spokes_per_frame, _cptr(traj), _cptr(dens), kernel_width, sector_width,
                                             osf, ctypes.byref(self.handle)))

    def backward(self, x, b1, out=None):
        torch = _torch()
        if out is None:
            out = torch.empty((self.T, self.C, self.S), dtype=torch.complex64, device=x.device)
        check(lib.avx_operator_backward(self.handle, _cptr(x), _cptr(out), _cptr(b1)))
        return out


class Solver:
    """``TV`` / ``TGV2`` / ``ICTGV2`` (PDRecon, CUDA/include/pd_recon.h:88-185)."""

    def __init__(self, method, op, params=None):
        if isinstance(method, str):
            method = METHODS[method.upper()]
        self.method, self.op = method, op
        self.handle = ctypes.c_void_p()
        pp = ctypes.byref(params) if params is not None else None
        check(lib.avx_solver_create(method, op.W, op.H, op.C, op.T, pp, op.handle, ctypes.byref(self.handle)))

    @property
    def params(self):
        p = PDParams()
        check(lib.avx_solver_get_params(self.handle, ctypes.byref(p)))
        return p

    @params.setter
    def params(self, p):
        check(lib.avx_solver_set_params(self.handle, ctypes.byref(p)))

    def set_debug(self, debug, debugstep=1):
        check(lib.avx_solver_set_debug(self.handle, int(debug), int(debugstep)))

    def set_relative_stop(self, rel):
        """Also stop once the gap falls to rel times the run's first gap."""
        check(lib.avx_solver_set_relative_stop(self.handle, float(rel)))

    def set_verbose(self, verbose):
        check(lib.avx_solver_set_verbose(self.handle, int(verbose)))

    def set_tuning(self, autotune=True, primal_tile=0, dual_block=0):
        """Launch shapes of the dual and primal kernels (avx_solver_set_tuning)."""
        check(lib.avx_solver_set_tuning(self.handle, int(autotune), primal_tile, dual_block))

    def tuning(self):
        """(primal tile index, dual block index, primal tile name, dual threads) in use."""
        p, d, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        name = ctypes.c_char_p()
        check(lib.avx_solver_get_tuning(self.handle, ctypes.byref(p), ctypes.byref(d), ctypes.byref(name),
                                        ctypes.byref(t)))
        return p.value, d.value, name.value.decode(), t.value

    def set_kspace_schedule(self, rows_per_pass=16, runtime_plan=False):
        """Row-FFT schedule of the Cartesian row kernel (avx_solver_set_kspace_schedule)."""
        check(lib.avx_solver_set_kspace_schedule(self.handle, int(rows_per_pass), int(bool(runtime_plan))))

    def kspace_schedule(self):
        """(rows per pass, run-time radix plan) in use."""
        k, r = ctypes.c_int(), ctypes.c_int()
        check(lib.avx_solver_get_kspace_schedule(self.handle, ctypes.byref(k), ctypes.byref(r)))
        return k.value, bool(r.value)

    def set_stream(self, stream):
        check(lib.avx_solver_set_stream(self.handle, ctypes.c_void_p(stream)))

    def run(self, data, x, b1):
        """IterativeReconstruction(data, x, b1); x is updated in place."""
        check(lib.avx_solver_run(self.handle, _cptr(data), _cptr(x), _cptr(b1)))
        return x

    def adapt_step_size(self, diffs, b1):
        check(lib.avx_solver_adapt_step_size(self.handle, _ptr_array(diffs), _cptr(b1)))
        p = self.params
        return p.sigma, p.tau

    def compute_gap(self, xs, ys, z, data, b1):
        gs, gap = ctypes.c_double(), ctypes.c_double()
        check(lib.avx_solver_compute_gap(self.handle, _ptr_array(xs), _ptr_array(ys), _cptr(z), _cptr(data),
                                         _cptr(b1), ctypes.byref(gs), ctypes.byref(gap)))
        return gs.value, gap.value

    def opnorm(self, x0, b1, iters=10, set_steps=False, history=False):
        """Power-iteration estimate of ||K||^2 for the solver's whole
        primal-dual operator (regularisation part stacked on the encoding
        operator), started from the image x0 with the auxiliary components
        at zero.  set_steps=True makes the initial steps sigma = r/||K||,
        tau = 1/(r ||K||) (r = sigmaTauRatio)."""
        v = ctypes.c_double()
        h = (ctypes.c_double * (iters + 1))()
        check(lib.avx_solver_opnorm(self.handle, _cptr(x0), _cptr(b1), int(iters), int(bool(set_steps)),
                                    ctypes.byref(v), h))
        return (v.value, list(h)) if history else v.value

    def set_timing(self, on):
        check(lib.avx_solver_set_timing(self.handle, int(on)))

    def kernel_times(self):
        """Mean ms of the five stages (dual, forward transform, k-space rows,
        adjoint, primal) of the iterations of the last timed run."""
        arr = (ctypes.c_float * 5)()
        n = ctypes.c_uint()
        check(lib.avx_solver_kernel_times(self.handle, arr, ctypes.byref(n)))
        return list(arr), n.value

    def stats(self):
        s = RunStats()
        check(lib.avx_solver_get_stats(self.handle, ctypes.byref(s)))
        return s

    def export(self, output_dir=""):
        """ExportAdditionalResults: returns {name: complex numpy array}."""
        import numpy as np
        out = {}

        def cb(d, name, vals, n, user):
            arr = np.ctypeslib.as_array(ctypes.cast(vals, ctypes.POINTER(ctypes.c_float)), shape=(2 * n,))
            out[name.decode()] = (arr[0::2] + 1j * arr[1::2]).astype(np.complex64).copy()

        cbf = _abi.EXPORT_CB(cb)
        check(lib.avx_solver_export(self.handle, output_dir.encode(), cbf, None))
        return out

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and h.value and lib is not None:  # lib is None once the interpreter is shutting down
            lib.avx_solver_destroy(h)
            self.handle = ctypes.c_void_p()


# ---------------------------------------------------------------------------
# utils
# ---------------------------------------------------------------------------

def _empty_like_n(u, n):
    torch = _torch()
    return [torch.empty_like(u) for _ in range(n)]


def gradient(u, dx=1.0, dy=1.0, dt=1.0):
    T, H, W = u.shape
    g = _empty_like_n(u, 3)
    check(lib.avx_gradient(_cptr(u), _ptr_array(g), W, H, T, dx, dy, dt))
    return g


def divergence(y, dx=1.0, dy=1.0, dt=1.0):
    torch = _torch()
    T, H, W = y[0].shape
    out = torch.empty_like(y[0])
    check(lib.avx_divergence(_ptr_array(y), _cptr(out), W, H, T, dx, dy, dt))
    return out


def sym_gradient(v, dx=1.0, dy=1.0, dt=1.0):
    T, H, W = v[0].shape
    e = _empty_like_n(v[0], 6)
    check(lib.avx_sym_gradient(_ptr_array(v), _ptr_array(e), W, H, T, dx, dy, dt))
    return e


def sym_divergence(w, dx=1.0, dy=1.0, dt=1.0):
    T, H, W = w[0].shape
    d = _empty_like_n(w[0], 3)
    check(lib.avx_sym_divergence(_ptr_array(w), _ptr_array(d), W, H, T, dx, dy, dt))
    return d


def prox(y, scale):
    n = y[0].numel()
    fn = lib.avx_prox3 if len(y) == 3 else lib.avx_prox6
    check(fn(_ptr_array(y), n, ctypes.c_float(scale)))
    return y


def norm(g):
    torch = _torch()
    out = torch.empty(g[0].shape, dtype=torch.float32, device=g[0].device)
    fn = lib.avx_norm3 if len(g) == 3 else lib.avx_norm6
    check(fn(_ptr_array(g), _cptr(out), g[0].numel()))
    return out


def tv_norm(u, dx=1.0, dy=1.0, dt=1.0):
    T, H, W = u.shape
    v = ctypes.c_double()
    check(lib.avx_tv_norm(_cptr(u), W, H, T, dx, dy, dt, ctypes.byref(v)))
    return v.value


def tgv2_norm(x1, x2, alpha0, alpha1, dx=1.0, dy=1.0, dt=1.0):
    T, H, W = x1.shape
    v = ctypes.c_double()
    check(lib.avx_tgv2_norm(_cptr(x1), _ptr_array(x2), alpha0, alpha1, W, H, T, dx, dy, dt, ctypes.byref(v)))
    return v.value


def ictgv2_norm(x1, x2, x3, x4, alpha0, alpha1, alpha, w1, w2):
    T, H, W = x1.shape
    v = ctypes.c_double()
    a1 = (ctypes.c_float * 3)(*w1)
    a2 = (ctypes.c_float * 3)(*w2)
    check(lib.avx_ictgv2_norm(_cptr(x1), _ptr_array(x2), _cptr(x3), _ptr_array(x4), alpha0, alpha1, alpha, W, H, T,
                              a1, a2, ctypes.byref(v)))
    return v.value


def ellipke(m):
    return lib.avx_ellipke(ctypes.c_float(m))


def time_space_weights(tsw):
    ds, dt = ctypes.c_float(), ctypes.c_float()
    check(lib.avx_time_space_weights(ctypes.c_float(tsw), ctypes.byref(ds), ctypes.byref(dt)))
    return ds.value, dt.value


def normalize_data(kdata, mask=None, traj=None, dens=None, width=None, height=None):
    """The CLI's -o data normalisation (avx_normalize_data): scales the CUDA
    k-space tensor kdata in place and returns the factor.  Cartesian: kdata
    (T, C, H, W) and the mask (T, H, W); radial: kdata (T, C, S), traj
    (T, 2, S), dens (T, S) and the image size."""
    f = ctypes.c_float()
    if traj is None:
        T, C_, H, W = kdata.shape
        check(lib.avx_normalize_data(W, H, C_, T, 0, _cptr(mask), None, _cptr(kdata), ctypes.byref(f)))
    else:
        T, C_, S = kdata.shape
        check(lib.avx_normalize_data(width, height, C_, T, S, _cptr(traj), _cptr(dens), _cptr(kdata),
                                     ctypes.byref(f)))
    return f.value


def reconstruct_host(method, kdata, mask, b1, u0=None, params=None, debugstep=0):
    """Host-buffer reconstruction (the CLI path).  numpy in, numpy out."""
    import numpy as np
    if isinstance(method, str):
        method = METHODS[method.upper()]
    T, C, H, W = kdata.shape
    k = np.ascontiguousarray(kdata, dtype=np.complex64)
    b = np.ascontiguousarray(b1, dtype=np.complex64)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float32)
    u = None if u0 is None else np.ascontiguousarray(u0, dtype=np.complex64)
    x = np.empty((T, H, W), dtype=np.complex64)
    st = RunStats()
    pp = ctypes.byref(params) if params is not None else None
    check(lib.avx_reconstruct_host(
        method, W, H, C, T, pp, int(debugstep), k.ctypes.data_as(ctypes.c_void_p),
        None if m is None else m.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p),
        None if u is None else u.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p),
        ctypes.byref(st)))
    return x, st


# ---------------------------------------------------------------------------
# batched / served reconstructions
# ---------------------------------------------------------------------------

Request = _abi.Request
Completion = _abi.Completion


def cartesian_request(method, data, x, b1, mask=None, params=None, centered=False, dft_mode=DFT_SPLIT_BF16X3,
                      tag=0, stop_gap_rel=0.0):
    """avx_request for a Cartesian reconstruction.  data (T,C,H,W), x (T,H,W)
    initial image in / result out, b1 (C,H,W), mask (T,H,W) float32 or None:
    CUDA tensors that must stay alive until the completion is polled."""
    if isinstance(method, str):
        method = METHODS[method.upper()]
    T, C, H, W = data.shape
    r = Request()
    r.method, r.op_kind = method, 0
    r.width, r.height, r.coils, r.frames = W, H, C, T
    r.params = params if params is not None else default_params(method)
    r.dft_mode = int(dft_mode)
    r.d_mask = _cptr(mask) if mask is not None else None
    r.centered = int(centered)
    r.d_data, r.d_x, r.d_b1 = _cptr(data), _cptr(x), _cptr(b1)
    r.tag = int(tag)
    r.stop_gap_rel = float(stop_gap_rel)
    return r


def radial_request(method, data, x, b1, traj, dens, spokes_per_frame, n_fe, params=None, kernel_width=3.0,
                   sector_width=8.0, osf=2.0, tag=0, stop_gap_rel=0.0):
    """avx_request for a radial reconstruction: data (T,C,S) sqrt(w)-weighted,
    traj (T,2,S), dens (T,S) float32, x (T,H,W), b1 (C,H,W)."""
    if isinstance(method, str):
        method = METHODS[method.upper()]
    T, C, S = data.shape
    _, H, W = x.shape
    r = Request()
    r.method, r.op_kind = method, 1
    r.width, r.height, r.coils, r.frames = W, H, C, T
    r.params = params if params is not None else default_params(method)
    r.n_fe, r.spokes_per_frame = n_fe, spokes_per_frame
    r.d_traj, r.d_dens = _cptr(traj), _cptr(dens)
    r.kernel_width, r.sector_width, r.osf = kernel_width, sector_width, osf
    r.d_data, r.d_x, r.d_b1 = _cptr(data), _cptr(x), _cptr(b1)
    r.tag = int(tag)
    r.stop_gap_rel = float(stop_gap_rel)
    return r


def query_workspace(request):
    n = ctypes.c_size_t()
    check(lib.avx_query_workspace(ctypes.byref(request), ctypes.byref(n)))
    return n.value


class BatchEngine:
    """Continuous batching at iteration granularity (avx_batch_*): queued
    requests are admitted as their workspace fits the HBM budget, set up on
    streams of their own, advanced together (at most ``workers`` at a time)
    20 iterations at a time, and retired at their stop test or last
    iteration; each result equals the request run alone."""

    def __init__(self, device=0, hbm_budget=150 << 30, workers=8):
        self.handle = ctypes.c_void_p()
        check(lib.avx_batch_create(int(device), int(hbm_budget), int(workers), ctypes.byref(self.handle)))

    def submit(self, request):
        check(lib.avx_batch_submit(self.handle, ctypes.byref(request)))

    def poll(self, max_items=64, wait_ms=0):
        out = (Completion * max_items)()
        n = ctypes.c_int()
        check(lib.avx_serve_poll(self.handle, out, max_items, ctypes.byref(n), int(wait_ms)))
        return [out[i] for i in range(n.value)]

    def drain(self):
        check(lib.avx_batch_drain(self.handle))

    @property
    def pending(self):
        return lib.avx_batch_pending(self.handle)

    def close(self):
        if self.handle:
            lib.avx_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# coil-sensitivity estimation (CoilConstruction)
# ---------------------------------------------------------------------------

CoilParams = _abi.CoilParams


def coil_default_params():
    p = CoilParams()
    check(lib.avx_coil_default_params(ctypes.byref(p)))
    return p


def coil_time_averaged(kdata, mask, apply_phase=True):
    """kdata (T,C,H,W), mask (T,H,W) or None -> (u (H,W), crec (C,H,W))."""
    torch = _torch()
    T, C, H, W = kdata.shape
    u = torch.empty((H, W), dtype=torch.complex64, device=kdata.device)
    crec = torch.empty((C, H, W), dtype=torch.complex64, device=kdata.device)
    check(lib.avx_coil_time_averaged(W, H, C, T, _cptr(kdata), None if mask is None else _cptr(mask), _cptr(u),
                                     _cptr(crec), int(apply_phase)))
    return u, crec


def coil_b1_from_u_h1(u, crec, params=None):
    torch = _torch()
    C, H, W = crec.shape
    out = torch.empty_like(crec)
    p = params or coil_default_params()
    check(lib.avx_coil_b1_from_u_h1(W, H, C, ctypes.byref(p), _cptr(u), _cptr(crec), _cptr(out)))
    return out


def coil_utgv2(b1, crec, inds, x1, params=None):
    H, W = x1.shape
    arr = (ctypes.c_int * len(inds))(*inds)
    p = params or coil_default_params()
    check(lib.avx_coil_utgv2(W, H, ctypes.byref(p), _cptr(b1), _cptr(crec), arr, len(inds), _cptr(x1)))
    return x1


def coil_b1_recon(u0, crec, coils, max_it=500, mu=2.0, params=None):
    torch = _torch()
    H, W = u0.shape
    out = torch.empty((coils, H, W), dtype=torch.complex64, device=u0.device)
    p = params or coil_default_params()
    check(lib.avx_coil_b1_recon(W, H, coils, max_it, ctypes.c_float(mu), ctypes.byref(p), _cptr(u0), _cptr(crec),
                                _cptr(out)))
    return out


def coil_construction(kdata, mask, params=None):
    """PerformCoilConstruction: (u (C,H,W), b1 (C,H,W))."""
    torch = _torch()
    T, C, H, W = kdata.shape
    u = torch.empty((C, H, W), dtype=torch.complex64, device=kdata.device)
    b1 = torch.empty((C, H, W), dtype=torch.complex64, device=kdata.device)
    pp = ctypes.byref(params) if params is not None else None
    check(lib.avx_coil_construction(W, H, C, T, pp, _cptr(kdata), None if mask is None else _cptr(mask), _cptr(u),
                                    _cptr(b1)))
    return u, b1
