"""ctypes binding of the C ABI in include/tdscha_b200.h (libtdscha_b200.so, built in-tree).

There is no CPU fallback: importing the binding without the library, or calling it without an
sm_100 GPU, raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

PREC = {"fp64": 0, "tf32": 1, "bf16x3": 2, "tf32x3": 3, "bf16": 4}
ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "ENOSUPPORT", -5: "ETIMEOUT"}

_lib = None

dp = ctypes.POINTER(ctypes.c_double)
ip = ctypes.POINTER(ctypes.c_int)
vp = ctypes.c_void_p


class ApplyOpts(ctypes.Structure):
    _fields_ = [("use_wigner", ctypes.c_int), ("ignore_harmonic", ctypes.c_int), ("ignore_v3", ctypes.c_int),
                ("ignore_v4", ctypes.c_int), ("reverse_L", ctypes.c_int), ("shift_value", ctypes.c_double)]


class RunSystem(ctypes.Structure):
    """tdscha_run_system: one system of tdscha_lanczos_run_device."""
    _fields_ = [("ens", vp), ("n_chains", ctypes.c_int), ("qp", vp), ("sc", vp), ("coef", vp), ("opts", ApplyOpts),
                ("precision", ctypes.c_int)]


class TdschaError(RuntimeError):
    pass


def library_path():
    return _build.LIB_PATH


def load():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise TdschaError(f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    lib.tdscha_last_error.restype = ctypes.c_char_p
    lib.tdscha_version.restype = ctypes.c_char_p
    lib.tdscha_ensemble_create.argtypes = [dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_int, ip, ctypes.POINTER(ip), ctypes.POINTER(dp), ip,
                                           ctypes.POINTER(vp)]
    lib.tdscha_ensemble_destroy.argtypes = [vp]
    lib.tdscha_ensemble_info.argtypes = [vp, ip, ip, ip, ip, dp, dp]
    lib.tdscha_ensemble_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    lib.tdscha_ensemble_cosets.argtypes = [vp, ip, ip, ip, dp]
    lib.tdscha_symmetry_cosets.argtypes = [ctypes.c_int, ctypes.c_int, ip, ctypes.POINTER(dp), ip, ip, ip, ip, dp, dp]
    lib.tdscha_ensemble_classes.argtypes = [vp, ip, ip, ip, dp]
    lib.tdscha_symmetry_classes.argtypes = [ctypes.c_int, ctypes.c_int, ip, ctypes.POINTER(dp), ip, dp, ip, ip, dp, ip, dp,
                                            ip, dp, ip]
    lib.tdscha_perturb_average_sym.argtypes = [vp, dp, dp, ctypes.c_int, ctypes.c_int, dp, dp]
    lib.tdscha_perturb_average_sym_device.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp]
    lib.tdscha_GetPerturbAverageSym.argtypes = [dp, dp, dp, dp, dp, dp, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.POINTER(dp), ip, ctypes.POINTER(ip), ip,
                                                ctypes.c_int, ctypes.c_int, dp, dp]
    lib.tdscha_apply_full_L_device.argtypes = [vp, ctypes.c_int, vp, ip, ctypes.POINTER(ApplyOpts), ctypes.c_int, vp, vp]
    lib.tdscha_lanczos_step_device.argtypes = [ctypes.c_int, ctypes.c_longlong, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                               vp, vp]
    lib.tdscha_lanczos_step_device_noalloc.argtypes = list(lib.tdscha_lanczos_step_device.argtypes)
    lib.tdscha_continued_fraction_device.argtypes = [ctypes.c_int, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                     vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                     ctypes.c_int, ctypes.c_double, ctypes.c_double, vp, vp]
    lib.tdscha_tc_contract.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_longlong,
                                       vp, vp, ctypes.c_longlong, vp, ctypes.c_longlong, vp]
    lib.tdscha_perturb_average_vjp_device.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, vp, vp, vp, vp, vp]
    lib.tdscha_perturb_average_vjp_precision_device.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_int, vp,
                                                                vp, vp, vp, vp]
    lib.tdscha_project_ensemble.argtypes = [dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
    lib.tdscha_symmetries_on_modes.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, dp, ctypes.c_int, ip,
                                               ctypes.POINTER(ip), ctypes.POINTER(dp)]
    lib.tdscha_apply_prologue_device.argtypes = [vp, ctypes.c_int, vp, ip, ctypes.POINTER(ApplyOpts), vp, vp, vp]
    lib.tdscha_apply_epilogue_device.argtypes = [vp, ctypes.c_int, vp, ip, ctypes.POINTER(ApplyOpts), vp, vp, vp, vp]
    lib.tdscha_apply_L1_static_device.argtypes = [vp, ctypes.c_int, vp, ctypes.c_double, vp, vp]
    lib.tdscha_apply_static_L_device.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp]
    lib.tdscha_lanczos_run_device.argtypes = [ctypes.c_int, ctypes.POINTER(RunSystem), ctypes.c_int, ctypes.c_int, vp]
    lib.tdscha_set_wait_budget.argtypes = [ctypes.c_double]
    lib.tdscha_debug_stall_next_contraction.argtypes = []
    lib.tdscha_set_error_check.argtypes = [ctypes.c_int]
    lib.tdscha_check_errors.argtypes = [vp, vp]
    lib.tdscha_set_profiling.argtypes = [vp, ctypes.c_int]
    lib.tdscha_read_profile.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
    for name in ("tdscha_perturb_average_vjp_precision_device", "tdscha_set_wait_budget", "tdscha_debug_stall_next_contraction", "tdscha_apply_L1_static_device", "tdscha_apply_static_L_device", "tdscha_lanczos_run_device", "tdscha_lanczos_step_device_noalloc", "tdscha_apply_prologue_device", "tdscha_apply_epilogue_device", "tdscha_set_profiling", "tdscha_read_profile", "tdscha_tc_contract", "tdscha_ensemble_create", "tdscha_ensemble_destroy", "tdscha_ensemble_info",
                 "tdscha_ensemble_device_bytes", "tdscha_perturb_average_sym", "tdscha_perturb_average_sym_device",
                 "tdscha_GetPerturbAverageSym", "tdscha_apply_full_L_device", "tdscha_lanczos_step_device",
                 "tdscha_continued_fraction_device"):
        getattr(lib, name).restype = ctypes.c_int
    _lib = lib
    return lib


def check(rc):
    if rc != 0:
        msg = _lib.tdscha_last_error().decode() if _lib is not None else ""
        raise TdschaError(f"tdscha_b200 error {ERRORS.get(rc, rc)}: {msg}")


def _d(a):
    return a.ctypes.data_as(dp)


def _i(a):
    return a.ctypes.data_as(ip)


class DeviceEnsemble:
    """Owner of a ``tdscha_ensemble`` handle (X, Y, rho, w and the symmetry tables resident in HBM)."""

    def __init__(self, X, Y, w, rho, T, symmetries, deg_space, blocks_ids):
        lib = load()
        self.X = np.ascontiguousarray(X, dtype=np.float64)
        self.Y = np.ascontiguousarray(Y, dtype=np.float64)
        self.w = np.ascontiguousarray(w, dtype=np.float64)
        self.rho = np.ascontiguousarray(rho, dtype=np.float64)
        self.T = float(T)
        N, n = self.X.shape
        self.N, self.n = N, n
        syms = [np.ascontiguousarray(s, dtype=np.float64) for s in symmetries]
        degs = [np.ascontiguousarray(d, dtype=np.intc) for d in deg_space]
        self.N_sym = int(syms[0].shape[0])
        n_deg = np.array([len(d) for d in degs], dtype=np.intc)
        bid = np.ascontiguousarray(blocks_ids, dtype=np.intc)
        sym_ptrs = (dp * len(syms))(*[_d(s) for s in syms])
        deg_ptrs = (ip * len(degs))(*[_i(d) for d in degs])
        h = vp()
        check(lib.tdscha_ensemble_create(_d(self.X), _d(self.Y), _d(self.w), _d(self.rho), N, n, self.T, self.N_sym,
                                         len(syms), _i(n_deg), deg_ptrs, sym_ptrs, _i(bid), ctypes.byref(h)))
        self.handle = h
        self._lib = lib

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self._lib.tdscha_ensemble_destroy(self.handle)
            self.handle = vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def classes(self):
        """dict(n_class, Kq, Kmq, flops_ratio) of the character-class contractions (n_class 0: off)."""
        nc, kq, kmq, r = ensemble_classes(self.handle)
        return dict(n_class=nc, Kq=kq, Kmq=kmq, flops_ratio=r)

    def device_bytes(self):
        b = ctypes.c_longlong()
        check(self._lib.tdscha_ensemble_device_bytes(self.handle, ctypes.byref(b)))
        return b.value

    def cosets(self):
        """The factorised symmetry path: dict(rotated, n_cosets, coset_size, offpattern)
        (tdscha_ensemble_cosets; n_cosets = 0 when the general symmetry kernels run)."""
        r, nc, cs, off = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(self._lib.tdscha_ensemble_cosets(self.handle, ctypes.byref(r), ctypes.byref(nc), ctypes.byref(cs),
                                               ctypes.byref(off)))
        return dict(rotated=bool(r.value), n_cosets=nc.value, coset_size=cs.value, offpattern=off.value)

    STAGES = ("transform", "gemm_ab", "gemm_cd", "weights", "gemm_z", "gemm_f", "fold", "other", "operands")

    def set_profiling(self, enable=True):
        check(self._lib.tdscha_set_profiling(self.handle, int(enable)))

    def read_profile(self):
        """{stage: (milliseconds, launches)} since the last read (synchronises)."""
        ms = np.zeros(len(self.STAGES))
        cnt = (ctypes.c_longlong * len(self.STAGES))()
        check(self._lib.tdscha_read_profile(self.handle, _d(ms), cnt, len(self.STAGES)))
        return {s: (float(ms[i]), int(cnt[i])) for i, s in enumerate(self.STAGES)}

    def perturb_average(self, R1, Y1, apply_d4=1, precision="fp64"):
        """Host-buffer drop-in of GetPerturbAverageSym: returns (f_av (n), d2v (n, n))."""
        R1 = np.ascontiguousarray(R1, dtype=np.float64)
        Y1 = np.ascontiguousarray(Y1, dtype=np.float64)
        f = np.zeros(self.n)
        d = np.zeros((self.n, self.n))
        check(self._lib.tdscha_perturb_average_sym(self.handle, _d(R1), _d(Y1), int(apply_d4), PREC[precision], _d(f), _d(d)))
        return f, d

    def perturb_average_device(self, R1, Y1, f_out, d_out, apply_d4=1, precision="fp64", stream=None):
        """Batched device version on torch tensors: R1 (nb, n), Y1 (nb, n, n) float64 CUDA."""
        nb = R1.shape[0]
        check(self._lib.tdscha_perturb_average_sym_device(self.handle, nb, R1.data_ptr(), Y1.data_ptr(), int(apply_d4),
                                                          PREC[precision], f_out.data_ptr(), d_out.data_ptr(),
                                                          _stream_ptr(stream)))

    def perturb_average_vjp(self, R1, Ys, fbar, Dbar, Ybar, rhobar, apply_d4=1, stream=None, precision="fp64"):
        """d[sum_k <fbar_k, f_k> + <Dbar_k, D_k>] / d(Y, rho) into Ybar (N, n), rhobar (N); all float64
        CUDA tensors, Ys and Dbar symmetric (nb, n, n); `precision` of the eight ensemble contractions."""
        nb = R1.shape[0]
        if precision == "fp64":
            check(self._lib.tdscha_perturb_average_vjp_device(self.handle, nb, R1.data_ptr(), Ys.data_ptr(), int(apply_d4),
                                                              fbar.data_ptr(), Dbar.data_ptr(), Ybar.data_ptr(),
                                                              rhobar.data_ptr(), _stream_ptr(stream)))
            return
        check(self._lib.tdscha_perturb_average_vjp_precision_device(
            self.handle, nb, R1.data_ptr(), Ys.data_ptr(), int(apply_d4), PREC[precision], fbar.data_ptr(),
            Dbar.data_ptr(), Ybar.data_ptr(), rhobar.data_ptr(), _stream_ptr(stream)))

    def apply_full_L(self, psi, out, transpose, opts, precision="fp64", stream=None):
        """psi, out: (nb, len) float64 CUDA tensors; transpose: sequence of nb ints."""
        nb = psi.shape[0]
        tr = np.ascontiguousarray(np.asarray(transpose, dtype=np.intc).reshape(nb))
        check(self._lib.tdscha_apply_full_L_device(self.handle, nb, psi.data_ptr(), _i(tr), ctypes.byref(opts),
                                                   PREC[precision], out.data_ptr(), _stream_ptr(stream)))


    def apply_prologue(self, psi, R_out, Y_out, transpose, opts, stream=None):
        nb = psi.shape[0]
        tr = np.ascontiguousarray(np.asarray(transpose, dtype=np.intc).reshape(nb))
        check(self._lib.tdscha_apply_prologue_device(self.handle, nb, psi.data_ptr(), _i(tr), ctypes.byref(opts),
                                                     R_out.data_ptr(), Y_out.data_ptr(), _stream_ptr(stream)))

    def apply_epilogue(self, psi, f_av, d_av, out, transpose, opts, stream=None):
        nb = psi.shape[0]
        tr = np.ascontiguousarray(np.asarray(transpose, dtype=np.intc).reshape(nb))
        check(self._lib.tdscha_apply_epilogue_device(self.handle, nb, psi.data_ptr(), _i(tr), ctypes.byref(opts),
                                                     f_av.data_ptr(), d_av.data_ptr(), out.data_ptr(),
                                                     _stream_ptr(stream)))


def _static_check(ens, psi, out):
    n = ens.n
    ln = n + n * (n + 1) // 2
    if psi.dim() != 2 or psi.shape[1] != ln or tuple(out.shape) != tuple(psi.shape):
        raise ValueError(f"static vectors must be (nb, {ln}); got {tuple(psi.shape)} -> {tuple(out.shape)}")
    for t in (psi, out):
        if not t.is_contiguous() or str(t.dtype) != "torch.float64" or not t.is_cuda:
            raise ValueError("static vectors must be contiguous float64 CUDA tensors")


def apply_L1_static(ens, psi, out, power=1.0, stream=None):
    """tdscha_apply_L1_static_device on (nb, n + n(n+1)/2) tensors (power already signed)."""
    _static_check(ens, psi, out)
    check(ens._lib.tdscha_apply_L1_static_device(ens.handle, psi.shape[0], psi.data_ptr(), float(power), out.data_ptr(),
                                                 _stream_ptr(stream)))


def apply_static_L(ens, psi, out, ignore_v4=False, include_L1=True, precision="fp64", stream=None):
    """tdscha_apply_static_L_device on (nb, n + n(n+1)/2) tensors, in batches of 64 vectors."""
    _static_check(ens, psi, out)
    for k0 in range(0, psi.shape[0], 64):
        k1 = min(psi.shape[0], k0 + 64)
        check(ens._lib.tdscha_apply_static_L_device(ens.handle, k1 - k0, psi[k0:k1].data_ptr(), int(bool(ignore_v4)),
                                                    int(bool(include_L1)), PREC[precision], out[k0:k1].data_ptr(),
                                                    _stream_ptr(stream)))


def _stream_ptr(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return stream


def lanczos_step(Lq, pL, q, p, q_prev, p_prev, sc_in, mask, q_next, p_next, sc_out, stream=None):
    lib = load()
    nc, length = Lq.shape
    ptr = lambda t: None if t is None else t.data_ptr()   # noqa: E731
    check(lib.tdscha_lanczos_step_device(nc, length, ptr(Lq), ptr(pL), ptr(q), ptr(p), ptr(q_prev), ptr(p_prev),
                                         ptr(sc_in), ptr(mask), ptr(q_next), ptr(p_next), ptr(sc_out),
                                         _stream_ptr(stream)))


def lanczos_run(systems, n_steps, use_graph=True, stream=None):
    """tdscha_lanczos_run_device.  systems: list of (DeviceEnsemble, qp, sc, coef, ApplyOpts, precision)
    with qp (4, nc, len), sc (nc, 6), coef (n_steps, nc, 4) contiguous float64 CUDA tensors."""
    lib = load()
    arr = (RunSystem * len(systems))()
    for i, (ens, qp, sc, coef, opts, prec) in enumerate(systems):
        nc = qp.shape[1]
        if qp.shape[0] != 4 or tuple(sc.shape) != (nc, 6) or tuple(coef.shape) != (n_steps, nc, 4):
            raise ValueError(f"system {i}: shapes qp {tuple(qp.shape)}, sc {tuple(sc.shape)}, coef {tuple(coef.shape)}")
        for t in (qp, sc, coef):
            if not t.is_contiguous() or str(t.dtype) != "torch.float64" or not t.is_cuda:
                raise ValueError(f"system {i}: state tensors must be contiguous float64 CUDA tensors")
        arr[i] = RunSystem(ens.handle.value, nc, qp.data_ptr(), sc.data_ptr(), coef.data_ptr(), opts, PREC[prec])
    check(lib.tdscha_lanczos_run_device(len(systems), arr, int(n_steps), int(bool(use_graph)), _stream_ptr(stream)))


def lanczos_step_noalloc(Lq, pL, q, p, q_prev, p_prev, sc_in, mask, q_next, p_next, sc_out, stream=None):
    """Same step through tdscha_lanczos_step_device_noalloc (fixed in-library scratch, <= 32 chains)."""
    lib = load()
    nc, length = Lq.shape
    ptr = lambda t: None if t is None else t.data_ptr()   # noqa: E731
    check(lib.tdscha_lanczos_step_device_noalloc(nc, length, ptr(Lq), ptr(pL), ptr(q), ptr(p), ptr(q_prev),
                                                 ptr(p_prev), ptr(sc_in), ptr(mask), ptr(q_next), ptr(p_next),
                                                 ptr(sc_out), _stream_ptr(stream)))


def continued_fraction(a, b, c, omega, gf_out, use_terminator, last_average, smearing, use_wigner, reverse_L,
                       shift_value, modulus, stream=None):
    lib = load()
    nb = 0 if b is None else b.numel()
    ncc = 0 if c is None else c.numel()
    check(lib.tdscha_continued_fraction_device(a.numel(), a.data_ptr(), None if b is None else b.data_ptr(),
                                               None if c is None else c.data_ptr(), nb, ncc, omega.numel(),
                                               omega.data_ptr(), int(use_terminator), int(last_average),
                                               float(smearing), int(use_wigner), int(reverse_L), float(shift_value),
                                               float(modulus), gf_out.data_ptr(), _stream_ptr(stream)))


def tc_contract(precision, A_hi, A_lo, B_hi, B_lo, D, stream=None):
    """D (M x N fp32 CUDA tensor, row stride D.stride(0)) = A (M x K) . B (N x K)^T on the tensor cores.
    A_*/B_* are row-major CUDA tensors (bf16, or fp32 holding tf32 values); *_lo may be None for
    the one-product modes."""
    lib = load()
    M, K = A_hi.shape
    N = B_hi.shape[0]
    for t in (A_hi, B_hi, D) + tuple(x for x in (A_lo, B_lo) if x is not None):
        if not t.is_cuda or t.stride(-1) != 1:
            raise ValueError("operands must be CUDA tensors with unit inner stride")
    if D.dtype.itemsize != 4 or D.shape[0] < M or D.shape[1] < N:
        raise ValueError("D must be an fp32 tensor of at least M x N")
    ptr = lambda t: None if t is None else t.data_ptr()   # noqa: E731
    check(lib.tdscha_tc_contract(PREC[precision], M, N, K, ptr(A_hi), ptr(A_lo), A_hi.stride(0), ptr(B_hi),
                                 ptr(B_lo), B_hi.stride(0), D.data_ptr(), D.stride(0), _stream_ptr(stream)))


def set_wait_budget(seconds):
    """Budget of every bounded wait of the tensor-core kernels launched afterwards (default 4 s)."""
    check(load().tdscha_set_wait_budget(float(seconds)))


def set_error_check(per_call):
    """tdscha_set_error_check: read the error word after every device call (True, default) or only
    in check_errors (False)."""
    check(load().tdscha_set_error_check(1 if per_call else 0))


def check_errors(handle, stream=None):
    """tdscha_check_errors: wait for the stream, raise on a bounded wait that ran out since the last check."""
    check(load().tdscha_check_errors(handle, _stream_ptr(stream)))


def debug_stall_next_contraction():
    """The next tensor-core contraction launch issues no operand copy: its waits run out and the call
    returns TDSCHA_ETIMEOUT (a test of the abort path)."""
    check(load().tdscha_debug_stall_next_contraction())


def get_perturb_average_sym(X, Y, w, rho, R1, Y1, T, apply_D4, N_syms, sym_list, n_deg, deg_space_list, blocks_ids,
                            f_out, d2v_out):
    """Same argument list and in-place outputs as ``sscha_HP_odd.GetPerturbAverageSym``
    (CModules/odd_corr_module.c:519-520), FP64 on the GPU.  Unlike the reference, bad arguments
    raise instead of terminating the process."""
    lib = load()
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    R1 = np.ascontiguousarray(R1, dtype=np.float64)
    Y1 = np.ascontiguousarray(Y1, dtype=np.float64)
    N, n = X.shape
    if len(w) != n:
        raise ValueError(f"N_modes from X is {n}, while len(w) = {len(w)}")
    syms = [np.ascontiguousarray(s, dtype=np.float64) for s in sym_list]
    degs = [np.ascontiguousarray(d, dtype=np.intc) for d in deg_space_list]
    n_deg = np.ascontiguousarray(n_deg, dtype=np.intc)
    bid = np.ascontiguousarray(blocks_ids, dtype=np.intc)
    for name, arr, shape in (("f_out", f_out, (n,)), ("d2v_out", d2v_out, (n, n))):
        if arr.dtype != np.float64 or arr.shape != shape or not arr.flags.c_contiguous:
            raise ValueError(f"{name} must be a C-contiguous float64 array of shape {shape}")
    sym_ptrs = (dp * len(syms))(*[_d(s) for s in syms])
    deg_ptrs = (ip * len(degs))(*[_i(d) for d in degs])
    check(lib.tdscha_GetPerturbAverageSym(_d(X), _d(Y), _d(w), _d(rho), _d(R1), _d(Y1), float(T), int(apply_D4),
                                          int(N_syms), len(syms), sym_ptrs, _i(n_deg), deg_ptrs, _i(bid), N, n,
                                          _d(f_out), _d(d2v_out)))


def project_ensemble(u, f, masses, pols):
    """X = (u o sqrt(m)) . pols, Y = (f / sqrt(m)) . pols on the GPU (tdscha_project_ensemble)."""
    lib = load()
    u = np.ascontiguousarray(u, dtype=np.float64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    m = np.ascontiguousarray(masses, dtype=np.float64)
    P = np.ascontiguousarray(pols, dtype=np.float64)
    N, nat3 = u.shape
    if f.shape != u.shape or m.shape != (nat3,) or P.shape[0] != nat3:
        raise ValueError(f"shapes: u {u.shape}, f {f.shape}, masses {m.shape}, pols {P.shape}")
    n = P.shape[1]
    X = np.empty((N, n))
    Y = np.empty((N, n))
    check(lib.tdscha_project_ensemble(_d(u), _d(f), _d(m), _d(P), N, nat3, n, _d(X), _d(Y)))
    return X, Y


def symmetry_cosets(symmetries):
    """Host analysis of per-block symmetry tables (list of (N_sym, d, d)) behind the factorised
    symmetry path (tdscha_symmetry_cosets; no device needed).  Returns None when the group has no
    such structure, else dict(n_cosets, coset_size, order (N_sym), partner (n), R (list of d x d
    rotations, R_b[q', q] = component q' of rotated mode q), offpattern)."""
    lib = load()
    tabs = [np.ascontiguousarray(t, dtype=np.float64) for t in symmetries]
    N_sym = tabs[0].shape[0]
    dims = [t.shape[1] for t in tabs]
    n = sum(dims)
    n_deg = np.array(dims, dtype=np.intc)
    ptrs = (dp * len(tabs))(*[_d(t) for t in tabs])
    nc, cs, off = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    order = np.zeros(N_sym, dtype=np.intc)
    partner = np.zeros(n, dtype=np.intc)
    R = np.zeros(sum(d * d for d in dims))
    check(lib.tdscha_symmetry_cosets(N_sym, len(tabs), _i(n_deg), ptrs, ctypes.byref(nc), ctypes.byref(cs), _i(order),
                                     _i(partner), _d(R), ctypes.byref(off)))
    if nc.value == 0:
        return None
    Rs, o = [], 0
    for d in dims:
        Rs.append(R[o:o + d * d].reshape(d, d).copy())
        o += d * d
    return dict(n_cosets=nc.value, coset_size=cs.value, order=order, partner=partner, R=Rs, offpattern=off.value)


def symmetry_classes(symmetries):
    """Character classes of the factorised path on per-block symmetry tables (host, no device):
    tdscha_symmetry_classes.  None when the group has no such structure, else a dict of the layout
    arrays (see include/tdscha_b200.h)."""
    lib = load()
    tabs = [np.ascontiguousarray(t, dtype=np.float64) for t in symmetries]
    N_sym = tabs[0].shape[0]
    n_deg = np.array([t.shape[1] for t in tabs], dtype=np.intc)
    n = int(n_deg.sum())
    ptrs = (dp * len(tabs))(*[_d(t) for t in tabs])
    sizes = np.zeros(4, dtype=np.intc)
    ratio = ctypes.c_double()
    check(lib.tdscha_symmetry_classes(N_sym, len(tabs), _i(n_deg), ptrs, _i(sizes), ctypes.byref(ratio), None, None, None,
                                      None, None, None, None, None))
    nC, Kq, Kmq, P = (int(x) for x in sizes)
    if nC == 0:
        return None
    cls = np.zeros((nC, 5), dtype=np.intc)
    pcol_i = np.zeros((Kq, 5), dtype=np.intc)
    pcol_d = np.zeros((Kq, 5))
    pp_i = np.zeros((P, 2), dtype=np.intc)
    pp_d = np.zeros((P, 2))
    mcol_i = np.zeros((max(Kmq, 1), 2), dtype=np.intc)
    mcol_d = np.zeros((max(Kmq, 1), 4))
    mode_col = np.zeros(n, dtype=np.intc)
    check(lib.tdscha_symmetry_classes(N_sym, len(tabs), _i(n_deg), ptrs, _i(sizes), ctypes.byref(ratio), _i(cls), _i(pcol_i),
                                      _d(pcol_d), _i(pp_i), _d(pp_d), _i(mcol_i), _d(mcol_d), _i(mode_col)))
    return dict(n_class=nC, Kq=Kq, Kmq=Kmq, flops_ratio=ratio.value, cls=cls, pcol_i=pcol_i, pcol_d=pcol_d, pp_i=pp_i,
                pp_d=pp_d, mcol_i=mcol_i[:Kmq], mcol_d=mcol_d[:Kmq], mode_col=mode_col)


def ensemble_classes(handle):
    """(n_class, Kq, Kmq, flops_ratio) of a resident ensemble (tdscha_ensemble_classes)."""
    lib = load()
    nc, kq, kmq, r = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    check(lib.tdscha_ensemble_classes(handle, ctypes.byref(nc), ctypes.byref(kq), ctypes.byref(kmq), ctypes.byref(r)))
    return nc.value, kq.value, kmq.value, r.value


def symmetries_on_modes(pols, perm, rot, deg_space):
    """Per degenerate block the (N_sym, d, d) tables S_b^j = E_b^T P_j E_b on the GPU
    (tdscha_symmetries_on_modes); perm (N_sym, nat) image atoms, rot (N_sym, 3, 3)."""
    lib = load()
    P = np.ascontiguousarray(pols, dtype=np.float64)
    perm = np.ascontiguousarray(perm, dtype=np.intc)
    rot = np.ascontiguousarray(rot, dtype=np.float64)
    N_sym, nat = perm.shape
    if rot.shape != (N_sym, 3, 3) or P.shape[0] != 3 * nat:
        raise ValueError(f"shapes: perm {perm.shape}, rot {rot.shape}, pols {P.shape}")
    degs = [np.ascontiguousarray(d, dtype=np.intc) for d in deg_space]
    out = [np.empty((N_sym, len(d), len(d))) for d in degs]
    n_deg = np.array([len(d) for d in degs], dtype=np.intc)
    deg_ptrs = (ip * len(degs))(*[_i(d) for d in degs])
    out_ptrs = (dp * len(out))(*[_d(o) for o in out])
    check(lib.tdscha_symmetries_on_modes(_d(P), nat, P.shape[1], N_sym, _i(perm), _d(rot), len(degs), _i(n_deg), deg_ptrs,
                                         out_ptrs))
    return out
