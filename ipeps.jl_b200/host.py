"""Host side of the B200 CTMRG engine: the reference's Julia API, in Python.

The names, argument meaning and defaults mirror iPEPS.jl (paths relative to
its source tree):

    CTMTensors(A, cfg)          src/ctm/ctm_tensor.jl:57-69 (init_ctm1 :97-130)
    run_ctm(ts, conv_fun=...)   src/ctm/ctmrg.jl:1-55
    rg_step(ts, chi)            src/ctm/ctmrg.jl:57-64
    left_rg/right_rg/top_rg/bottom_rg   src/ctm/ctmrg.jl:66-120
    get_gs_energy(ts, H)        src/graph/evaluation.jl:15-29
    get_gs_norm(ts)             src/graph/evaluation.jl:47-59
    compute_gs_energy(A, H, cfg) src/graph/evaluation.jl:1-13
    get_es_energy(ts, H)        src/graph/evaluation.jl:31-45
    get_all_norm(ts)            src/graph/evaluation.jl:61-77

Every call goes through the C ABI of libipeps_b200.so (include/ipeps_b200.h);
there is no CPU fallback: if the shared library is missing the import fails.
Arrays are numpy arrays with Julia (column-major) semantics: shapes are the
Julia shapes and data is passed in Fortran order.
"""
from __future__ import annotations

import ctypes as ct
import os
from typing import Any, Dict, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libipeps_b200.so")

OK, ENOTCONV, ENONFINITE, EOOM, EINVAL, ECUDA = range(6)
PREC_FP64, PREC_MIXED = 0, 1
CONV_ENERGY, CONV_SPECTRUM, CONV_ES = 0, 1, 2

EXPORTED = [
    "ipeps_ctx_create", "ipeps_ctx_destroy", "ipeps_last_error", "ipeps_ctx_set_precision",
    "ipeps_ctx_set_seed", "ipeps_stats", "ipeps_stats_reset", "ipeps_env_create", "ipeps_env_destroy",
    "ipeps_env_set_params", "ipeps_env_set_svd_params", "ipeps_env_set_parallel", "ipeps_env_set_A", "ipeps_env_init",
    "ipeps_env_get_CT", "ipeps_env_set_CT", "ipeps_ctm_move", "ipeps_ctm_step", "ipeps_ctm_run",
    "ipeps_ctm_log", "ipeps_energy", "ipeps_gs_norm", "ipeps_nested_set_B", "ipeps_es_energy",
    "ipeps_all_norm", "ipeps_tcon", "ipeps_projector", "ipeps_projector_c", "ipeps_ctx_stream", "ipeps_prof_enable",
    "ipeps_prof_query", "ipeps_prof_phases", "ipeps_energy_grad", "ipeps_env_set_mixed", "ipeps_es_energy_grad",
    "ipeps_single_dm_Ad", "ipeps_wp_grad", "ipeps_energy_4x4", "ipeps_ctm_run_4x4", "ipeps_energy_grad_4x4", "ipeps_es_energy_grad_4x4", "ipeps_gemm_f64", "ipeps_gemm_tf32x3", "ipeps_orth", "ipeps_gemm_bf16", "ipeps_mlp_create", "ipeps_mlp_destroy", "ipeps_mlp_num_params",
    "ipeps_mlp_get_params", "ipeps_mlp_set_params", "ipeps_mlp_forward", "ipeps_mlp_grad", "ipeps_mlp_train_step",
]


class IPEPSError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[ipeps status {code}] {msg}")
        self.code = code


class CTensor(ct.Structure):
    """ipeps_ctensor_t: a complex128 column-major array of rank <= 4."""
    _fields_ = [("data", ct.c_void_p), ("nd", ct.c_int), ("dims", ct.c_int64 * 4)]


class Stats(ct.Structure):
    _fields_ = [("launches", ct.c_uint64 * 8), ("flops", ct.c_double * 8), ("bytes", ct.c_double * 8),
                ("moves", ct.c_uint64), ("move_seconds", ct.c_double), ("projector_calls", ct.c_uint64),
                ("jacobi_sweeps", ct.c_uint64), ("extra_passes", ct.c_uint64), ("series_cap_hits", ct.c_uint64),
                ("series_terms", ct.c_uint64), ("series_retries", ct.c_uint64), ("resid_misses", ct.c_uint64)]

    FAMILIES = ["permute", "gemm_f64", "gemm_tf32x3", "reduce", "elementwise", "small_linalg", "jacobi"]

    def as_dict(self):
        fam = {n: {"launches": int(self.launches[i]), "flops": float(self.flops[i]), "bytes": float(self.bytes[i])}
               for i, n in enumerate(self.FAMILIES)}
        return {"families": fam, "moves": int(self.moves), "move_seconds": float(self.move_seconds),
                "projector_calls": int(self.projector_calls), "jacobi_sweeps": int(self.jacobi_sweeps),
                "extra_passes": int(self.extra_passes), "series_cap_hits": int(self.series_cap_hits),
                "series_terms": int(self.series_terms), "series_retries": int(self.series_retries),
                "resid_misses": int(self.resid_misses)}


_lib = None


def load_library(path: str = LIB_PATH) -> ct.CDLL:
    """Load libipeps_b200.so and declare the C signatures (fails loudly when absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libipeps_b200.so not found at {path}: build it with "
                          "`python ipeps.jl_b200/build.py` (the engine has no CPU fallback)")
    lib = ct.CDLL(path)
    P, I, D, U64 = ct.c_void_p, ct.c_int, ct.c_double, ct.c_uint64
    dp = ct.POINTER(ct.c_double)
    ip = ct.POINTER(ct.c_int)
    lp = ct.POINTER(ct.c_int64)
    fp = ct.POINTER(ct.c_float)
    sig = {
        "ipeps_ctx_create": [I, ct.POINTER(P)],
        "ipeps_ctx_destroy": [P],
        "ipeps_ctx_set_precision": [P, I],
        "ipeps_ctx_set_seed": [P, U64],
        "ipeps_stats": [P, ct.POINTER(Stats)],
        "ipeps_stats_reset": [P],
        "ipeps_env_create": [P, I, I, I, I, ct.POINTER(P)],
        "ipeps_env_destroy": [P],
        "ipeps_env_set_params": [P, I, I, I, I, D],
        "ipeps_env_set_svd_params": [P, I, I, I, I, I, I, D, I, I, I],
        "ipeps_env_set_parallel": [P, I],
        "ipeps_env_set_A": [P, dp, dp],
        "ipeps_env_init": [P],
        "ipeps_env_get_CT": [P, I, dp, lp, dp, lp],
        "ipeps_env_set_CT": [P, I, dp, lp, dp, lp],
        "ipeps_ctm_move": [P, I, dp, ip],
        "ipeps_ctm_step": [P, dp, ip],
        "ipeps_ctm_run": [P, I, dp, dp, I, ip, dp, ip],
        "ipeps_ctm_log": [P, dp, ip],
        "ipeps_energy": [P, dp, dp, I, dp, dp],
        "ipeps_gs_norm": [P, dp],
        "ipeps_nested_set_B": [P, dp, D, D],
        "ipeps_es_energy": [P, dp, dp, I, dp],
        "ipeps_all_norm": [P, dp, dp],
        "ipeps_tcon": [P, I, dp, I, lp, ip, dp, I, lp, ip, dp, ct.c_int64, lp, ip],
        "ipeps_projector": [P, dp, dp, ct.c_int64, ct.c_int64, ct.c_int64, I, dp, dp, dp, ip],
        "ipeps_projector_c": [P, dp, dp, ct.c_int64, ct.c_int64, ct.c_int64, I, dp, dp, dp, ip],
        "ipeps_ctx_stream": [P, ct.POINTER(P)],
        "ipeps_prof_enable": [P, I],
        "ipeps_prof_query": [P, dp, ct.POINTER(ct.c_uint64), dp, dp],
        "ipeps_prof_phases": [P, dp],
        "ipeps_energy_grad": [P, dp, dp, I, I, dp, dp],
        "ipeps_env_set_mixed": [P, I, D],
        "ipeps_es_energy_grad": [P, dp, dp, I, I, dp, dp],
        "ipeps_energy_4x4": [P, ct.POINTER(CTensor), I, dp],
        "ipeps_ctm_run_4x4": [P, ct.POINTER(CTensor), I, ip, dp, ip],
        "ipeps_energy_grad_4x4": [P, ct.POINTER(CTensor), I, dp, dp],
        "ipeps_es_energy_grad_4x4": [P, ct.POINTER(CTensor), I, dp, dp],
        "ipeps_wp_grad": [P, ct.POINTER(CTensor), I, dp, dp, dp, dp],
        "ipeps_single_dm_Ad": [P, dp],
        "ipeps_gemm_f64": [P, ct.c_char, ct.c_char, ct.c_int64, ct.c_int64, ct.c_int64, D, dp, ct.c_int64, dp,
                           ct.c_int64, D, dp, ct.c_int64, I],
        "ipeps_gemm_tf32x3": [P, ct.c_char, ct.c_char, ct.c_int64, ct.c_int64, ct.c_int64, D, dp, ct.c_int64, dp,
                              ct.c_int64, D, dp, ct.c_int64, I, dp],
        "ipeps_orth": [P, dp, ct.c_int64, I, I, dp, dp],
        "ipeps_gemm_bf16": [P, ct.c_char, ct.c_char, ct.c_int64, ct.c_int64, ct.c_int64, ct.c_float, fp,
                            ct.c_int64, fp, ct.c_int64, ct.c_float, fp, ct.c_int64],
        "ipeps_mlp_create": [P, I, I, I, I, U64, ct.POINTER(P)],
        "ipeps_mlp_destroy": [P],
        "ipeps_mlp_num_params": [P, lp],
        "ipeps_mlp_get_params": [P, fp],
        "ipeps_mlp_set_params": [P, fp],
        "ipeps_mlp_forward": [P, fp, I, fp],
        "ipeps_mlp_grad": [P, fp, fp, I, dp, fp],
        "ipeps_mlp_train_step": [P, fp, fp, I, ct.c_float, dp],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = I
    lib.ipeps_last_error.argtypes = [P]
    lib.ipeps_last_error.restype = ct.c_char_p
    _lib = lib
    return lib


def _dp(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def _fortran(a, dtype) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=dtype))


class Engine:
    """One device context (one CUDA stream).  Not thread-safe."""

    def __init__(self, device: int = 0, precision: str = "fp64", seed: int = 0x1234ABCD):
        self.lib = load_library()
        h = ct.c_void_p()
        st = self.lib.ipeps_ctx_create(int(device), ct.byref(h))
        if st != OK:
            raise IPEPSError(st, f"ipeps_ctx_create(device={device}) failed")
        self.h = h
        self.set_precision(precision)
        self.check(self.lib.ipeps_ctx_set_seed(self.h, ct.c_uint64(seed)))

    def check(self, st: int):
        if st != OK:
            msg = self.lib.ipeps_last_error(self.h)
            raise IPEPSError(st, msg.decode() if msg else "")

    def set_precision(self, precision: str):
        p = {"fp64": PREC_FP64, "mixed": PREC_MIXED}[precision]
        self.precision = precision
        self.check(self.lib.ipeps_ctx_set_precision(self.h, p))

    def stats(self) -> Dict[str, Any]:
        s = Stats()
        self.check(self.lib.ipeps_stats(self.h, ct.byref(s)))
        return s.as_dict()

    def stream_ptr(self) -> int:
        """The engine's cudaStream_t as an int (for torch.cuda.ExternalStream)."""
        p = ct.c_void_p()
        self.check(self.lib.ipeps_ctx_stream(self.h, ct.byref(p)))
        return int(p.value or 0)

    def prof_enable(self, on: bool = True):
        self.check(self.lib.ipeps_prof_enable(self.h, int(on)))

    def prof_phases(self) -> Dict[str, float]:
        """Wall ms of the pullback's phases while profiling (then cleared)."""
        ms = np.zeros(5)
        self.check(self.lib.ipeps_prof_phases(self.h, _dp(ms)))
        return dict(zip(["checkpoint_iterations", "energy_tape", "recompute_on_tapes", "backward",
                         "projector_adjoints_in_backward"], [float(x) for x in ms]))

    def prof_query(self) -> Dict[str, Dict[str, float]]:
        ms = np.zeros(8)
        fl = np.zeros(8)
        by = np.zeros(8)
        la = (ct.c_uint64 * 8)()
        self.check(self.lib.ipeps_prof_query(self.h, _dp(ms), la, _dp(fl), _dp(by)))
        return {n: {"ms": float(ms[i]), "launches": int(la[i]), "flops": float(fl[i]), "bytes": float(by[i])}
                for i, n in enumerate(Stats.FAMILIES)}

    def reset_stats(self):
        self.check(self.lib.ipeps_stats_reset(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.ipeps_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_engine: Optional[Engine] = None


def default_engine() -> Engine:
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine(int(os.environ.get("IPEPS_DEVICE", "0")))
    return _default_engine


def default_config() -> Dict[str, Any]:
    """src/optimize/default_config.toml:1-49 (keys the hot path reads)."""
    return {"gc": True, "dir": 0, "out_prefix": "test", "model": "test", "D": 2, "chi": 32,
            "min_iter": 4, "max_iter": 20, "ad_max_iter": 4, "rg_tol": 1e-6, "resume": False,
            "basis": False, "basis_t": "default", "basis_cut": 1e-3, "basis_name": 0,
            "es_resume": 1, "es_num": 0, "ad": True, "save": True, "part_save": False,
            "nrmB_cut": 1e-3, "wp": 1}


def load_config(filename: Optional[str] = None) -> Dict[str, Any]:
    """The config dict of optim_gs / prepare_basis / optim_es (optim_gs.jl:1-12,
    optim_es.jl:22-32): TOML.parsefile(filename) when the file exists, else the
    reference's default config.  Keys absent from the file are not added (as
    TOML.parsefile), so a custom file must carry what the run reads."""
    if filename and os.path.isfile(filename):
        import tomllib
        with open(filename, "rb") as f:
            return tomllib.load(f)
    return default_config()


def get_dir(params: Dict[str, Any], cwd: Optional[str] = None) -> str:
    """get_dir (src/utility/io.jl:72-90): simulation/$(model)_$(out_prefix)_D$(D)_X$(chi)
    under the working directory when dir == 0, else params["dir"] (not created here)."""
    if params.get("dir", 0) == 0:
        return os.path.join(cwd or os.getcwd(), "simulation", "%s_%s_D%s_X%s" % (
            params.get("model", "none"), params.get("out_prefix", "none"), params.get("D", "none"),
            params.get("chi", "none")))
    return str(params["dir"])


def get_gs_name(params: Dict[str, Any], cwd: Optional[str] = None) -> str:
    """get_gs_name (src/utility/io.jl:1-6)"""
    return os.path.join(get_dir(params, cwd), "gs.jld2")


def get_basis_name(params: Dict[str, Any], cwd: Optional[str] = None) -> str:
    """get_basis_name (src/utility/io.jl:8-18)"""
    name = params.get("basis_name", 0)
    return os.path.join(get_dir(params, cwd), "basis.jld2" if name == 0 else f"{name}.jld2")


def _jl_num(x) -> str:
    """Julia's string() of a momentum: 0.1 -> "0.1", 1.0 -> "1.0", 1 -> "1"."""
    return repr(x) if isinstance(x, float) else str(x)


def get_es_name(params: Dict[str, Any], px, py, cwd: Optional[str] = None) -> str:
    """get_es_name (src/utility/io.jl:20-40) for the whole-momentum file
    (part_save = false): es_$(px)_$(py).jld2"""
    return os.path.join(get_dir(params, cwd), f"es_{_jl_num(px)}_{_jl_num(py)}.jld2")


def _H_pair(H):
    hs = [_fortran(h, np.complex128) for h in H]
    d2 = hs[0].shape[0]
    return hs[0], hs[1], d2


class CTMTensors:
    """Environment state on the device (ctm_tensor.jl:3-18).

    ``CTMTensors(A, cfg)`` sets Ad = conj(A) and runs init_ctm1, like the
    reference constructor.  The Params dict is ``self.Params``; keys chi,
    min_iter, max_iter, ad_max_iter, rg_tol are pushed to the device before
    every run/step.  Extra keys (not read by the reference): ``svd_oversample``
    (num, den, min), ``svd_power_iters`` (cold, warm), ``svd_warm_start``,
    ``parallel_moves`` (left || right and top || bottom on two streams).
    """

    def __init__(self, A, cfg: Optional[Dict[str, Any]] = None, Ad=None, engine: Optional[Engine] = None,
                 init: bool = True):
        self.engine = engine or default_engine()
        self.lib = self.engine.lib
        A = np.asarray(A)
        self.is_complex = np.iscomplexobj(A) or (Ad is not None and np.iscomplexobj(Ad))
        self.dtype = np.complex128 if self.is_complex else np.float64
        self.D, self.d = int(A.shape[0]), int(A.shape[4])
        self.Params = dict(default_config() if cfg is None else cfg)
        h = ct.c_void_p()
        self.engine.check(self.lib.ipeps_env_create(self.engine.h, self.D, self.d, int(self.Params.get("chi", 30)),
                                                    int(self.is_complex), ct.byref(h)))
        self.h = h
        self._push_params()
        self.set_A(A, Ad)
        if init:
            self.engine.check(self.lib.ipeps_env_init(self.h))
        self.B = None

    # -------------------------------------------------------------- state
    def set_A(self, A, Ad=None):
        self._A = _fortran(A, self.dtype)
        self._Ad = None if Ad is None else _fortran(Ad, self.dtype)
        self.engine.check(self.lib.ipeps_env_set_A(self.h, _dp(self._A), _dp(self._Ad)))

    @property
    def A(self):
        return self._A

    @property
    def Ad(self):
        return np.conj(self._A) if self._Ad is None else self._Ad

    def _push_params(self):
        p = self.Params
        self.engine.check(self.lib.ipeps_env_set_params(
            self.h, int(p.get("chi", 30)), int(p.get("min_iter", 4)), int(p.get("max_iter", 20)),
            int(p.get("ad_max_iter", 4)), float(p.get("rg_tol", 1e-6))))
        over = p.get("svd_oversample", (1, 1, 16))
        pit = p.get("svd_power_iters", (3, 2))
        self.engine.check(self.lib.ipeps_env_set_svd_params(
            self.h, int(over[0]), int(over[1]), int(over[2]), int(pit[0]), int(pit[1]),
            int(bool(p.get("svd_warm_start", True))), float(p.get("svd_resid_tol", 1e-10)),
            int(p.get("svd_max_extra", 6)), int(p.get("svd_inter_passes", 1)),
            int(bool(p.get("svd_seed_older", True)))))
        self.engine.check(self.lib.ipeps_env_set_parallel(self.h, int(bool(p.get("parallel_moves", True)))))
        self.engine.check(self.lib.ipeps_env_set_mixed(
            self.h, int(p.get("mixed_polish_iters", 4)), float(p.get("mixed_polish_tol", 100.0))))

    def get_CT(self, k: int):
        """(C_k, E_k) as column-major numpy arrays, k = 1..4."""
        cd = (ct.c_int64 * 2)()
        ed = (ct.c_int64 * 4)()
        self.engine.check(self.lib.ipeps_env_get_CT(self.h, k, None, cd, None, ed))
        C = np.empty(tuple(cd), dtype=self.dtype, order="F")
        E = np.empty(tuple(ed), dtype=self.dtype, order="F")
        self.engine.check(self.lib.ipeps_env_get_CT(self.h, k, _dp(C), cd, _dp(E), ed))
        return C, E

    def set_CT(self, k: int, C, E):
        C = _fortran(C, self.dtype)
        E = _fortran(E, self.dtype)
        cd = (ct.c_int64 * 2)(*C.shape)
        ed = (ct.c_int64 * 4)(*E.shape)
        self.engine.check(self.lib.ipeps_env_set_CT(self.h, k, _dp(C), cd, _dp(E), ed))

    @property
    def Cs(self):
        return [self.get_CT(k)[0] for k in range(1, 5)]

    @property
    def Es(self):
        return [self.get_CT(k)[1] for k in range(1, 5)]

    def set_B(self, B, px: float, py: float):
        """setproperties(ts, B=B, Bd=conj(B)) with Params px, py (optim_es.jl:124-125,171)."""
        self.B = _fortran(B, np.complex128)
        self.Params["px"], self.Params["py"] = float(px), float(py)
        self.engine.check(self.lib.ipeps_nested_set_B(self.h, _dp(self.B), float(px), float(py)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.ipeps_env_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tcon(xs, ind_xs, engine: Optional[Engine] = None):
    """``tcon(xs, ind_xs)`` (wrapper.jl:15-23) on the device: positive labels
    are summed, negative labels -1, -2, ... give the output order."""
    eng = engine or default_engine()
    A, B = xs
    la, lb = ind_xs
    cplx = np.iscomplexobj(A) or np.iscomplexobj(B)
    dt = np.complex128 if cplx else np.float64
    A = _fortran(A, dt)
    B = _fortran(B, dt)
    ext = {}
    for l, n in zip(la, A.shape):
        ext[l] = n
    for l, n in zip(lb, B.shape):
        ext[l] = n
    nout = sum(1 for l in list(la) + list(lb) if l < 0)
    oshape = tuple(ext[-(i + 1)] for i in range(nout))
    out = np.empty(oshape, dtype=dt, order="F")
    od = (ct.c_int64 * 16)()
    ond = ct.c_int(0)
    dA = (ct.c_int64 * max(1, A.ndim))(*A.shape)
    dB = (ct.c_int64 * max(1, B.ndim))(*B.shape)
    lA = (ct.c_int * max(1, len(la)))(*la)
    lB = (ct.c_int * max(1, len(lb)))(*lb)
    eng.check(eng.lib.ipeps_tcon(eng.h, int(cplx), _dp(A), A.ndim, dA, lA, _dp(B), B.ndim, dB, lB, _dp(out),
                                 int(max(out.size, 1)), od, ct.byref(ond)))
    return out


def get_projector(R1, R2, chi: int, engine: Optional[Engine] = None):
    """get_projector(R1, R2, chi) (ctmrg.jl:254-265) on the device: (P1, P2, S)."""
    eng = engine or default_engine()
    cplx = np.iscomplexobj(R1) or np.iscomplexobj(R2)
    dt = np.complex128 if cplx else np.float64
    R1 = _fortran(R1, dt)
    R2 = _fortran(R2, dt)
    N1, K1 = R1.shape
    K1b, N2 = R2.shape
    if K1b != K1:
        raise ValueError("get_projector: inner dimensions of R1 * R2 differ")
    P1 = np.empty(K1 * (chi + 1), dtype=dt)
    P2 = np.empty(K1 * (chi + 1), dtype=dt)
    s = np.empty(chi + 1)
    n = ct.c_int(0)
    fn = eng.lib.ipeps_projector_c if cplx else eng.lib.ipeps_projector
    eng.check(fn(eng.h, _dp(R1), _dp(R2), N1, K1, N2, int(chi), _dp(P1), _dp(P2), _dp(s), ct.byref(n)))
    k = n.value
    return (P1[: K1 * k].reshape((K1, k), order="F"), P2[: K1 * k].reshape((k, K1), order="F"), s[:k].copy())


# ------------------------------------------------------------------ moves
def _spectrum_call(ts, fn, *args):
    n = ct.c_int(4096)
    buf = np.empty(4096, dtype=np.float64)
    ts.engine.check(fn(ts.h, *args, _dp(buf), ct.byref(n)))
    return buf[: n.value].copy()


def rg_step(ts: CTMTensors, chi: Optional[int] = None):
    """ctmrg.jl:57-64: returns (ts, s) with s the left-move spectrum."""
    if chi is not None:
        ts.Params["chi"] = int(chi)
    ts._push_params()
    return ts, _spectrum_call(ts, ts.lib.ipeps_ctm_step)


def _move(ts, chi, d):
    if chi is not None:
        ts.Params["chi"] = int(chi)
    ts._push_params()
    return ts, _spectrum_call(ts, ts.lib.ipeps_ctm_move, d)


def left_rg(ts, chi=None):
    """ctmrg.jl:66-78"""
    return _move(ts, chi, 0)


def right_rg(ts, chi=None):
    """ctmrg.jl:80-92"""
    return _move(ts, chi, 1)


def top_rg(ts, chi=None):
    """ctmrg.jl:94-106"""
    return _move(ts, chi, 2)


def bottom_rg(ts, chi=None):
    """ctmrg.jl:108-120"""
    return _move(ts, chi, 3)


class _H4:
    """The plaquette MPO [s1, s2, s3, s4] (get_local_h) as C-ABI tensors; keeps
    the column-major complex copies alive for the duration of a call."""

    def __init__(self, H4):
        if len(H4) != 4:
            raise ValueError("the plaquette Hamiltonian is the MPO list [s1, s2, s3, s4]")
        self.arrs = [_fortran(h, np.complex128) for h in H4]
        self.c = (CTensor * 4)()
        for k, a in enumerate(self.arrs):
            self.c[k].data = a.ctypes.data
            self.c[k].nd = a.ndim
            for i, d in enumerate(a.shape):
                self.c[k].dims[i] = d


def get_gs_energy_4x4(ts: CTMTensors, H4) -> complex:
    """get_gs_energy_4x4 (evaluation.jl:339-356): plaquette energy of the 2 x 2 cluster."""
    h = _H4(H4)
    out = np.zeros(2)
    ts.engine.check(ts.lib.ipeps_energy_4x4(ts.h, h.c, 0, _dp(out)))
    return complex(out[0], out[1])


def get_es_energy_4x4(ts: CTMTensors, H4) -> complex:
    """get_es_energy_4x4 (evaluation.jl:358-398): nested plaquette energy (B set)."""
    h = _H4(H4)
    out = np.zeros(2)
    ts.engine.check(ts.lib.ipeps_energy_4x4(ts.h, h.c, 1, _dp(out)))
    return complex(out[0], out[1])


def run_ctm_4x4(ts: CTMTensors, H4, nested: bool = False):
    """run_ctm with conv_fun = get_gs_energy_4x4 (nested False) or
    get_es_energy_4x4 / get_all_norm (nested True) (optim_es_h4.jl:33,139).
    Returns (ts, info) as run_ctm."""
    ts._push_params()
    h = _H4(H4)
    iters, conv = ct.c_int(0), ct.c_int(0)
    diff = ct.c_double(0)
    ts.engine.check(ts.lib.ipeps_ctm_run_4x4(ts.h, h.c, int(bool(nested)), ct.byref(iters), ct.byref(diff),
                                             ct.byref(conv)))
    return ts, _run_info(ts, iters, diff, conv)


def energy_grad_4x4(ts: CTMTensors, H4, ad_iters: Optional[int] = None):
    """Pullback of run_gs_h4 (optim_gs_h4.jl:113-123) from the environment held
    by ts: returns (real(E), dE/dA) with dE/dA a real (D,D,D,D,d) array."""
    h = _H4(H4)
    n = int(ts.Params.get("ad_max_iter", 4) if ad_iters is None else ad_iters)
    ts._push_params()
    E = np.zeros(1)
    g = np.empty(ts.A.shape, dtype=np.float64, order="F")
    ts.engine.check(ts.lib.ipeps_energy_grad_4x4(ts.h, h.c, n, _dp(E), _dp(g)))
    return float(E[0]), g


def fg_h4(x, H4, cfg, engine: Optional[Engine] = None):
    """E+grad unit of optim_gs_h4 (fg!, optim_gs_h4.jl:53-91): x renormalised
    (max-abs), CTMRG converged from init_ctm1 with the plaquette energy
    (get_conv_boundary_h4), then the pullback of ad_max_iter iterations.
    H4 is the MPO [s1, s2, s3, s4] of get_local_h.  Returns (E, g, info)."""
    x = np.asarray(x, dtype=np.float64)
    x = x / np.abs(x).max()
    ts = CTMTensors(x, cfg, engine=engine)
    ts, info = run_ctm_4x4(ts, H4, nested=False)
    E, g = energy_grad_4x4(ts, H4)
    ts.close()
    return E, g, info


def es_energy_grad_4x4(ts: CTMTensors, H4, ad_iters: Optional[int] = None):
    """Pullback of run_es_h4 (optim_es_h4.jl:159-168) w.r.t. B from the nested
    environment held by ts: returns (E, gH), gH complex (D,D,D,D,d)."""
    h = _H4(H4)
    n = int(ts.Params.get("ad_max_iter", 4) if ad_iters is None else ad_iters)
    ts._push_params()
    E = np.zeros(1)
    g = np.empty(ts.A.shape, dtype=np.complex128, order="F")
    ts.engine.check(ts.lib.ipeps_es_energy_grad_4x4(ts.h, h.c, n, _dp(E), _dp(g)))
    return float(E[0]), g


def get_es_grad_h4(ts: CTMTensors, H4, Bi):
    """get_es_grad_h4 (optim_es_h4.jl:133-157) on the device; as get_es_grad
    with the plaquette energy.  Returns (gH, gN) flat complex (column-major)."""
    B = np.asarray(Bi, dtype=np.complex128).reshape(ts.A.shape, order="F")
    ts.set_B(B, ts.Params.get("px", 0.0), ts.Params.get("py", 0.0))
    run_ctm_4x4(ts, H4, nested=True)
    E, gH = es_energy_grad_4x4(ts, H4)
    Nb, gN = get_all_norm(ts)
    return gH.reshape(-1, order="F"), gN.reshape(-1, order="F")


def get_wp_grad(ts: CTMTensors, wp4, Bi, site: Optional[int] = None):
    """get_wp_grad (optim_wp.jl:195-220) on the device, in the environment held
    by ts (no CTMRG): the basis tensor Bi at plaquette site ``site`` (default
    ts.Params["wp"], else 1), the plaquette operator as the MPO wp4 = [s1, s2,
    s3, s4] (get_local_h of the operator).  Returns (gH, gN) flat complex
    (column-major) and the operator value and norm (run_wp, :222-238)."""
    site = int(ts.Params.get("wp", 1) if site is None else site)
    h = _H4(wp4)
    B = np.asarray(Bi, dtype=np.complex128).reshape(ts.A.shape, order="F").copy(order="F")
    out = np.zeros(4)
    gH = np.empty(ts.A.shape, dtype=np.complex128, order="F")
    gN = np.empty(ts.A.shape, dtype=np.complex128, order="F")
    ts.engine.check(ts.lib.ipeps_wp_grad(ts.h, h.c, site, _dp(B), _dp(out), _dp(gH), _dp(gN)))
    return gH.reshape(-1, order="F"), gN.reshape(-1, order="F"), complex(out[0], out[1]), complex(out[2], out[3])


def _run_info(ts, iters, diff, conv):
    n = ct.c_int(100000)
    log = np.empty((100000, 4))
    ts.engine.check(ts.lib.ipeps_ctm_log(ts.h, _dp(log), ct.byref(n)))
    return {"iters": iters.value, "diff": diff.value, "converged": bool(conv.value),
            "log": [{"iter": i + 1, "diff": float(r[0]), "obj": complex(r[1], r[2]), "chi": int(r[3])}
                    for i, r in enumerate(log[: n.value])]}


def run_ctm(ts: CTMTensors, conv_fun: Optional[str] = None, H=None):
    """ctmrg.jl:1-55.

    ``conv_fun`` selects the reference's convergence criterion: None (left
    spectrum), "energy" (get_gs_energy, as in optim_gs / compute_gs_energy) or
    "es" (get_es_energy / get_all_norm, as in optim_es).  Returns (ts, info)
    with info = {"iters", "diff", "converged", "log"}.
    """
    ts._push_params()
    mode = {None: CONV_SPECTRUM, "spectrum": CONV_SPECTRUM, "energy": CONV_ENERGY, "es": CONV_ES}[conv_fun]
    if mode != CONV_SPECTRUM:
        Hh, Hv, d2 = _H_pair(H)
    else:
        Hh = Hv = None
        d2 = 0
    iters, conv = ct.c_int(0), ct.c_int(0)
    diff = ct.c_double(0)
    ts.engine.check(ts.lib.ipeps_ctm_run(ts.h, mode, _dp(Hh), _dp(Hv), d2, ct.byref(iters), ct.byref(diff),
                                         ct.byref(conv)))
    n = ct.c_int(100000)
    log = np.empty((100000, 4))
    ts.engine.check(ts.lib.ipeps_ctm_log(ts.h, _dp(log), ct.byref(n)))
    info = {"iters": iters.value, "diff": diff.value, "converged": bool(conv.value),
            "log": [{"iter": i + 1, "diff": float(r[0]), "obj": complex(r[1], r[2]), "chi": int(r[3])}
                    for i, r in enumerate(log[: n.value])]}
    return ts, info


# ------------------------------------------------------------ observables
def get_gs_energy(ts: CTMTensors, H):
    """evaluation.jl:15-29: returns (E, Na) as complex numbers."""
    Hh, Hv, d2 = _H_pair(H)
    E = np.zeros(2)
    Na = np.zeros(2)
    ts.engine.check(ts.lib.ipeps_energy(ts.h, _dp(Hh), _dp(Hv), d2, _dp(E), _dp(Na)))
    return complex(E[0], E[1]), complex(Na[0], Na[1])


def get_gs_norm(ts: CTMTensors):
    """evaluation.jl:47-59"""
    out = np.zeros(2)
    ts.engine.check(ts.lib.ipeps_gs_norm(ts.h, _dp(out)))
    return complex(out[0], out[1])


def single_dm_Ad(ts: CTMTensors) -> np.ndarray:
    """ndm_Ad of get_tangent_basis (optim_es.jl:247-251)."""
    out = np.empty(ts.A.shape, dtype=ts.dtype, order="F")
    ts.engine.check(ts.lib.ipeps_single_dm_Ad(ts.h, _dp(out)))
    return out


def get_es_energy(ts: CTMTensors, H) -> float:
    """evaluation.jl:31-45"""
    Hh, Hv, d2 = _H_pair(H)
    out = np.zeros(1)
    ts.engine.check(ts.lib.ipeps_es_energy(ts.h, _dp(Hh), _dp(Hv), d2, _dp(out)))
    return float(out[0])


def get_all_norm(ts: CTMTensors):
    """evaluation.jl:61-77: returns (Nb, envB)."""
    nb = np.zeros(2)
    envB = np.empty(ts.A.shape, dtype=np.complex128, order="F")
    ts.engine.check(ts.lib.ipeps_all_norm(ts.h, _dp(nb), _dp(envB)))
    return complex(nb[0], nb[1]), envB


def energy_grad(ts: CTMTensors, H, ad_iters: Optional[int] = None):
    """Pullback of run_gs (optim_gs.jl:133-143) from the environment held by ts:
    returns (real(E), dE/dA) with dE/dA a real (D,D,D,D,d) array."""
    Hh, Hv, d2 = _H_pair(H)
    n = int(ts.Params.get("ad_max_iter", 4) if ad_iters is None else ad_iters)
    ts._push_params()
    E = np.zeros(1)
    g = np.empty(ts.A.shape, dtype=np.float64, order="F")
    ts.engine.check(ts.lib.ipeps_energy_grad(ts.h, _dp(Hh), _dp(Hv), d2, n, _dp(E), _dp(g)))
    return float(E[0]), g


def fg(x, H, cfg, engine: Optional[Engine] = None):
    """E+grad unit of optim_gs (fg!, optim_gs.jl:53-91): x is renormalised
    (max-abs), CTMRG converges from init_ctm1 with the energy criterion
    (get_conv_boundary, :120-131), then the pullback of ad_max_iter further
    iterations + get_gs_energy gives (E, dE/dx).  Returns (E, g, info)."""
    x = np.asarray(x, dtype=np.float64)
    x = x / np.abs(x).max()
    ts = CTMTensors(x, cfg, engine=engine)
    ts, info = run_ctm(ts, conv_fun="energy", H=H)
    E, g = energy_grad(ts, H)
    ts.close()
    return E, g, info


def es_energy_grad(ts: CTMTensors, H, ad_iters: Optional[int] = None):
    """Pullback of run_es (optim_es.jl:196-210) w.r.t. B from the nested
    environment held by ts: returns (E, gH) with gH complex (D,D,D,D,d)."""
    Hh, Hv, d2 = _H_pair(H)
    n = int(ts.Params.get("ad_max_iter", 4) if ad_iters is None else ad_iters)
    ts._push_params()
    E = np.zeros(1)
    g = np.empty(ts.A.shape, dtype=np.complex128, order="F")
    ts.engine.check(ts.lib.ipeps_es_energy_grad(ts.h, _dp(Hh), _dp(Hv), d2, n, _dp(E), _dp(g)))
    return float(E[0]), g


def get_es_grad(ts: CTMTensors, H, Bi):
    """get_es_grad (optim_es.jl:167-194) on the device.

    ts holds the (normalised) ground-state environment; it is modified in
    place (B set, nested iterations run).  Returns (gH, gN) as flat complex
    vectors in column-major order, gN = envB of get_all_norm after the
    pullback iterations (optim_es.jl:189)."""
    B = np.asarray(Bi, dtype=np.complex128).reshape(ts.A.shape, order="F")
    ts.set_B(B, ts.Params.get("px", 0.0), ts.Params.get("py", 0.0))
    run_ctm(ts, conv_fun="es", H=H)
    E, gH = es_energy_grad(ts, H)
    Nb, gN = get_all_norm(ts)
    return gH.reshape(-1, order="F"), gN.reshape(-1, order="F")


def compute_gs_energy(A, H, cfg, engine: Optional[Engine] = None):
    """evaluation.jl:1-13: converge from init_ctm1 with the energy criterion."""
    ts = CTMTensors(A, cfg, engine=engine)
    ts, info = run_ctm(ts, conv_fun="energy", H=H)
    E, Na = get_gs_energy(ts, H)
    return (E, Na), ts, info


# ------------------------------------------------------------ warm-start network
def _fp(a: np.ndarray):
    return a.ctypes.data_as(ct.POINTER(ct.c_float))


def _f32(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.float32))


def gemm_f64(opA: str, opB: str, A, B, alpha: float = 1.0, beta: float = 0.0, C=None,
             engine: Optional[Engine] = None, reps: int = 1) -> np.ndarray:
    """C = alpha op(A) op(B) + beta C on the engine's FP64 (DMMA) GEMM; host arrays."""
    eng = engine or default_engine()
    A = _fortran(A, np.float64)
    B = _fortran(B, np.float64)
    m = A.shape[0] if opA == "N" else A.shape[1]
    k = A.shape[1] if opA == "N" else A.shape[0]
    n = B.shape[1] if opB == "N" else B.shape[0]
    C = np.zeros((m, n), order="F") if C is None else _fortran(C, np.float64).copy(order="F")
    eng.check(eng.lib.ipeps_gemm_f64(eng.h, opA.encode(), opB.encode(), m, n, k, float(alpha), _dp(A), A.shape[0],
                                     _dp(B), B.shape[0], float(beta), _dp(C), C.shape[0], int(reps)))
    return C


def orth(Y, passes: int = 3, engine: Optional[Engine] = None):
    """Orthonormal basis of range(Y) by the projector's CholeskyQR (first pass
    shifted; passes = 3 is sCholQR3): returns (Q, R) with Q^T Q = I, Q R = Y."""
    eng = engine or default_engine()
    Y = _fortran(Y, np.float64)
    N, k = Y.shape
    Q = np.empty((N, k), order="F")
    R = np.empty((k, k), order="F")
    eng.check(eng.lib.ipeps_orth(eng.h, _dp(Y), N, k, int(passes), _dp(Q), _dp(R)))
    return Q, R


def gemm_tf32x3(opA: str, opB: str, A, B, alpha: float = 1.0, beta: float = 0.0, C=None,
                engine: Optional[Engine] = None, reps: int = 1, timing: bool = False):
    """C = alpha op(A) op(B) + beta C on the engine's 3xTF32 tcgen05 GEMM; host
    arrays.  With timing=True returns (C, device ms of one product)."""
    eng = engine or default_engine()
    A = _fortran(A, np.float64)
    B = _fortran(B, np.float64)
    m = A.shape[0] if opA == "N" else A.shape[1]
    k = A.shape[1] if opA == "N" else A.shape[0]
    n = B.shape[1] if opB == "N" else B.shape[0]
    C = np.zeros((m, n), order="F") if C is None else _fortran(C, np.float64).copy(order="F")
    ms = np.zeros(1)
    eng.check(eng.lib.ipeps_gemm_tf32x3(eng.h, opA.encode(), opB.encode(), m, n, k, float(alpha), _dp(A),
                                        A.shape[0], _dp(B), B.shape[0], float(beta), _dp(C), C.shape[0], int(reps),
                                        _dp(ms)))
    return (C, float(ms[0])) if timing else C


def gemm_bf16(opA: str, opB: str, A, B, alpha: float = 1.0, beta: float = 0.0, C=None,
              engine: Optional[Engine] = None) -> np.ndarray:
    """C = alpha op(A) op(B) + beta C on the BF16 tensor-core GEMM (host buffers, float32)."""
    eng = engine or default_engine()
    A, B = _f32(A), _f32(B)
    m = A.shape[0] if opA == "N" else A.shape[1]
    k = A.shape[1] if opA == "N" else A.shape[0]
    n = B.shape[1] if opB == "N" else B.shape[0]
    C = np.zeros((m, n), dtype=np.float32, order="F") if C is None else _f32(C).copy(order="F")
    eng.check(eng.lib.ipeps_gemm_bf16(eng.h, opA.encode(), opB.encode(), m, n, k, float(alpha), _fp(A), A.shape[0],
                                      _fp(B), B.shape[0], float(beta), _fp(C), m))
    return C


class Mlp:
    """The warm-start network on the device (ipeps_mlp_*): n_in -> n_hidden ->
    n_hidden -> n_out with GELU, BF16 tensor-core GEMMs, FP32 parameters, Adam."""

    def __init__(self, n_in: int, n_hidden: int, n_out: int, max_batch: int = 256, seed: int = 0,
                 engine: Optional[Engine] = None):
        self.engine = engine or default_engine()
        self.lib = self.engine.lib
        self.n_in, self.n_hidden, self.n_out, self.max_batch = n_in, n_hidden, n_out, max_batch
        h = ct.c_void_p()
        self.engine.check(self.lib.ipeps_mlp_create(self.engine.h, n_in, n_hidden, n_out, max_batch, seed,
                                                    ct.byref(h)))
        self.h = h
        n = ct.c_int64(0)
        self.lib.ipeps_mlp_num_params(self.h, ct.byref(n))
        self.num_params = n.value

    def params(self) -> np.ndarray:
        p = np.empty(self.num_params, dtype=np.float32)
        self.engine.check(self.lib.ipeps_mlp_get_params(self.h, _fp(p)))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.num_params
        self.engine.check(self.lib.ipeps_mlp_set_params(self.h, _fp(p)))

    def forward(self, X) -> np.ndarray:
        X = _f32(X)
        Y = np.empty((X.shape[0], self.n_out), dtype=np.float32, order="F")
        self.engine.check(self.lib.ipeps_mlp_forward(self.h, _fp(X), X.shape[0], _fp(Y)))
        return Y

    def grad(self, X, T):
        X, T = _f32(X), _f32(T)
        g = np.empty(self.num_params, dtype=np.float32)
        loss = ct.c_double(0)
        self.engine.check(self.lib.ipeps_mlp_grad(self.h, _fp(X), _fp(T), X.shape[0], ct.byref(loss), _fp(g)))
        return loss.value, g

    def train_step(self, X, T, lr: float) -> float:
        X, T = _f32(X), _f32(T)
        loss = ct.c_double(0)
        self.engine.check(self.lib.ipeps_mlp_train_step(self.h, _fp(X), _fp(T), X.shape[0], float(lr),
                                                        ct.byref(loss)))
        return loss.value

    def close(self):
        if getattr(self, "h", None):
            if getattr(self.engine, "h", None):  # a closed engine took the device state with it
                self.lib.ipeps_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

