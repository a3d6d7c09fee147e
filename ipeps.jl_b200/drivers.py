"""Host drivers above the engine: optim_gs, prepare_basis, optim_es, evaluate_es.

These stay on the host in the reference too (Julia + Optim.jl + LAPACK on
small matrices); only their calls into CTMRG go to the device.

    optim_gs(H, A0, cfg)        src/optimize/optim_gs.jl:14-118 (L-BFGS on the sphere)
    prepare_basis(H, A, cfg)    src/optimize/optim_es.jl:34-73
    optim_es(px, py, prep, cfg) src/optimize/optim_es.jl:91-165
    evaluate_es(effH, effN)     src/graph/expectation.jl:152-183 (band_energies: its real parts)
    prepare_basis_h4 / optim_es_h4 (the plaquette Hamiltonian)
                                src/optimize/optim_es_h4.jl

The L-BFGS is a plain two-loop recursion with the sphere manifold of
Optim.jl (gradient projected onto the tangent space, iterate retracted by
normalisation) and a backtracking Armijo line search; the reference uses
Optim's HagerZhang line search, so trajectories differ and only final energies
are compared.
"""
from __future__ import annotations

import math
import os
from typing import Any, Callable, Dict, List, Optional

import numpy as np

from . import host


def _sphere_project(x, g):
    return g - np.vdot(x, g).real * x


def load_gs(path: str) -> Dict[str, Any]:
    """A ground-state checkpoint: the reference's gs.jld2 (A, energies,
    gradnorms; optim_gs.jl:36) or this package's gs.npz (the same keys)."""
    if path.endswith(".jld2"):
        from . import jld2
        d = jld2.load(path)
    else:
        d = dict(np.load(path))
    return {"A": np.asarray(d["A"]), "energies": list(np.atleast_1d(d.get("energies", []))),
            "gradnorms": list(np.atleast_1d(d.get("gradnorms", [])))}


def _save_gs(path: str, A, energies, gradnorms):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, A=A, energies=np.asarray(energies), gradnorms=np.asarray(gradnorms))


def optim_gs(H, A0, cfg, m: int = 10, g_tol: float = 1e-6, f_tol: float = 1e-7,
             iterations: int = 200, engine: Optional[host.Engine] = None,
             callback: Optional[Callable[[int, float, float], None]] = None,
             fg_fn: Optional[Callable] = None, save_dir: Optional[str] = None):
    """L-BFGS over A on the unit sphere with the device E+grad unit (fg!).

    cfg: a config dict, or a TOML file name (optim_gs.jl:1-12; the default
    config when the file does not exist).  With cfg["resume"] and a checkpoint
    in the run directory (get_dir: the reference's gs.jld2, or gs.npz), the
    run restarts from its A and continues its energy/gradnorm lists
    (optim_gs.jl:47-53).  With cfg["save"] and an explicit directory (save_dir,
    or cfg["dir"] != 0) A, energies and gradnorms are written to gs.npz there
    after every step (the reference writes gs.jld2; nothing is written under
    the working directory by default).
    ``fg_fn(A, H, cfg, engine=...) -> (E, g, info)`` replaces host.fg (e.g. the
    warm-started unit of warmstart.WarmStart.fg).  Returns dict(A, energies,
    gradnorms, evals)."""
    if isinstance(cfg, str):
        cfg = host.load_config(cfg)
    run_dir = save_dir or host.get_dir(cfg)
    prev_E: List[float] = []
    prev_g: List[float] = []
    if cfg.get("resume", False):
        for name in ("gs.npz", "gs.jld2"):
            path = os.path.join(run_dir, name)
            if os.path.exists(path):
                ck = load_gs(path)
                A0, prev_E, prev_g = ck["A"], ck["energies"], ck["gradnorms"]
                break
    if np.iscomplexobj(A0):
        raise ValueError("optim_gs: complex A has no device gradient (real A only)")
    x = np.asarray(A0, dtype=np.float64).ravel(order="F")
    shape = np.asarray(A0).shape
    x = x / np.linalg.norm(x)
    evals = 0

    def fg(xv):
        nonlocal evals
        evals += 1
        A = xv.reshape(shape, order="F")
        # fg! renormalises x by max|x| before the energy (optim_gs.jl:55); the
        # energy is scale invariant, the gradient scales by max|x|
        s = np.abs(A).max()
        E, g, _ = (fg_fn or host.fg)(A, H, cfg, engine=engine)
        return E, g.ravel(order="F") / s

    f, g = fg(x)
    gp = _sphere_project(x, g)
    energies, gradnorms = prev_E + [f], prev_g + [float(np.linalg.norm(gp))]
    save = bool(cfg.get("save", False)) and (save_dir is not None or cfg.get("dir", 0) != 0)
    S: List[np.ndarray] = []
    Y: List[np.ndarray] = []
    for it in range(iterations):
        if np.linalg.norm(gp) < g_tol:
            break
        # two-loop recursion on the tangent space
        q = gp.copy()
        alphas = []
        for s_, y_ in reversed(list(zip(S, Y))):
            rho = 1.0 / np.dot(y_, s_)
            a = rho * np.dot(s_, q)
            alphas.append((a, rho, s_, y_))
            q -= a * y_
        if S:
            q *= np.dot(S[-1], Y[-1]) / np.dot(Y[-1], Y[-1])
        else:
            q *= 0.1 / max(np.linalg.norm(q), 1e-300)
        for a, rho, s_, y_ in reversed(alphas):
            b = rho * np.dot(y_, q)
            q += (a - b) * s_
        d = -_sphere_project(x, q)
        if np.dot(d, gp) >= 0:
            d = -gp
        # backtracking Armijo on the retraction x -> (x + t d)/|x + t d|
        t = 1.0
        slope = np.dot(d, gp)
        while True:
            xn = x + t * d
            xn /= np.linalg.norm(xn)
            fn, gn = fg(xn)
            if fn <= f + 1e-4 * t * slope or t < 1e-8:
                break
            t *= 0.5
        gpn = _sphere_project(xn, gn)
        s_vec = xn - x
        y_vec = gpn - gp
        if np.dot(s_vec, y_vec) > 1e-16:
            S.append(s_vec)
            Y.append(y_vec)
            if len(S) > m:
                S.pop(0)
                Y.pop(0)
        df = abs(fn - f)
        x, f, gp = xn, fn, gpn
        energies.append(f)
        gradnorms.append(float(np.linalg.norm(gp)))
        if callback:
            callback(it + 1, f, gradnorms[-1])
        if save:
            _save_gs(os.path.join(run_dir, "gs.npz"), x.reshape(shape, order="F"), energies, gradnorms)
        if df < f_tol * max(abs(f), 1.0):
            break
    return {"A": x.reshape(shape, order="F"), "energies": energies, "gradnorms": gradnorms, "evals": evals}


def normalize_gs(ts: host.CTMTensors):
    """optim_es.jl:212-222: A <- A / sqrt|<A|A>|, environment kept."""
    nrm = host.get_gs_norm(ts)
    A1 = ts.A / math.sqrt(abs(nrm))
    ts.set_A(A1)
    return ts


def substract_gs_energy(ts: host.CTMTensors, H):
    """optim_es.jl:224-234: H_i - (E0/2) I."""
    E0, _ = host.get_gs_energy(ts, H)
    e = (E0 / 2).real
    return [np.asarray(h, dtype=np.complex128) - e * np.eye(h.shape[0]) for h in H]


def tangent_basis(ts: host.CTMTensors, n_dm_Ad: np.ndarray):
    """get_tangent_basis (optim_es.jl:236-258, "default"): null space of the
    row vector vec(ndm_Ad) (D^4 d - 1 vectors), from its full SVD."""
    row = n_dm_Ad.reshape(1, -1, order="F").astype(np.complex128)
    _, _, vh = np.linalg.svd(row, full_matrices=True)
    return vh.conj().T[:, 1:]


def prepare_basis(H, A, cfg: Dict[str, Any], engine: Optional[host.Engine] = None):
    """prepare_basis (optim_es.jl:34-73) on the device, for a ground state A
    (the reference loads it from gs.jld2): renormalise A (max-abs), converge
    the environment from init_ctm1 with the energy criterion at 2 max_iter and
    rg_tol^2, restore the configured Params, normalise A (normalize_gs),
    subtract E0/2 from both bond Hamiltonians (substract_gs_energy) and take
    the default tangent basis.  Returns (ts, H_sub, basis) with basis
    (D^4 d, D^4 d - 1) complex; ts stays on the device for optim_es."""
    A = np.asarray(A)
    A = A / np.abs(A).max()
    cfg0 = dict(cfg)
    ts = host.CTMTensors(A, cfg0, engine=engine)
    ts.Params["max_iter"] = 2 * int(cfg0.get("max_iter", 20))
    ts.Params["rg_tol"] = float(cfg0.get("rg_tol", 1e-6)) ** 2
    host.run_ctm(ts, conv_fun="energy", H=H)
    ts.Params = dict(cfg0)
    normalize_gs(ts)
    H2 = substract_gs_energy(ts, H)
    basis = tangent_basis(ts, host.single_dm_Ad(ts))
    return ts, H2, basis


def _es_subspace(effH: np.ndarray, effN: np.ndarray, nrmB_cut=1e-3):
    """The common part of compute_es / evaluate_es (expectation.jl:13-56,
    152-183): Hermitian parts, the eigenvectors of N sorted by decreasing
    eigenvalue, and the selection by nrmB_cut (a ratio to the largest
    eigenvalue, or, when an int, the values above the (cut+1)-th)."""
    H2 = (effH + effH.conj().T) / 2
    N2 = (effN + effN.conj().T) / 2
    ev, P = np.linalg.eigh(N2)
    idx = np.argsort(ev)[::-1]
    ev, P = ev[idx], P[:, idx]
    if isinstance(nrmB_cut, (int, np.integer)) and not isinstance(nrmB_cut, bool):
        keep = ev > ev[nrmB_cut]
    else:
        keep = ev / ev.max() > nrmB_cut
    P = P[:, keep]
    Hp = P.conj().T @ H2 @ P
    Np = P.conj().T @ N2 @ P
    return (Hp + Hp.conj().T) / 2, (Np + Np.conj().T) / 2, P


def compute_es(effH: np.ndarray, effN: np.ndarray, nrmB_cut=1e-3):
    """compute_es (expectation.jl:13-56): the generalised eigenproblem
    H x = E N x on the selected subspace.  Returns (es, vecs, P) sorted by
    real part (es complex, as Julia's eigen(H2, N2))."""
    import scipy.linalg as sl
    Hp, Np, P = _es_subspace(effH, effN, nrmB_cut)
    es, vecs = sl.eig(Hp, Np)
    ix = np.argsort(es.real)
    return es[ix], vecs[:, ix], P


def evaluate_es(effH: np.ndarray, effN: np.ndarray, nrmB_cut=1e-3):
    """evaluate_es (expectation.jl:152-183): (es, vecs), the generalised
    eigenvalues (complex) and eigenvectors of H x = E N x on the selected
    subspace, sorted by real part."""
    es, vecs, _ = compute_es(effH, effN, nrmB_cut)
    return es, vecs


def band_energies(effH: np.ndarray, effN: np.ndarray, nrmB_cut=1e-3) -> np.ndarray:
    """The real parts of evaluate_es's eigenvalues, ascending: the band
    energies of one momentum."""
    es, _ = evaluate_es(effH, effN, nrmB_cut)
    return np.sort(es.real)


def es_column(px: float, py: float, ts: host.CTMTensors, H, basis: np.ndarray, i: int, C=None,
              engine: Optional[host.Engine] = None):
    """One basis vector of optim_es (optim_es.jl:127-153): a nested
    environment started from the ground-state C/T, the pullback w.r.t. B
    (get_es_grad), projected on the basis: (effH[:, i], effN[:, i]).  engine:
    the context to run it on (default: the one holding ts)."""
    C = C if C is not None else [ts.get_CT(k) for k in range(1, 5)]
    t = host.CTMTensors(ts.A, dict(ts.Params), engine=engine or ts.engine, init=False)
    try:
        for k in range(4):
            t.set_CT(k + 1, *C[k])
        t.Params["px"], t.Params["py"] = px * math.pi, py * math.pi
        gH, gN = host.get_es_grad(t, H, basis[:, i])
    finally:
        t.close()
    return basis.conj().T @ gH / 2, basis.conj().T @ gN


def optim_es(px: float, py: float, ts: host.CTMTensors, H, basis: np.ndarray,
             indices: Optional[List[int]] = None, engines: Optional[List[host.Engine]] = None):
    """optim_es (optim_es.jl:91-165) for one momentum (px, py in units of pi).

    ts: normalised ground-state environment (copied per basis vector from its
    C/T), H: Hamiltonian with E0/2 subtracted, basis: (D^4 d, nb) complex.
    indices: which basis columns to compute (all by default).  engines: more
    contexts on the same GPU (each with its own stream) to run the independent
    basis vectors concurrently, one host thread per context (the library
    releases the interpreter lock during its calls); the columns do not depend
    on which context computed them beyond the projectors' random sketches.
    Returns (effH, effN) with those columns filled (others zero)."""
    nb = basis.shape[1]
    effH = np.zeros((nb, nb), dtype=np.complex128)
    effN = np.zeros((nb, nb), dtype=np.complex128)
    C = [ts.get_CT(k) for k in range(1, 5)]
    cols = list(range(nb) if indices is None else indices)
    if not engines:
        for i in cols:
            effH[:, i], effN[:, i] = es_column(px, py, ts, H, basis, i, C)
        return effH, effN
    import threading
    lock = threading.Lock()
    queue = list(cols)

    errors = []

    def worker(eng):
        while True:
            with lock:
                if not queue or errors:
                    return
                i = queue.pop(0)
            try:
                h, n = es_column(px, py, ts, H, basis, i, C, engine=eng)
            except BaseException as exc:  # re-raised in the calling thread
                with lock:
                    errors.append(exc)
                return
            effH[:, i], effN[:, i] = h, n

    threads = [threading.Thread(target=worker, args=(e,)) for e in engines]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return effH, effN


def correlation_TM(ts: host.CTMTensors, direction: str = "h", N: int = 10, full: bool = False):
    """correlation_TM (expectation.jl:193-220): the transfer matrix of two
    edge tensors, TM = tcon([E4, E2], [[-1,-3,1,2],[-2,-4,1,2]]) ("h") or of
    E1, E3 ("v"), reshaped to (chi^2, chi^2), contracted on the device; its
    N largest-magnitude eigenvalues (all when full), as the reference returns
    them: (|es| sorted descending and > 0, es, TM)."""
    Es = [ts.get_CT(k)[1] for k in range(1, 5)]
    a, b = (Es[3], Es[1]) if direction == "h" else (Es[0], Es[2])
    TM = host.tcon([a, b], [[-1, -3, 1, 2], [-2, -4, 1, 2]], engine=ts.engine)
    n = TM.shape[0] * TM.shape[1]
    TM = TM.reshape(n, -1, order="F")
    if full or N >= n - 1:
        es = np.linalg.eigvals(TM)
    else:
        from scipy.sparse.linalg import eigs
        es = eigs(TM, k=N, which="LM", return_eigenvectors=False)
    es1 = np.sort(np.abs(es))[::-1]
    return es1[es1 > 0], es, TM


def correlation_TM_A(A, cfg: Dict[str, Any], direction: str = "h", engine: Optional[host.Engine] = None):
    """correlation_TM_A (expectation.jl:185-191): CTMTensors(A, cfg), run_ctm
    with the spectrum criterion, then correlation_TM of the converged edges."""
    ts = host.CTMTensors(A, cfg, engine=engine)
    try:
        ts, _ = host.run_ctm(ts)
        return correlation_TM(ts, direction=direction)
    finally:
        ts.close()


# ---------------------------------------------------------------- plaquette (h4) drivers
def _wrap_svd(M: np.ndarray):
    """wrap_svd (wrapper.jl:25-55) without a rank cap: SVD sorted descending,
    keep s/s_max > 1e-12 (plus one when |s[n+1] - s[n]| < 1e-10)."""
    u, s, vh = np.linalg.svd(M, full_matrices=False)
    n = int(np.sum(s / s[0] > 1e-12)) if s[0] > 0 else 1
    if n < len(s) and abs(s[n] - s[n - 1]) < 1e-10:
        n += 1
    return u[:, :n], s[:n], vh[:n].conj().T


def get_local_h(h: np.ndarray) -> List[np.ndarray]:
    """get_local_h (local_h.jl:1-31): the plaquette Hamiltonian h of shape
    (d^2, d^2, d^2, d^2) as the MPO [s1, s2, s3, s4] by successive SVDs
    (column-major reshapes, as Julia)."""
    h = np.asarray(h, dtype=np.complex128)
    dims = h.shape
    d = int(round(math.sqrt(dims[0])))
    sl = []
    u, s, v = _wrap_svd(h.reshape(dims[0], -1, order="F"))
    sl.append((u * np.sqrt(s)).reshape(d, d, -1, order="F"))
    sdots = np.sqrt(s)[:, None] * v.conj().T
    for i in range(len(dims) - 2):
        dl = sdots.shape[0]
        sdots = sdots.reshape(dl * dims[i], -1, order="F")
        u, s, v = _wrap_svd(sdots)
        sl.append((u * np.sqrt(s)).reshape(dl, d, d, -1, order="F"))
        sdots = np.sqrt(s)[:, None] * v.conj().T
    sl.append(sdots.reshape(sdots.shape[0], d, d, order="F"))
    return sl


def tout_site(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """tout_site (honeycomb.jl:37-42): c[i,j,k,l] = a[i,j] b[k,l] reshaped to (d1 d2, d3 d4)."""
    c = np.einsum("ij,kl->ijkl", a, b)
    s = c.shape
    return c.reshape(s[0] * s[1], s[2] * s[3], order="F")


def substract_gs_energy_h4(ts: host.CTMTensors, h: np.ndarray) -> np.ndarray:
    """substract_gs_energy_h4 (optim_es_h4.jl:170-183): h - E0 hI with E0 the
    plaquette energy of the environment in ts."""
    E0 = host.get_gs_energy_4x4(ts, get_local_h(h))
    d = int(round(math.sqrt(h.shape[0])))
    II = np.eye(d, dtype=np.complex128)
    hI = tout_site(tout_site(II, II), tout_site(II, II)).reshape(d * d, d * d, d * d, d * d, order="F")
    return np.asarray(h, dtype=np.complex128) - E0 * hI


def prepare_basis_h4(h: np.ndarray, A, cfg: Dict[str, Any], engine: Optional[host.Engine] = None):
    """prepare_basis_h4 (optim_es_h4.jl:13-55): converge with the plaquette
    energy at 2 max_iter and rg_tol^2, normalise A, subtract E0 hI, take the
    default tangent basis.  Returns (ts, H4, basis) with H4 the MPO of the
    subtracted Hamiltonian (what the reference saves in basis.jld2)."""
    A = np.asarray(A)
    A = A / np.abs(A).max()
    cfg0 = dict(cfg)
    ts = host.CTMTensors(A, cfg0, engine=engine)
    ts.Params["max_iter"] = 2 * int(cfg0.get("max_iter", 20))
    ts.Params["rg_tol"] = float(cfg0.get("rg_tol", 1e-6)) ** 2
    host.run_ctm_4x4(ts, get_local_h(h), nested=False)
    ts.Params = dict(cfg0)
    normalize_gs(ts)
    H4 = get_local_h(substract_gs_energy_h4(ts, h))
    basis = tangent_basis(ts, host.single_dm_Ad(ts))
    return ts, H4, basis


def optim_gs_h4(h: np.ndarray, A0, cfg, engine: Optional[host.Engine] = None, **kw):
    """optim_gs_h4 (optim_gs_h4.jl:14-98): optim_gs with the plaquette
    Hamiltonian h (d^2, d^2, d^2, d^2), split into its MPO by get_local_h, and
    the plaquette E+grad unit (host.fg_h4)."""
    return optim_gs(get_local_h(h), A0, cfg, engine=engine, fg_fn=host.fg_h4, **kw)


def es_column_h4(px: float, py: float, ts: host.CTMTensors, H4, basis: np.ndarray, i: int, C=None):
    """One basis vector of optim_es_h4 (optim_es_h4.jl:92-108): (effH[:, i], effN[:, i])."""
    C = C if C is not None else [ts.get_CT(k) for k in range(1, 5)]
    t = host.CTMTensors(ts.A, dict(ts.Params), engine=ts.engine, init=False)
    try:
        for k in range(4):
            t.set_CT(k + 1, *C[k])
        t.Params["px"], t.Params["py"] = px * math.pi, py * math.pi
        gH, gN = host.get_es_grad_h4(t, H4, basis[:, i])
    finally:
        t.close()
    return basis.conj().T @ gH / 2, basis.conj().T @ gN


def optim_es_h4(px: float, py: float, ts: host.CTMTensors, H4, basis: np.ndarray,
                indices: Optional[List[int]] = None):
    """optim_es_h4 (optim_es_h4.jl:57-131) for one momentum (units of pi)."""
    nb = basis.shape[1]
    effH = np.zeros((nb, nb), dtype=np.complex128)
    effN = np.zeros((nb, nb), dtype=np.complex128)
    C = [ts.get_CT(k) for k in range(1, 5)]
    for i in (range(nb) if indices is None else indices):
        effH[:, i], effN[:, i] = es_column_h4(px, py, ts, H4, basis, i, C)
    return effH, effN


def shard_indices(n: int, rank: int, world: int) -> List[int]:
    """Basis columns of one rank: i = rank, rank + world, ... (round robin, so
    that the ranks' shares differ by at most one column)."""
    return list(range(rank, n, world))


# ---------------------------------------------------------------- optim_wp
_SIGX = np.array([[0, 1], [1, 0]], dtype=np.complex128)
_SIGY = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
_SIGZ = np.array([[1, 0], [0, -1]], dtype=np.complex128)
_SI = np.eye(2, dtype=np.complex128)


def tout(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """tout (basis.jl:16-21): c[i,k,j,l] = a[i,j] b[k,l] reshaped to (d1 d2, d3 d4)."""
    c = np.einsum("ij,kl->ikjl", a, b)
    s = c.shape
    return c.reshape(s[0] * s[1], s[2] * s[3], order="F")


def get_w_op() -> np.ndarray:
    """get_w_op (honeycomb.jl:82-101): the XX plaquette operator of the
    honeycomb model, shape (d^2, d^2, d^2, d^2) with d = 4."""
    Ix, yz = tout(_SI, _SIGX), tout(_SIGY, _SIGZ)
    xI, zy = tout(_SIGX, _SI), tout(_SIGZ, _SIGY)
    wp = tout_site(tout_site(Ix, yz), tout_site(xI, zy))
    return wp.reshape(16, 16, 16, 16, order="F")


def optim_wp(ts: host.CTMTensors, wp_op: np.ndarray, basis: np.ndarray, site: Optional[int] = None,
             es_resume: int = 1, es_num: int = 0, effH: Optional[np.ndarray] = None,
             effN: Optional[np.ndarray] = None):
    """optim_wp (optim_wp.jl:133-193) in the fixed environment held by ts (the
    reference loads ts and the basis from basis.jld2): for every basis vector,
    get_wp_grad at plaquette site ``site`` (Params["wp"], default 1) on the
    device, effH[:, i] = basis' gH / 2, effN[:, i] = basis' gN / 2.  As the
    reference: vectors before es_resume (1-based) are skipped, and with
    es_num > 0 the loop stops after es_num vectors; effH/effN of an earlier
    partial run can be passed in to continue it.  Returns (effH, effN)."""
    basis = np.asarray(basis, dtype=np.complex128)
    nb = basis.shape[1]
    effH = np.zeros((nb, nb), dtype=np.complex128) if effH is None else np.array(effH, dtype=np.complex128)
    effN = np.zeros((nb, nb), dtype=np.complex128) if effN is None else np.array(effN, dtype=np.complex128)
    wp4 = get_local_h(wp_op)
    bh = basis.conj().T
    for i in range(1, nb + 1):
        if i < es_resume:
            continue
        if es_num > 0 and i >= es_resume + es_num:
            break
        gH, gN, _, _ = host.get_wp_grad(ts, wp4, basis[:, i - 1], site)
        effH[:, i - 1] = bh @ gH / 2
        effN[:, i - 1] = bh @ gN / 2
    return effH, effN


def _eig_sorted(H2, N2):
    import scipy.linalg as sl
    es, vecs = sl.eig(H2, N2)
    ix = np.argsort(es.real, kind="stable")
    return es[ix], vecs[:, ix]


def get_wp_basis(effH: np.ndarray, effN: np.ndarray, basis: np.ndarray):
    """get_wp_basis (optim_wp.jl:25-72): effH, effN hermitised, the metric
    diagonalised (eigenvalues descending), eigen(H2, N2) in that frame, and the
    basis split by the sign of the eigenvalues.  Returns (es, basis_p,
    basis_m): the new bases basis P vecs of the positive and negative sectors
    (the reference saves them as <basis>_<wp>p.jld2 and _<wp>m.jld2)."""
    H = (effH + effH.conj().T) / 2
    N = (effN + effN.conj().T) / 2
    ev, P = np.linalg.eigh(N)
    P = P[:, np.argsort(ev)[::-1]]
    N2 = P.conj().T @ N @ P
    H2 = P.conj().T @ H @ P
    es, vecs = _eig_sorted((H2 + H2.conj().T) / 2, (N2 + N2.conj().T) / 2)
    exci = np.asarray(basis, dtype=np.complex128) @ P @ vecs
    return es, exci[:, es.real > 0.0], exci[:, es.real < 0.0]


def evaluate_wp(effH: np.ndarray, effN: np.ndarray, nrmB_cut=1e-3):
    """evaluate_wp (optim_wp.jl:86-119): as compute_es, the generalised
    eigenproblem on the metric's leading subspace (nrmB_cut relative, or an
    integer count).  Returns (es, vecs, P)."""
    return compute_es(effH, effN, nrmB_cut)


def optim_es_sharded(px: float, py: float, ts: Optional[host.CTMTensors], H, basis: np.ndarray, group=None,
                     column_fn=None):
    """optim_es over the ranks of a torch.distributed job (one process per GPU).

    The basis vectors of one momentum are independent units (each a nested
    CTMRG + pullback); rank r computes columns shard_indices(nb, r, world) and
    one all-reduce (sum; the other ranks' columns are zero) gives every rank
    the full effH and effN (nb x nb complex, ~0.4 MB each at nb = 161).  The
    collective runs on the process group's backend (NCCL on GPUs, gloo on CPU).
    column_fn(i) -> (effH[:, i], effN[:, i]) replaces the GPU computation
    (es_column) when given.  Without an initialised process group this is
    optim_es on one process."""
    import torch
    import torch.distributed as dist

    nb = basis.shape[1]
    dist_on = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if dist_on else 0
    world = dist.get_world_size(group) if dist_on else 1
    if column_fn is None:
        C = [ts.get_CT(k) for k in range(1, 5)]
        column_fn = lambda i: es_column(px, py, ts, H, basis, i, C)  # noqa: E731
    effH = np.zeros((nb, nb), dtype=np.complex128)
    effN = np.zeros((nb, nb), dtype=np.complex128)
    for i in shard_indices(nb, rank, world):
        effH[:, i], effN[:, i] = column_fn(i)
    if world > 1:
        backend = dist.get_backend(group)
        dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        buf = torch.from_numpy(np.stack([effH.real, effH.imag, effN.real, effN.imag])).to(dev)
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
        b = buf.cpu().numpy()
        effH = b[0] + 1j * b[1]
        effN = b[2] + 1j * b[3]
    return effH, effN
