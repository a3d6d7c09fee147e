"""Learned warm start for CTMRG (no counterpart in the reference, whose run_ctm
always starts from init_ctm1, ctm_tensor.jl:97-130).

A small network (host.Mlp: BF16 tensor-core GEMMs, FP32 parameters) maps the
flattened iPEPS tensor A to a rank-r environment in a canonical gauge; CTMRG
then iterates from that environment to rg_tol.  Plain CTMRG stays the arbiter
and the fallback: a warm start that has not converged within its iteration
budget, or that converged outside the energy bound of H (a spurious fixed
point), is dropped and the run restarts from init_ctm1.  The tests compare the
warm-started energies with plain CTMRG's.

Canonical gauge.  With a one-site unit cell an environment has four bond
gauges, one per boundary (top, right, bottom, left), each an invertible
chi x chi matrix X: the boundary's edge E becomes X^-1 E X (its two legs meet
each other between neighbouring sites) and the two corner legs on the
boundary absorb X or X^-T, so every contraction is unchanged.  CTMRG's
truncation (an SVD of the half-system matrix) is invariant only under the
orthogonal part of that freedom: from an environment in another GL(chi) gauge
it keeps a slightly different subspace and has to relax back (a fixed point
re-gauged by a well-conditioned X needs about as many iterations as a cold
start to get back to 1e-10 in the energy).  So the network's target keeps
CTMRG's own gauge and fixes only the orthogonal part: C1 = U S V^T fixes the
left (U) and top (V) gauges; the sign of singular pair a >= 1 makes the
leading entry of E1[b, a, :, :] positive in that gauge, b < a the pair coupled
most strongly to a (flipping every pair at once is a trivial gauge); the
right gauge makes V^T C2 Q_right lower triangular with a positive diagonal
(an LQ factorisation), the bottom gauge does the same for U^T C4; C3 and the
edges follow.  "Leading" is the first entry in storage order whose modulus is
within 1e-6 of the largest, so that exact ties of symmetric tensors break the
same way.  Rectangular corners (bonds of different dimensions after a
cutoff-limited truncation) leave basis vectors past a corner's rank; they are
ordered by the next corner on their boundary and signed by its edge in the
same way.  Truncating every bond to its leading r directions (zero-padding
narrower ones) gives the network's target: 4 r^2 corner entries and 4 r^2 D^2
edge entries.

Which corner legs face which edge legs follows the reference's contractions
(ctmrg.jl:122-252, evaluation.jl:124-248): E1 (top) leg 0 faces C1 leg 1 and
leg 1 faces C2 leg 0; E2 (right) leg 0 faces C2 leg 1, leg 1 faces C3 leg 0;
E3 (bottom) leg 0 faces C4 leg 1, leg 1 faces C3 leg 1; E4 (left) leg 0 faces
C1 leg 0, leg 1 faces C4 leg 0.  A corner leg facing an edge's leg 0 absorbs
X, one facing leg 1 absorbs X^-T.
"""
from __future__ import annotations

import time
from typing import Any, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import host

# boundary j (0 top, 1 right, 2 bottom, 3 left), 0-based: (corner, leg) facing
# edge j's leg 0, and (corner, leg) facing its leg 1
FACING = [((0, 1), (1, 0)), ((1, 1), (2, 0)), ((3, 1), (2, 1)), ((0, 0), (3, 0))]


def _apply_leg(E: np.ndarray, leg: int, Q: np.ndarray) -> np.ndarray:
    """E with leg `leg` (0 or 1) contracted against Q (new index = column of Q)."""
    if leg == 0:
        return np.einsum("iabc,ij->jabc", E, Q)
    return np.einsum("aibc,ij->ajbc", E, Q)


def _corner_leg(C: np.ndarray, leg: int, Q: np.ndarray) -> np.ndarray:
    return Q.T @ C if leg == 0 else C @ Q


def gauge_transform(Cs: Sequence[np.ndarray], Es: Sequence[np.ndarray], Xs: Sequence[np.ndarray]):
    """Apply the boundary gauges Xs[j] (invertible): E_j -> X^-1 E_j X, the
    corner leg facing E_j's leg 0 absorbs X, the one facing leg 1 absorbs X^-T."""
    Cn = [np.array(C) for C in Cs]
    En = [np.array(E) for E in Es]
    for j, ((k0, l0), (k1, l1)) in enumerate(FACING):
        X = np.asarray(Xs[j])
        XiT = np.linalg.inv(X).T
        Cn[k0] = _corner_leg(Cn[k0], l0, X)
        Cn[k1] = _corner_leg(Cn[k1], l1, XiT)
        En[j] = _apply_leg(_apply_leg(En[j], 0, XiT), 1, X)
    return Cn, En


def _lead(x: np.ndarray, rel: float = 1e-6) -> int:
    """Flat index of the first entry whose modulus is within rel of the largest
    (a tie-proof "entry of largest modulus": symmetric tensors have exact ties)."""
    a = np.abs(np.ravel(x))
    return int(np.argmax(a >= (1.0 - rel) * a.max()))


def _lq_gauge(M: np.ndarray) -> np.ndarray:
    """Square orthogonal Q with M Q lower triangular with a non-negative
    diagonal (M may be rectangular; columns past its rank stay as QR gives them)."""
    Q, R = np.linalg.qr(M.T, mode="complete")
    d = np.sign(np.diag(R))
    d[d == 0] = 1.0
    Q[:, :len(d)] *= d
    return Q


def _null_basis(B: np.ndarray, C: np.ndarray) -> np.ndarray:
    """Basis of span(B) (orthonormal columns) ordered by the corner C whose
    first leg it indexes: the left singular vectors of B^T C, which do not
    depend on the gauge of C's other leg (signs are fixed separately)."""
    if B.shape[1] == 0:
        return B
    P, _, _ = np.linalg.svd(B.T @ C)
    return B @ P


def _signs(E: np.ndarray, start: int, sgn: np.ndarray) -> None:
    """Signs sgn[c], c >= start, of the basis vectors of a boundary whose edge,
    in that basis, is E: the leading entry of E[b, c, :, :] * sgn[b] is made
    positive, b < c the vector coupled most strongly to c."""
    for c in range(max(start, 1), E.shape[0]):
        blk = E[:c, c] * sgn[:c, None, None]
        b = _lead(np.abs(blk).reshape(c, -1).max(1))
        row = blk[b]
        sgn[c] = -1.0 if row.flat[_lead(row)] < 0 else 1.0


def canonical(Cs: Sequence[np.ndarray], Es: Sequence[np.ndarray]):
    """The environment with its orthogonal boundary gauges fixed (full rank)."""
    Cs = [np.asarray(C, dtype=np.float64) for C in Cs]
    Es = [np.asarray(E, dtype=np.float64) for E in Es]
    U, s, Vt = np.linalg.svd(Cs[0])
    V = Vt.T.copy()
    ns = len(s)
    # corners may be rectangular (the boundaries' bond dimensions differ after a
    # cutoff-limited truncation): basis vectors past C1's rank are ordered by the
    # next corner on their boundary (C4 for the left one, C2 for the top one)
    U[:, ns:] = _null_basis(U[:, ns:], Cs[3])
    V[:, ns:] = _null_basis(V[:, ns:], Cs[1])
    # signs: singular pairs and the top boundary's extra vectors from E1 (pair 0
    # is free: flipping every pair at once is a trivial gauge), then the left
    # boundary's extra vectors from E4
    st = np.ones(V.shape[1])
    _signs(_apply_leg(_apply_leg(Es[0], 0, V), 1, V), 1, st)
    V = V * st
    U[:, :ns] *= st[:ns]
    sl = np.ones(U.shape[1])
    _signs(_apply_leg(_apply_leg(Es[3], 0, U), 1, U), ns, sl)
    U = U * sl
    # right and bottom gauges: LQ of C2 and C4 in the fixed top and left gauges;
    # vectors past the corner's rank are ordered by C3 and signed by the edge
    Qs = []
    for M, C3leg, E in ((V.T @ Cs[1], Cs[2], Es[1]), (U.T @ Cs[3], Cs[2].T, Es[2])):
        Q = _lq_gauge(M)
        rk = min(M.shape)
        Q[:, rk:] = _null_basis(Q[:, rk:], C3leg)
        sq = np.ones(Q.shape[1])
        _signs(_apply_leg(_apply_leg(E, 0, Q), 1, Q), max(rk, 1), sq)
        Qs.append(Q * sq)
    return gauge_transform(Cs, Es, [V, Qs[0], Qs[1], U])


def gauge_fix(Cs: Sequence[np.ndarray], Es: Sequence[np.ndarray], r: Optional[int] = None) -> np.ndarray:
    """Canonical-gauge vector of a real environment truncated (or zero-padded)
    to rank r on every bond: [C1 .. C4 (r x r), E1 .. E4 (r, r, D, D)], each
    column-major and scaled to max-abs 1."""
    Cn, En = canonical(Cs, Es)
    r = r or max(max(C.shape) for C in Cn)
    parts = []
    for X in list(Cn) + list(En):
        # bonds narrower than r are padded with zeros
        P = np.zeros((r, r) + X.shape[2:])
        a, b = min(r, X.shape[0]), min(r, X.shape[1])
        P[:a, :b] = X[:a, :b] / np.abs(X).max()
        parts.append(P.ravel(order="F"))
    return np.concatenate(parts)


def unpack(vec: np.ndarray, r: int, D: int):
    """(Cs, Es) of a rank-r environment in the canonical gauge from its vector."""
    vec = np.asarray(vec, dtype=np.float64)
    Cs = [np.asfortranarray(vec[j * r * r:(j + 1) * r * r].reshape((r, r), order="F")) for j in range(4)]
    o = 4 * r * r
    n = r * r * D * D
    Es = [np.asfortranarray(vec[o + j * n:o + (j + 1) * n].reshape((r, r, D, D), order="F")) for j in range(4)]
    return Cs, Es


def read_env(ts: host.CTMTensors):
    Cs, Es = [], []
    for k in range(1, 5):
        C, E = ts.get_CT(k)
        Cs.append(np.asarray(C))
        Es.append(np.asarray(E))
    return Cs, Es


def energy_bound(H) -> float:
    """|E| per site can not exceed ||Hh||_2 + ||Hv||_2 (one horizontal and one
    vertical bond per site); a converged run outside it is a spurious fixed
    point (from a bad starting environment) and is rejected."""
    return float(sum(np.linalg.norm(np.asarray(h).reshape(int(np.sqrt(np.asarray(h).size)), -1), 2) for h in H)) * (1 + 1e-9)


def converge_default(A, H, cfg: Dict[str, Any], engine=None):
    """Plain CTMRG from init_ctm1 with the energy criterion (the arbiter)."""
    ts = host.CTMTensors(A, cfg, engine=engine)
    ts, info = host.run_ctm(ts, conv_fun="energy", H=H)
    return ts, info


class WarmStart:
    """Network + standardisation of inputs and targets for one (D, d, r)."""

    def __init__(self, D: int, d: int, r: int = 8, hidden: int = 512, max_batch: int = 256, seed: int = 0,
                 engine=None):
        self.D, self.d, self.r = D, d, r
        self.n_in = D ** 4 * d
        self.n_out = 4 * r * r + 4 * r * r * D * D
        self.engine = engine or host.default_engine()
        self.net = host.Mlp(self.n_in, hidden, self.n_out, max_batch=max_batch, seed=seed, engine=self.engine)
        self.max_batch = max_batch
        self.xm = self.xs = self.ym = self.ys = None

    def _x(self, As) -> np.ndarray:
        return np.stack([np.asarray(A, dtype=np.float64).ravel(order="F") for A in As])

    def fit(self, As, targets: np.ndarray, epochs: int = 400, lr: float = 1e-3, seed: int = 0) -> List[float]:
        X = self._x(As)
        Y = np.asarray(targets, dtype=np.float64)
        self.xm, self.xs = X.mean(0), X.std(0) + 1e-8
        self.ym, self.ys = Y.mean(0), Y.std(0) + 1e-8
        Xn = ((X - self.xm) / self.xs).astype(np.float32)
        Yn = ((Y - self.ym) / self.ys).astype(np.float32)
        rng = np.random.default_rng(seed)
        losses = []
        n = len(X)
        for _ in range(epochs):
            perm = rng.permutation(n)
            ep = []
            for b0 in range(0, n, self.max_batch):
                idx = perm[b0:b0 + self.max_batch]
                ep.append(self.net.train_step(Xn[idx], Yn[idx], lr))
            losses.append(float(np.mean(ep)))
        return losses

    def predict(self, As) -> np.ndarray:
        Xn = ((self._x(As) - self.xm) / self.xs).astype(np.float32)
        out = []
        for b0 in range(0, len(Xn), self.max_batch):
            out.append(self.net.forward(Xn[b0:b0 + self.max_batch]))
        return np.concatenate(out).astype(np.float64) * self.ys + self.ym

    def converge(self, A, H, cfg: Dict[str, Any], warm_max_iter: Optional[int] = None):
        """CTMRG from the predicted environment; falls back to init_ctm1 when it
        has not converged within warm_max_iter iterations (default max_iter)
        or converged outside the energy bound of H.  Returns (ts, info,
        used_warm_start, iterations in total)."""
        Cs, Es = unpack(self.predict([A])[0], self.r, self.D)
        wcfg = dict(cfg)
        if warm_max_iter is not None:
            wcfg["max_iter"] = int(warm_max_iter)
        ts = host.CTMTensors(A, wcfg, engine=self.engine, init=False)
        for k in range(4):
            ts.set_CT(k + 1, Cs[k], Es[k])
        ts, info = host.run_ctm(ts, conv_fun="energy", H=H)
        if info["converged"] and abs(info["log"][-1]["obj"]) <= energy_bound(H):
            return ts, info, True, len(info["log"])
        spent = len(info["log"])
        ts.close()
        ts, info = converge_default(A, H, cfg, engine=self.engine)
        return ts, info, False, spent + len(info["log"])

    def fg(self, A, H, cfg: Dict[str, Any], engine=None, warm_max_iter: Optional[int] = None):
        """The E+grad unit of optim_gs (host.fg) started from the predicted
        environment; same return value (E, g, info), info["warm_start"] telling
        whether the prediction was used and info["iterations"] the CTMRG
        iterations spent (fallback included)."""
        A = np.asarray(A, dtype=np.float64)
        A = A / np.abs(A).max()
        ts, info, used, iters = self.converge(A, H, cfg, warm_max_iter=warm_max_iter)
        E, g = host.energy_grad(ts, H)
        ts.close()
        info = dict(info, warm_start=used, iterations=iters)
        return E, g, info

    def close(self):
        self.net.close()


def path_family(D: int, d: int, seeds: Sequence[int], n_points: int, scale: float = 0.3):
    """A family of iPEPS tensors on straight paths A(t) = A0 + t (A1 - A0),
    t in [0, 1], around near-product states (a product state plus `scale`
    times a random tensor, so that CTMRG converges): one path per seed."""
    out = []
    for sd in seeds:
        rng = np.random.default_rng(sd)
        prod = np.zeros((D, D, D, D, d))
        prod[0, 0, 0, 0, :] = rng.standard_normal(d)
        A0 = prod + scale * rng.standard_normal(prod.shape)
        A1 = prod + scale * rng.standard_normal(prod.shape)
        for t in np.linspace(0.0, 1.0, n_points):
            A = A0 + t * (A1 - A0)
            out.append((sd, float(t), np.asfortranarray(A / np.abs(A).max())))
    return out


def evaluate(As, H, cfg: Dict[str, Any], ws: WarmStart, engine=None) -> Dict[str, Any]:
    """Iterations and time to rg_tol from init_ctm1 and from the warm start, and
    the converged energies of both (they must agree)."""
    rows = []
    for A in As:
        t0 = time.time()
        ts0, info0 = converge_default(A, H, cfg, engine=engine)
        t1 = time.time()
        E0 = host.get_gs_energy(ts0, H)[0].real
        ts0.close()
        t2 = time.time()
        ts1, info1, used, iters = ws.converge(A, H, cfg)
        t3 = time.time()
        E1 = host.get_gs_energy(ts1, H)[0].real
        ts1.close()
        rows.append(dict(iters_default=len(info0["log"]), iters_warm=iters, used_warm=used, E_default=E0, E_warm=E1,
                         s_default=t1 - t0, s_warm=t3 - t2, converged_default=info0.get("converged", True)))
    return dict(rows=rows, mean_iters_default=float(np.mean([r["iters_default"] for r in rows])),
                mean_iters_warm=float(np.mean([r["iters_warm"] for r in rows])),
                max_dE=float(max(abs(r["E_default"] - r["E_warm"]) for r in rows)),
                warm_used=sum(r["used_warm"] for r in rows), n=len(rows))
