"""CPU FP64 oracle for the iPEPS.jl CTMRG hot path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker or the timed CPU baseline.  The product path
(``ipeps.jl_b200``) never calls it.

What it is: a line-by-line restatement of the reference's Julia code in
torch-CPU float64 / complex128 (torch is used for ``einsum`` and for autograd;
the SVD is LAPACK ``gesdd`` through ``torch.linalg.svd``, the same routine as
Julia's default ``svd``).  Every function cites the reference file:line it
follows.  Julia arrays are column-major, so every reshape here goes through
``freshape`` (Fortran order) to keep the fused-leg order identical.

Pins: the honeycomb known-answer test of the reference (test/test_model.jl:9-16,
test/test_ctmrg.jl:5-12: ``real(e0)/8 == -0.16349 +- 1e-5``) and the nested
product rule (test/test_nest.jl:20-26) are re-asserted against this module in
``tests/test_oracle.py``.  The gradient (Zygote in the reference) has no pin
in the reference's tests; it is checked against central finite differences.

Sign/gauge: the reference takes the SVD of ``R1*R2`` via LAPACK; singular
vectors are defined up to phase, which cancels in every projector product
``P1*P2`` and therefore in energies and gradients.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional

import numpy as np
import torch

_F64 = torch.float64
_C128 = torch.complex128

# --------------------------------------------------------------------------
# array helpers (Julia semantics)
# --------------------------------------------------------------------------


def freshape(x: torch.Tensor, *shape: int) -> torch.Tensor:
    """Julia ``reshape`` (column-major) for a torch tensor."""
    if len(shape) == 1 and isinstance(shape[0], (tuple, list)):
        shape = tuple(shape[0])
    shape = list(shape)
    if -1 in shape:
        known = 1
        for s in shape:
            if s != -1:
                known *= s
        shape[shape.index(-1)] = x.numel() // known
    xt = x.permute(*reversed(range(x.dim()))) if x.dim() > 1 else x
    y = xt.reshape(tuple(reversed(shape)))
    return y.permute(*reversed(range(len(shape)))) if len(shape) > 1 else y


def permutedims(x: torch.Tensor, perm) -> torch.Tensor:
    """Julia ``permutedims`` with a 1-based permutation."""
    return x.permute(*[p - 1 for p in perm])


_LETTERS = "abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ"


def _einsum_spec(ind_xs):
    labels = {}
    for ind in ind_xs:
        for l in ind:
            if l not in labels:
                labels[l] = _LETTERS[len(labels)]
    n_out = sum(1 for ind in ind_xs for l in ind if l < 0)
    ins = ["".join(labels[l] for l in ind) for ind in ind_xs]
    out = "".join(labels[-(i + 1)] for i in range(n_out))
    return ",".join(ins) + "->" + out


# --------------------------------------------------------------------------
# EmptyT / NestedTensor (src/nested_tensor/emptyT.jl:1-29,
# src/nested_tensor/nested_tensor.jl:1-66).  EmptyT is ``None`` here.
# --------------------------------------------------------------------------


class NestedTensor:
    """4-component first-order tensor (nested_tensor.jl:1-3)."""

    def __init__(self, data):
        self.data = list(data)

    def __getitem__(self, i):  # 1-based like Julia
        return self.data[i - 1]

    def size(self, i=None):
        return self.data[0].shape if i is None else self.data[0].shape[i - 1]

    def __mul__(self, b):  # nested_tensor.jl:44 (componentwise, b scalar or matrix)
        return NestedTensor([_mul(a, b) for a in self.data])

    def __rmul__(self, a):  # nested_tensor.jl:43
        return NestedTensor([_mul(a, x) for x in self.data])

    def __add__(self, other):  # nested_tensor.jl:51
        return NestedTensor([_add(a, b) for a, b in zip(self.data, other.data)])


def _mul(a, b):
    if a is None or b is None:
        return None  # emptyT.jl:3-6
    if isinstance(a, torch.Tensor) and isinstance(b, torch.Tensor) and a.dim() == 2 and b.dim() == 2:
        if a.dtype != b.dtype:
            dt = torch.promote_types(a.dtype, b.dtype)
            a, b = a.to(dt), b.to(dt)
        return a @ b
    return a * b


def _add(a, b):
    if a is None:
        return b  # emptyT.jl:8-10
    if b is None:
        return a
    return a + b


def _tcon_plain(ind_xs, A, B):
    if A is None or B is None:
        return None  # emptyT.jl:24-26
    if A.dtype != B.dtype:  # Julia promotes Float64 x ComplexF64
        dt = torch.promote_types(A.dtype, B.dtype)
        A, B = A.to(dt), B.to(dt)
    return torch.einsum(_einsum_spec(ind_xs), A, B)


def tcon(xs, ind_xs):
    """``tcon(xs, ind_xs)`` (wrapper.jl:15-23) with nested dispatch (nested_tensor.jl:77-92).

    Positive labels are contracted, negative labels -1, -2, ... give the output
    order.
    """
    A, B = xs
    if isinstance(A, NestedTensor) and isinstance(B, NestedTensor):
        r1 = _tcon_plain(ind_xs, A[1], B[1])
        r2 = _add(_tcon_plain(ind_xs, A[1], B[2]), _tcon_plain(ind_xs, A[2], B[1]))
        r3 = _add(_tcon_plain(ind_xs, A[1], B[3]), _tcon_plain(ind_xs, A[3], B[1]))
        r4 = _add(_add(_tcon_plain(ind_xs, A[1], B[4]), _tcon_plain(ind_xs, A[4], B[1])),
                  _add(_tcon_plain(ind_xs, A[2], B[3]), _tcon_plain(ind_xs, A[3], B[2])))
        return NestedTensor([r1, r2, r3, r4])
    if isinstance(A, NestedTensor):
        return NestedTensor([_tcon_plain(ind_xs, a, B) for a in A.data])
    if isinstance(B, NestedTensor):
        return NestedTensor([_tcon_plain(ind_xs, A, b) for b in B.data])
    return _tcon_plain(ind_xs, A, B)


def wrap_reshape(A, *dims):
    """nested_tensor.jl:54-55"""
    if isinstance(A, NestedTensor):
        return NestedTensor([None if a is None else freshape(a, *dims) for a in A.data])
    return freshape(A, *dims)


def wrap_permutedims(A, perm):
    """nested_tensor.jl:57-58"""
    if isinstance(A, NestedTensor):
        return NestedTensor([None if a is None else permutedims(a, perm) for a in A.data])
    return permutedims(A, perm)


def wrap_tr(A):
    """nested_tensor.jl:60-61"""
    if isinstance(A, NestedTensor):
        return NestedTensor([None if a is None else torch.diagonal(a).sum() for a in A.data])
    return torch.diagonal(A).sum()


def shift(A, phi):
    """nested_tensor.jl:65: component 2 times e^{i phi}, component 3 times e^{-i phi}."""
    ph = complex(math.cos(phi), math.sin(phi))
    return NestedTensor([A[1], _mul(A[2], ph), _mul(A[3], ph.conjugate()), A[4]])


def renormalize(A):
    """wrapper.jl:57 (max-abs), nested_tensor.jl:70-75 (all components / max|A[1]|)."""
    if A is None:
        return None
    if isinstance(A, NestedTensor):
        factor = A[1].abs().max()
        return A * (1.0 / factor)
    return A / A.abs().max()


def conj(A):
    if A is None:
        return None
    return A.conj() if A.is_complex() else A


# --------------------------------------------------------------------------
# SVD + reference adjoint (src/utility/autodiff.jl:22-74)
# --------------------------------------------------------------------------

SVD_ETA = 1e-12


def svd_back(U, S, V, dU, dS, dV, eta=SVD_ETA):
    """``svd_back`` (autodiff.jl:41-74): full-SVD adjoint with Lorentzian broadening."""
    if dU is None and dS is None and dV is None:
        return None
    S2 = S * S
    Sinv = S / (S2 + eta)
    F = S2[None, :] - S2[:, None]  # F[i,j] = S2[j] - S2[i]   (S2' .- S2)
    F = F / (F * F + eta)
    res = torch.zeros((S.shape[0], S.shape[0]), dtype=U.dtype)
    if dU is not None:
        UdU = U.mH @ dU
        J = F.to(U.dtype) * UdU
        res = res + (J + J.mH) @ torch.diag(S).to(U.dtype)
        if U.is_complex():
            res = res + torch.diag(1j * torch.diagonal(UdU).imag * Sinv)
    if dV is not None:
        VdV = V.mH @ dV
        K = F.to(V.dtype) * VdV
        res = res + torch.diag(S).to(V.dtype) @ (K + K.mH)
    if dS is not None:
        res = res + torch.diag(dS).to(res.dtype)
    res = U @ res @ V.mH
    if dU is not None and U.shape[0] != U.shape[1]:
        res = res + (dU - U @ (U.mH @ dU)) @ torch.diag(Sinv).to(U.dtype) @ V.mH
    if dV is not None and V.shape[0] != V.shape[1]:
        res = res + U @ torch.diag(Sinv).to(U.dtype) @ (dV.mH - (dV.mH @ V) @ V.mH)
    return res


class _SVD1(torch.autograd.Function):
    """``svd1`` + ``Zygote.@adjoint svd1`` (autodiff.jl:22-30)."""

    @staticmethod
    def forward(ctx, A):
        U, S, Vh = torch.linalg.svd(A, full_matrices=False)
        V = Vh.mH.contiguous()
        ctx.save_for_backward(U, S, V)
        return U, S, V

    @staticmethod
    def backward(ctx, dU, dS, dV):
        U, S, V = ctx.saved_tensors
        return svd_back(U, S, V, dU, dS, dV)


def svd1(A):
    return _SVD1.apply(A)


def cutoff_matrix(u, s, v, cutoff, n):
    """wrapper.jl:37-55: keep min(n, #{s/smax > cutoff}), +1 if |s[n+1]-s[n]| < 1e-10."""
    with torch.no_grad():
        n_above = int((s / s.max() > cutoff).sum().item())
    n = int(min(n, n_above))
    if s.shape[0] > n:
        with torch.no_grad():
            if abs(float(s[n]) - float(s[n - 1])) < 1e-10:
                n = n + 1
        u = u[:, :n]
        s = s[:n]
        v = v[:, :n]
    return u, s, v


def wrap_svd(A, n=math.inf):
    """wrapper.jl:25-35: SVD, sort descending, cutoff 1e-12."""
    u, s, v = svd1(A)
    with torch.no_grad():
        # sortperm(s)[end:-1:1]: stable ascending sort, then reversed.
        ix = torch.argsort(s, stable=True).flip(0)
    s = s[ix]
    u = u[:, ix]
    v = v[:, ix]
    return cutoff_matrix(u, s, v, 1e-12, n)


# --------------------------------------------------------------------------
# CTMTensors (src/ctm/ctm_tensor.jl)
# --------------------------------------------------------------------------


@dataclass
class CTMTensors:
    """Environment state (ctm_tensor.jl:3-18). ``None`` stands for EmptyT."""

    A: Any
    Ad: Any
    Cs: List[Any]
    Es: List[Any]
    B: Any = None
    Bd: Any = None
    B_Cs: List[Any] = field(default_factory=lambda: [None] * 4)
    Bd_Cs: List[Any] = field(default_factory=lambda: [None] * 4)
    BB_Cs: List[Any] = field(default_factory=lambda: [None] * 4)
    B_Es: List[Any] = field(default_factory=lambda: [None] * 4)
    Bd_Es: List[Any] = field(default_factory=lambda: [None] * 4)
    BB_Es: List[Any] = field(default_factory=lambda: [None] * 4)
    Params: Dict[str, Any] = field(default_factory=dict)

    def replace(self, **kw) -> "CTMTensors":
        d = dict(self.__dict__)
        d.update(kw)
        return CTMTensors(**d)


def make_ctm_tensors(A, cfg, Ad=None) -> CTMTensors:
    """``CTMTensors(A, cfg)`` / ``CTMTensors(A, Ad, cfg)`` (ctm_tensor.jl:63-69)."""
    if Ad is None:
        Ad = conj(A)
    Cs, Es = init_ctm1(A, Ad)
    return CTMTensors(A, Ad, Cs, Es, Params=dict(cfg))


def get_all_A(ts):
    """ctm_tensor.jl:20-27"""
    return ts.A if ts.B is None else NestedTensor([ts.A, ts.B, None, None])


def get_all_Ad(ts):
    """ctm_tensor.jl:29-36"""
    return ts.Ad if ts.B is None else NestedTensor([ts.Ad, None, ts.Bd, None])


def get_all_Cs(ts):
    """ctm_tensor.jl:38-45"""
    if ts.B is None:
        return ts.Cs
    return [NestedTensor([ts.Cs[i], ts.B_Cs[i], ts.Bd_Cs[i], ts.BB_Cs[i]]) for i in range(4)]


def get_all_Es(ts):
    """ctm_tensor.jl:47-55"""
    if ts.B is None:
        return ts.Es
    return [NestedTensor([ts.Es[i], ts.B_Es[i], ts.Bd_Es[i], ts.BB_Es[i]]) for i in range(4)]


def init_ctm1(A, Ad):
    """Default environment initialisation (ctm_tensor.jl:97-130)."""
    D = A.shape[0]
    C1 = freshape(tcon([A, Ad], [[1, 2, -1, -3, 3], [1, 2, -2, -4, 3]]), D * D, D * D)
    C2 = freshape(tcon([A, Ad], [[1, -1, -3, 2, 3], [1, -2, -4, 2, 3]]), D * D, D * D)
    C3 = freshape(tcon([A, Ad], [[-1, -3, 1, 2, 3], [-2, -4, 1, 2, 3]]), D * D, D * D)
    C4 = freshape(tcon([A, Ad], [[-1, 1, 2, -3, 3], [-2, 1, 2, -4, 3]]), D * D, D * D)
    Cs = [renormalize(c) for c in (C1, C2, C3, C4)]
    E1 = freshape(tcon([A, Ad], [[1, -1, -5, -3, 2], [1, -2, -6, -4, 2]]), D * D, D * D, D, D)
    E2 = freshape(tcon([A, Ad], [[-1, -5, -3, 1, 2], [-2, -6, -4, 1, 2]]), D * D, D * D, D, D)
    E3 = freshape(tcon([A, Ad], [[-5, -1, 1, -3, 2], [-6, -2, 1, -4, 2]]), D * D, D * D, D, D)
    E4 = freshape(tcon([A, Ad], [[-1, 1, -3, -5, 2], [-2, 1, -4, -6, 2]]), D * D, D * D, D, D)
    Es = [renormalize(e) for e in (E1, E2, E3, E4)]
    return Cs, Es


# --------------------------------------------------------------------------
# CTMRG (src/ctm/ctmrg.jl)
# --------------------------------------------------------------------------


def _norm(x):
    if isinstance(x, torch.Tensor):
        return float(torch.linalg.vector_norm(x.detach()).item()) if x.dim() > 0 else abs(complex(x.detach().item()))
    return abs(x)


def _length(x):
    if isinstance(x, torch.Tensor) and x.dim() > 0:
        return x.shape[0]
    return 1


def run_ctm(ts: CTMTensors, conv_fun=None, log=None):
    """``run_ctm`` (ctmrg.jl:1-55).  Returns (ts, conv).

    ``log`` (optional list) receives one dict per iteration: diff, s_diff, obj.
    """
    chi = ts.Params.get("chi", 30)
    min_iter = ts.Params.get("min_iter", 4)
    max_iter = ts.Params.get("max_iter", 20)
    tol = ts.Params.get("rg_tol", 1e-6)
    diffs = [1.0]
    conv: Any = 1.0
    diffs1 = [1.0]
    conv1: Any = 1.0
    for i in range(1, max_iter + 1):
        ts, s = rg_step(ts, chi)
        old_conv = conv
        if conv_fun is not None:
            with torch.no_grad():
                conv = conv_fun(ts)
            old_conv1 = conv1
            conv1 = s.detach()
            if _length(conv1) == _length(old_conv1):
                diffs1.append(_norm(conv1 - old_conv1))
        else:
            conv = s.detach()
        if _length(conv) == _length(old_conv):
            with torch.no_grad():
                diffs.append(_norm(conv - old_conv))
        if log is not None:
            log.append({"iter": i, "diff": diffs[-1], "s_diff": diffs1[-1],
                        "obj": conv if conv_fun is not None else None, "chi": int(s.shape[0])})
        if i >= min_iter and diffs[-1] < tol:
            break
    return ts, conv


def rg_step(ts, chi):
    """ctmrg.jl:57-64: left, right, top, bottom; returns s of the left move."""
    ts, s = left_rg(ts, chi)
    ts, _ = right_rg(ts, chi)
    ts, _ = top_rg(ts, chi)
    ts, _ = bottom_rg(ts, chi)
    return ts, s


def left_rg(ts, chi):
    """ctmrg.jl:66-78"""
    P, Pd, s = get_projector_left(ts, chi)
    newC1, newE4, newC4 = proj_left(ts, P, Pd)
    return up_left(ts, renormalize(newC1), renormalize(newE4), renormalize(newC4)), s


def right_rg(ts, chi):
    """ctmrg.jl:80-92"""
    P, Pd, s = get_projector_right(ts, chi)
    newC2, newE2, newC3 = proj_right(ts, P, Pd)
    return up_right(ts, renormalize(newC2), renormalize(newE2), renormalize(newC3)), s


def top_rg(ts, chi):
    """ctmrg.jl:94-106"""
    P, Pd, s = get_projector_top(ts, chi)
    newC1, newE1, newC2 = proj_top(ts, P, Pd)
    return up_top(ts, renormalize(newC1), renormalize(newE1), renormalize(newC2)), s


def bottom_rg(ts, chi):
    """ctmrg.jl:108-120"""
    P, Pd, s = get_projector_bottom(ts, chi)
    newC4, newE3, newC3 = proj_bottom(ts, P, Pd)
    return up_bottom(ts, renormalize(newC4), renormalize(newE3), renormalize(newC3)), s


def _prod3(x):
    return x.shape[0] * x.shape[1] * x.shape[2]


def get_projector_left(ts, chi):
    """ctmrg.jl:122-153 (plain C/T/A only, also in the nested move)."""
    C1, C4 = ts.Cs[0], ts.Cs[3]
    E1, E3, E4u, E4d = ts.Es[0], ts.Es[2], ts.Es[3], ts.Es[3]
    Au, Adu, Ad, Add = ts.A, ts.Ad, ts.A, ts.Ad
    C1E1 = tcon([C1, E1], [[-1, 1], [1, -2, -3, -4]])
    CEE4 = tcon([C1E1, E4u], [[1, -2, -5, -3], [1, -1, -6, -4]])
    CEEA = tcon([CEE4, Au], [[-1, -2, -3, -4, 1, 2], [1, 2, -5, -6, -7]])
    LU = tcon([CEEA, Adu], [[-1, -4, 1, 2, -2, -5, 3], [1, 2, -3, -6, 3]])
    R1 = permutedims(freshape(LU, _prod3(LU), -1), (2, 1))
    C4E3 = tcon([C4, E3], [[-1, 1], [1, -2, -3, -4]])
    CEE4 = tcon([C4E3, E4d], [[1, -2, -6, -4], [-1, 1, -5, -3]])
    CEEA = tcon([CEE4, Ad], [[-1, -2, -3, -4, 1, 2], [-5, 1, 2, -6, -7]])
    LB = tcon([CEEA, Add], [[-1, -4, 1, 2, -2, -5, 3], [-3, 1, 2, -6, 3]])
    R2 = freshape(LB, _prod3(LB), -1)
    return get_projector(R1, R2, chi)


def get_projector_right(ts, chi):
    """ctmrg.jl:155-186"""
    C2, C3 = ts.Cs[1], ts.Cs[2]
    E1, E2u, E2d, E3 = ts.Es[0], ts.Es[1], ts.Es[1], ts.Es[2]
    Au, Adu, Ad, Add = ts.A, ts.Ad, ts.A, ts.Ad
    C2E1 = tcon([C2, E1], [[1, -2], [-1, 1, -3, -4]])
    CEE2 = tcon([C2E1, E2u], [[-1, 1, -5, -3], [1, -2, -6, -4]])
    CEEA = tcon([CEE2, Au], [[-1, -2, -3, -4, 1, 2], [1, -5, -6, 2, -7]])
    RU = tcon([CEEA, Adu], [[-1, -4, 1, 2, -2, -5, 3], [1, -3, -6, 2, 3]])
    R1 = freshape(RU, _prod3(RU), -1)
    C3E3 = tcon([C3, E3], [[-1, 1], [-2, 1, -3, -4]])
    CEE2 = tcon([C3E3, E2d], [[1, -2, -5, -3], [-1, 1, -6, -4]])
    CEEA = tcon([CEE2, Ad], [[-1, -2, -5, -6, 1, 2], [-3, -4, 1, 2, -7]])
    RB = tcon([CEEA, Add], [[-1, -4, -2, -5, 1, 2, 3], [-3, -6, 1, 2, 3]])
    R2 = freshape(RB, _prod3(RB), -1)
    return get_projector(R1, R2, chi)


def get_projector_top(ts, chi):
    """ctmrg.jl:188-219"""
    C1, C2 = ts.Cs[0], ts.Cs[1]
    E1l, E1r, E2, E4 = ts.Es[0], ts.Es[0], ts.Es[1], ts.Es[3]
    Al, Adl, Ar, Adr = ts.A, ts.Ad, ts.A, ts.Ad
    C1E4 = tcon([C1, E4], [[1, -2], [1, -1, -3, -4]])
    CEE1 = tcon([C1E4, E1l], [[-1, 1, -6, -4], [1, -2, -5, -3]])
    CEEA = tcon([CEE1, Al], [[-1, -2, -5, -6, 1, 2], [1, 2, -3, -4, -7]])
    UL = tcon([CEEA, Adl], [[-1, -4, -2, -5, 1, 2, 3], [1, 2, -3, -6, 3]])
    R1 = freshape(UL, _prod3(UL), -1)
    C2E2 = tcon([C2, E2], [[-1, 1], [1, -2, -3, -4]])
    CEE1 = tcon([C2E2, E1r], [[1, -2, -6, -4], [-1, 1, -5, -3]])
    CEEA = tcon([CEE1, Ar], [[-1, -2, -5, -6, 1, 2], [1, -3, -4, 2, -7]])
    UR = tcon([CEEA, Adr], [[-1, -4, -2, -5, 1, 2, 3], [1, -3, -6, 2, 3]])
    R2 = freshape(UR, _prod3(UR), -1)
    return get_projector(R1, R2, chi)


def get_projector_bottom(ts, chi):
    """ctmrg.jl:221-252"""
    C3, C4 = ts.Cs[2], ts.Cs[3]
    E2, E3l, E3r, E4 = ts.Es[1], ts.Es[2], ts.Es[2], ts.Es[3]
    Al, Adl, Ar, Adr = ts.A, ts.Ad, ts.A, ts.Ad
    C4E4 = tcon([C4, E4], [[1, -2], [-1, 1, -3, -4]])
    CEE3 = tcon([C4E4, E3l], [[-1, 1, -5, -3], [1, -2, -6, -4]])
    CEEA = tcon([CEE3, Al], [[-1, -2, -5, -6, 1, 2], [-3, 1, 2, -4, -7]])
    BL = tcon([CEEA, Adl], [[-1, -4, -2, -5, 1, 2, 3], [-3, 1, 2, -6, 3]])
    R1 = freshape(BL, _prod3(BL), -1)
    C3E2 = tcon([C3, E2], [[1, -2], [-1, 1, -3, -4]])
    CEE3 = tcon([C3E2, E3r], [[-1, 1, -6, -4], [-2, 1, -5, -3]])
    CEEA = tcon([CEE3, Ar], [[-1, -2, -5, -6, 1, 2], [-3, -4, 1, 2, -7]])
    BR = tcon([CEEA, Adr], [[-1, -4, -2, -5, 1, 2, 3], [-3, -6, 1, 2, 3]])
    R2 = permutedims(freshape(BR, _prod3(BR), -1), (2, 1))
    return get_projector(R1, R2, chi)


def get_projector(R1, R2, chi):
    """ctmrg.jl:254-265: P1 = R2 V S^-1/2, P2 = S^-1/2 U' R1."""
    new_chi = min(chi, R1.shape[1])
    U, S, V = wrap_svd(R1 @ R2, new_chi)
    inv_sqrt_S = torch.diag(1.0 / torch.sqrt(S)).to(R1.dtype)
    P1 = R2 @ V @ inv_sqrt_S
    P2 = inv_sqrt_S @ U.mH @ R1
    return P1, P2, S


def _proj_E(E, A, Ad, P, Pd, ia, iad):
    """Shared body of newE in proj_* (ctmrg.jl:284-290 and analogues)."""
    EA = tcon([E, A], ia)
    EAAd = tcon([EA, Ad], iad)
    s = EAAd.size() if isinstance(EAAd, NestedTensor) else EAAd.shape
    EAAd = wrap_reshape(EAAd, s[0] * s[1] * s[2], s[3] * s[4] * s[5], s[6], -1)
    EPd = tcon([Pd, EAAd], [[-1, 1], [1, -2, -3, -4]])
    return tcon([EPd, P], [[-1, 1, -3, -4], [1, -2]])


def proj_left(ts, P, Pd):
    """ctmrg.jl:267-293"""
    A, Ad = get_all_A(ts), get_all_Ad(ts)
    C1, _, _, C4 = get_all_Cs(ts)
    E1, _, E3, E4 = get_all_Es(ts)
    C1E1 = tcon([C1, E1], [[-2, 1], [1, -1, -3, -4]])
    n1 = C1E1.size(1) if isinstance(C1E1, NestedTensor) else C1E1.shape[0]
    newC1 = wrap_permutedims(_matmul_r(wrap_reshape(C1E1, n1, -1), P), (2, 1))
    C4E3 = tcon([C4, E3], [[-1, 1], [1, -4, -2, -3]])
    n4 = C4E3.size(4) if isinstance(C4E3, NestedTensor) else C4E3.shape[3]
    newC4 = _matmul_l(Pd, wrap_reshape(C4E3, -1, n4))
    newE4 = _proj_E(E4, A, Ad, P, Pd,
                    [[-1, -3, 1, -6], [-2, 1, -4, -5, -7]],
                    [[-1, -2, -4, -5, -7, 1, 2], [-3, 1, -6, -8, 2]])
    return newC1, newE4, newC4


def proj_right(ts, P, Pd):
    """ctmrg.jl:295-320"""
    A, Ad = get_all_A(ts), get_all_Ad(ts)
    _, C2, C3, _ = get_all_Cs(ts)
    E1, E2, E3, _ = get_all_Es(ts)
    C2E1 = tcon([C2, E1], [[1, -2], [-1, 1, -3, -4]])
    n1 = C2E1.size(1) if isinstance(C2E1, NestedTensor) else C2E1.shape[0]
    newC2 = _matmul_r(wrap_reshape(C2E1, n1, -1), P)
    C3E3 = tcon([C3, E3], [[-1, 1], [-4, 1, -2, -3]])
    n4 = C3E3.size(4) if isinstance(C3E3, NestedTensor) else C3E3.shape[3]
    newC3 = _matmul_l(Pd, wrap_reshape(C3E3, -1, n4))
    newE2 = _proj_E(E2, A, Ad, P, Pd,
                    [[-1, -3, 1, -6], [-2, -5, -4, 1, -7]],
                    [[-1, -2, -4, -5, -7, 1, 2], [-3, -8, -6, 1, 2]])
    return newC2, newE2, newC3


def proj_top(ts, P, Pd):
    """ctmrg.jl:322-347"""
    A, Ad = get_all_A(ts), get_all_Ad(ts)
    C1, C2, _, _ = get_all_Cs(ts)
    E1, E2, _, E4 = get_all_Es(ts)
    C1E4 = tcon([C1, E4], [[1, -2], [1, -1, -3, -4]])
    n1 = C1E4.size(1) if isinstance(C1E4, NestedTensor) else C1E4.shape[0]
    newC1 = _matmul_r(wrap_reshape(C1E4, n1, -1), P)
    C2E2 = tcon([C2, E2], [[-1, 1], [1, -4, -2, -3]])
    n4 = C2E2.size(4) if isinstance(C2E2, NestedTensor) else C2E2.shape[3]
    newC2 = _matmul_l(Pd, wrap_reshape(C2E2, -1, n4))
    newE1 = _proj_E(E1, A, Ad, P, Pd,
                    [[-1, -3, 1, -6], [1, -2, -5, -4, -7]],
                    [[-1, -2, -4, -5, -7, 1, 2], [1, -3, -8, -6, 2]])
    return newC1, newE1, newC2


def proj_bottom(ts, P, Pd):
    """ctmrg.jl:349-375"""
    A, Ad = get_all_A(ts), get_all_Ad(ts)
    C1, C2, C3, C4 = get_all_Cs(ts)
    E1, E2, E3, E4 = get_all_Es(ts)
    C4E4 = tcon([C4, E4], [[1, -2], [-1, 1, -3, -4]])
    n1 = C4E4.size(1) if isinstance(C4E4, NestedTensor) else C4E4.shape[0]
    newC4 = _matmul_r(wrap_reshape(C4E4, n1, -1), P)
    C3E2 = tcon([C3, E2], [[1, -1], [-4, 1, -2, -3]])
    n4 = C3E2.size(4) if isinstance(C3E2, NestedTensor) else C3E2.shape[3]
    newC3 = wrap_permutedims(_matmul_l(Pd, wrap_reshape(C3E2, -1, n4)), (2, 1))
    newE3 = _proj_E(E3, A, Ad, P, Pd,
                    [[-1, -3, 1, -6], [-5, -2, 1, -4, -7]],
                    [[-1, -2, -4, -5, -7, 1, 2], [-8, -3, 1, -6, 2]])
    return newC4, newE3, newC3


def _matmul_r(X, P):
    return X * P if isinstance(X, NestedTensor) else X @ P


def _matmul_l(Pd, X):
    return Pd * X if isinstance(X, NestedTensor) else Pd @ X


def up_left(ts, C1, E4, C4):
    """ctmrg.jl:377-404 (plain and nested with shift(-px))."""
    if isinstance(C1, NestedTensor):
        px = ts.Params.get("px", 0.0)
        C1, E4, C4 = shift(C1, -px), shift(E4, -px), shift(C4, -px)
        return _up_nested(ts, {0: C1, 3: C4}, {3: E4})
    Cs = [C1, ts.Cs[1], ts.Cs[2], C4]
    Es = [ts.Es[0], ts.Es[1], ts.Es[2], E4]
    return ts.replace(Cs=Cs, Es=Es)


def up_right(ts, C2, E2, C3):
    """ctmrg.jl:406-433"""
    if isinstance(C2, NestedTensor):
        px = ts.Params.get("px", 0.0)
        C2, E2, C3 = shift(C2, px), shift(E2, px), shift(C3, px)
        return _up_nested(ts, {1: C2, 2: C3}, {1: E2})
    Cs = [ts.Cs[0], C2, C3, ts.Cs[3]]
    Es = [ts.Es[0], E2, ts.Es[2], ts.Es[3]]
    return ts.replace(Cs=Cs, Es=Es)


def up_top(ts, C1, E1, C2):
    """ctmrg.jl:435-461"""
    if isinstance(C1, NestedTensor):
        py = ts.Params.get("py", 0.0)
        C1, E1, C2 = shift(C1, -py), shift(E1, -py), shift(C2, -py)
        return _up_nested(ts, {0: C1, 1: C2}, {0: E1})
    Cs = [C1, C2, ts.Cs[2], ts.Cs[3]]
    Es = [E1, ts.Es[1], ts.Es[2], ts.Es[3]]
    return ts.replace(Cs=Cs, Es=Es)


def up_bottom(ts, C4, E3, C3):
    """ctmrg.jl:463-491"""
    if isinstance(C4, NestedTensor):
        py = ts.Params.get("py", 0.0)
        C4, E3, C3 = shift(C4, py), shift(E3, py), shift(C3, py)
        return _up_nested(ts, {3: C4, 2: C3}, {2: E3})
    Cs = [ts.Cs[0], ts.Cs[1], C3, C4]
    Es = [ts.Es[0], ts.Es[1], E3, ts.Es[3]]
    return ts.replace(Cs=Cs, Es=Es)


def _up_nested(ts, newC, newE):
    slots_C = [list(ts.Cs), list(ts.B_Cs), list(ts.Bd_Cs), list(ts.BB_Cs)]
    slots_E = [list(ts.Es), list(ts.B_Es), list(ts.Bd_Es), list(ts.BB_Es)]
    for k, X in newC.items():
        for c in range(4):
            slots_C[c][k] = X[c + 1]
    for k, X in newE.items():
        for c in range(4):
            slots_E[c][k] = X[c + 1]
    return ts.replace(Cs=slots_C[0], B_Cs=slots_C[1], Bd_Cs=slots_C[2], BB_Cs=slots_C[3],
                      Es=slots_E[0], B_Es=slots_E[1], Bd_Es=slots_E[2], BB_Es=slots_E[3])


# --------------------------------------------------------------------------
# Observables (src/graph/evaluation.jl)
# --------------------------------------------------------------------------


def get_gs_energy(ts, H):
    """evaluation.jl:15-29: E = tr(H_h rho_h)/tr rho_h + tr(H_v rho_v)/tr rho_v; returns (E, Na)."""
    roh, rov = get_dms(ts)
    Nh = wrap_tr(roh)
    Nv = wrap_tr(rov)
    Na = (Nh + Nv) / 2
    roh = roh / Nh
    rov = rov / Nv
    Eh = wrap_tr(_hmul(H[0], roh))
    Ev = wrap_tr(_hmul(H[1], rov))
    return Eh + Ev, Na


def get_es_energy(ts, H):
    """evaluation.jl:31-45: real part of component 4 of the nested energy."""
    roh, rov = get_dms(ts, only_gs=False)
    Nh = wrap_tr(roh[1]).real
    Nv = wrap_tr(rov[1]).real
    roh = roh * (1.0 / Nh)
    rov = rov * (1.0 / Nv)
    Eh = wrap_tr(NestedTensor([_hmul(H[0], x) for x in roh.data]))
    Ev = wrap_tr(NestedTensor([_hmul(H[1], x) for x in rov.data]))
    E = Eh + Ev
    return E[4].real


def _hmul(H, x):
    if x is None:
        return None
    dt = torch.promote_types(H.dtype, x.dtype)
    return H.to(dt) @ x.to(dt)


# --------------------------------------------------------------------------
# 4x4 plaquette energy (evaluation.jl:339-398, 443-518) and its ES driver
# (optim_es_h4.jl:133-168): H is the MPO list [s1, s2, s3, s4] of get_local_h
# --------------------------------------------------------------------------


def get_op_Ad4(s1, s2, s3, s4, A1d, A2d, A3d, A4d):
    """evaluation.jl:501-518: each Ad with its MPO factor, the virtual and
    Hamiltonian bonds fused."""
    op1 = tcon([s1, A1d], [[-6, 1, -4], [-1, -2, -3, -5, 1]])
    d = _shape(op1)
    op1 = wrap_reshape(op1, d[0], d[1], d[2], d[3] * d[4], d[5])
    op2 = tcon([s2, A2d], [[-2, -7, 1, -4], [-1, -3, -5, -6, 1]])
    d = _shape(op2)
    op2 = wrap_reshape(op2, d[0], d[1] * d[2], d[3] * d[4], d[5], d[6])
    op3 = tcon([s3, A3d], [[-1, -7, 1, -3], [-2, -4, -5, -6, 1]])
    d = _shape(op3)
    op3 = wrap_reshape(op3, d[0] * d[1], d[2] * d[3], d[4], d[5], d[6])
    op4 = tcon([s4, A4d], [[-4, -6, 1], [-1, -2, -3, -5, 1]])
    d = _shape(op4)
    op4 = wrap_reshape(op4, d[0], d[1], d[2], d[3] * d[4], d[5])
    return op1, op2, op3, op4


def _shape(x):
    return tuple((x[1] if isinstance(x, NestedTensor) else x).shape)


def _fuse3(x):
    d = _shape(x)
    return wrap_reshape(x, d[0] * d[1] * d[2], -1)


def energy_norm_4x4(C1, C2, C3, C4, E1l, E1r, E2u, E2d, E3l, E3r, E4u, E4d, A1, A2, A3, A4,
                    A1d, A2d, A3d, A4d, op1, op2, op3, op4):
    """evaluation.jl:443-498: <H_plaquette> and the norm of the 2x2 cluster."""
    C1E1 = tcon([C1, E1l], [[-1, 1], [1, -2, -3, -4]])
    CEE4 = tcon([C1E1, E4u], [[1, -2, -5, -3], [1, -1, -6, -4]])
    CEEA1 = tcon([CEE4, A1], [[-1, -2, -3, -4, 1, 2], [1, 2, -5, -6, -7]])
    e_LU = _fuse3(tcon([CEEA1, op1], [[-1, -4, 1, 2, -2, -5, 3], [1, 2, -3, -6, 3]]))
    n_LU = _fuse3(tcon([CEEA1, A1d], [[-1, -4, 1, 2, -2, -5, 3], [1, 2, -3, -6, 3]]))

    C4E3 = tcon([C4, E3l], [[-1, 1], [1, -2, -3, -4]])
    CEE4 = tcon([C4E3, E4d], [[1, -2, -6, -4], [-1, 1, -5, -3]])
    CEEA4 = tcon([CEE4, A4], [[-1, -2, -3, -4, 1, 2], [-5, 1, 2, -6, -7]])
    e_LB = _fuse3(tcon([CEEA4, op4], [[-1, -4, 1, 2, -2, -5, 3], [-3, 1, 2, -6, 3]]))
    n_LB = _fuse3(tcon([CEEA4, A4d], [[-1, -4, 1, 2, -2, -5, 3], [-3, 1, 2, -6, 3]]))

    C2E1 = tcon([C2, E1r], [[1, -2], [-1, 1, -3, -4]])
    CEE2 = tcon([C2E1, E2u], [[-1, 1, -5, -3], [1, -2, -6, -4]])
    CEEA2 = tcon([CEE2, A2], [[-1, -2, -3, -4, 1, 2], [1, -5, -6, 2, -7]])
    e_RU = _fuse3(tcon([CEEA2, op2], [[-1, -4, 1, 2, -2, -5, 3], [1, -3, -6, 2, 3]]))
    n_RU = _fuse3(tcon([CEEA2, A2d], [[-1, -4, 1, 2, -2, -5, 3], [1, -3, -6, 2, 3]]))

    C3E3 = tcon([C3, E3r], [[-1, 1], [-2, 1, -3, -4]])
    CEE2 = tcon([C3E3, E2d], [[1, -2, -5, -3], [-1, 1, -6, -4]])
    CEEA3 = tcon([CEE2, A3], [[-1, -2, -5, -6, 1, 2], [-3, -4, 1, 2, -7]])
    e_RB = _fuse3(tcon([CEEA3, op3], [[-1, -4, -2, -5, 1, 2, 3], [-3, -6, 1, 2, 3]]))
    n_RB = _fuse3(tcon([CEEA3, A3d], [[-1, -4, -2, -5, 1, 2, 3], [-3, -6, 1, 2, 3]]))

    e_left = tcon([wrap_permutedims(e_LU, [2, 1]), e_LB], [[-1, 1], [1, -2]])
    e_right = tcon([e_RU, e_RB], [[-1, 1], [1, -2]])
    energy = tcon([e_left, e_right], [[1, 2], [1, 2]])
    n_left = tcon([wrap_permutedims(n_LU, [2, 1]), n_LB], [[-1, 1], [1, -2]])
    n_right = tcon([n_RU, n_RB], [[-1, 1], [1, -2]])
    norm = tcon([n_left, n_right], [[1, 2], [1, 2]])
    return energy, norm


def get_gs_energy_4x4(ts, H):
    """evaluation.jl:339-356"""
    s1, s2, s3, s4 = H
    C1, C2, C3, C4 = ts.Cs
    E1, E2, E3, E4 = ts.Es
    A, Ad = ts.A, ts.Ad
    ops = get_op_Ad4(s1, s2, s3, s4, Ad, Ad, Ad, Ad)
    energy, norm = energy_norm_4x4(C1, C2, C3, C4, E1, E1, E2, E2, E3, E3, E4, E4, A, A, A, A,
                                   Ad, Ad, Ad, Ad, *ops)
    return energy / norm


def get_es_energy_4x4(ts, H):
    """evaluation.jl:358-398: component 4 of the nested energy over component 1 of the norm."""
    s1, s2, s3, s4 = H
    A, Ad = get_all_A(ts), get_all_Ad(ts)
    C1, C2, C3, C4 = get_all_Cs(ts)
    E1, E2, E3, E4 = get_all_Es(ts)
    px = ts.Params.get("px", 0.0)
    py = ts.Params.get("py", 0.0)
    A1, A2, A3, A4 = A, A, A, A
    A1d, A2d, A3d, A4d = Ad, Ad, Ad, Ad
    E1r = shift(E1, px)
    A2, A2d = shift(A2, px), shift(A2d, px)
    A3, A3d = shift(A3, px), shift(A3d, px)
    E3r = shift(E3, px)
    C2 = shift(C2, px)
    C3 = shift(C3, px)
    E2u = shift(E2, px)
    E2d = shift(E2, px)
    C4 = shift(C4, py)
    C3 = shift(C3, py)
    E3l = shift(E3, py)
    E3r = shift(E3r, py)
    E4d = shift(E4, py)
    E2d = shift(E2d, py)
    A4, A4d = shift(A4, py), shift(A4d, py)
    A3, A3d = shift(A3, py), shift(A3d, py)
    ops = get_op_Ad4(s1, s2, s3, s4, A1d, A2d, A3d, A4d)
    energy, norm = energy_norm_4x4(C1, C2, C3, C4, E1, E1r, E2u, E2d, E3l, E3r, E4, E4d, A1, A2, A3, A4,
                                   A1d, A2d, A3d, A4d, *ops)
    return energy[4] / norm[1]


def run_es_h4(ts, H, B):
    """optim_es_h4.jl:159-168"""
    ts1 = ts.replace(B=B, Bd=conj(B))
    ts1, _ = run_ctm(ts1, conv_fun=lambda t: get_es_energy_4x4(t, H) / get_all_norm(t)[0])
    return get_es_energy_4x4(ts1, H), ts1


def get_es_grad_h4(ts, H, Bi):
    """optim_es_h4.jl:133-157: (gH, gN) as flat complex vectors (column-major)."""
    B = freshape(Bi, *ts.A.shape)
    ts1 = ts.replace(B=B, Bd=conj(B))
    with torch.no_grad():
        ts1, _ = run_ctm(ts1, conv_fun=lambda t: get_es_energy_4x4(t, H) / get_all_norm(t)[0])
    ts1 = _detach_ts(ts1)
    p = dict(ts1.Params)
    p["max_iter"] = p.get("ad_max_iter", 4)
    ts1 = ts1.replace(Params=p)
    Bv = B.detach().clone().requires_grad_(True)
    y, ts2 = run_es_h4(ts1, H, Bv)
    (gH,) = torch.autograd.grad(y.real if torch.is_complex(y) else y, Bv)
    with torch.no_grad():
        Nb, gN = get_all_norm(_detach_ts(ts2))
    return freshape(gH.detach(), -1), freshape(gN.detach(), -1)


def tout_site(a, b):
    """honeycomb.jl:37-42: c[i,j,k,l] = a[i,j] b[k,l], reshaped to (d1 d2, d3 d4)."""
    a, b = _promote(a, b)
    c = tcon([a, b], [[-1, -2], [-3, -4]])
    s = c.shape
    return freshape(c, s[0] * s[1], s[2] * s[3])


def get_w_op():
    """honeycomb.jl:82-101 (the XX plaquette operator): (d^2, d^2, d^2, d^2), d = 4."""
    Ix, yz = tout(sI, sigmax), tout(sigmay, sigmaz)
    xI, zy = tout(sigmax, sI), tout(sigmaz, sigmay)
    wp = tout_site(tout_site(Ix, yz), tout_site(xI, zy))
    d = 4
    return freshape(wp, d * d, d * d, d * d, d * d)


def get_local_h(h):
    """local_h.jl:1-31: the plaquette operator h (d^2, d^2, d^2, d^2) as the MPO
    [s1, s2, s3, s4] by successive truncated SVDs (wrap_svd)."""
    h = h.to(_C128)
    dims = tuple(h.shape)
    d = int(round(math.sqrt(dims[0])))
    sl = []
    u, s, v = wrap_svd(freshape(h, dims[0], -1))
    sl.append(freshape(u * torch.sqrt(s).to(u.dtype), d, d, -1))
    sdots = torch.sqrt(s).to(v.dtype)[:, None] * v.mH
    for i in range(len(dims) - 2):
        dl = sdots.shape[0]
        sdots = freshape(sdots, dl * dims[i], -1)
        u, s, v = wrap_svd(sdots)
        sl.append(freshape(u * torch.sqrt(s).to(u.dtype), dl, d, d, -1))
        sdots = torch.sqrt(s).to(v.dtype)[:, None] * v.mH
    sl.append(freshape(sdots, sdots.shape[0], d, d))
    return sl


def run_wp(ts, wp, A1, A2, A3, A4):
    """optim_wp.jl:222-238: the plaquette operator and the norm of the 2x2
    cluster with its four sites A1..A4 (one of them the basis tensor B) in the
    fixed environment of ts (energy_norm_4x4, evaluation.jl:435-441)."""
    C1, C2, C3, C4 = ts.Cs
    E1, E2, E3, E4 = ts.Es
    s1, s2, s3, s4 = wp
    Ad = [conj(a) for a in (A1, A2, A3, A4)]
    ops = get_op_Ad4(s1, s2, s3, s4, *Ad)
    return energy_norm_4x4(C1, C2, C3, C4, E1, E1, E2, E2, E3, E3, E4, E4, A1, A2, A3, A4, *Ad, *ops)


def get_wp_grad(ts, wp_op, Bi, site=1):
    """optim_wp.jl:195-220: (gH, gN) of the plaquette operator and of the norm
    w.r.t. the basis tensor B placed at plaquette site ``site`` (Params["wp"]),
    as flat complex vectors (column-major).  Zygote's back((1, nothing)) of the
    complex pair is the gradient of the real part (dL/dRe + i dL/dIm), which is
    what torch returns for a real scalar."""
    A = ts.A.to(_C128)
    B = freshape(Bi.to(_C128), *A.shape).detach().clone().requires_grad_(True)
    wp = get_local_h(wp_op)
    Cs = [c.to(_C128) for c in ts.Cs]
    Es = [e.to(_C128) for e in ts.Es]
    t = ts.replace(Cs=Cs, Es=Es)
    sites = [A, A, A, A]
    sites[site - 1] = B
    e, n = run_wp(t, wp, *sites)
    (gH,) = torch.autograd.grad(e.real, B, retain_graph=True)
    (gN,) = torch.autograd.grad(n.real, B)
    return freshape(gH.detach(), -1), freshape(gN.detach(), -1), complex(e.detach()), complex(n.detach())


def optim_wp_columns(ts, wp_op, basis, cols, site=1):
    """The effH, effN columns of optim_wp (optim_wp.jl:164-166):
    effH[:, i] = basis' gH / 2, effN[:, i] = basis' gN / 2."""
    basis = basis.to(_C128)
    out = []
    for i in cols:
        gH, gN, _, _ = get_wp_grad(ts, wp_op, basis[:, i], site)
        out.append((basis.mH @ gH / 2, basis.mH @ gN / 2))
    return out


def get_wp_basis(effH, effN, basis):
    """optim_wp.jl:25-72: diagonalise the (hermitised) effH in the metric effN
    and split the basis into the positive- and negative-eigenvalue sectors
    (new basis = basis P vecs).  Returns (es, basis_p, basis_m)."""
    H = (effH + effH.mH) / 2
    N = (effN + effN.mH) / 2
    ev_N, P = torch.linalg.eigh(N)
    idx = torch.argsort(ev_N, descending=True)
    P = P[:, idx]
    N2 = P.mH @ N @ P
    H2 = P.mH @ H @ P
    H2 = (H2 + H2.mH) / 2
    N2 = (N2 + N2.mH) / 2
    # eigen(H2, N2) on plain matrices: the generalised (QZ) problem, as LAPACK ggev
    import scipy.linalg as sla
    es, vecs = sla.eig(H2.numpy(), N2.numpy())
    ixs = np.argsort(es.real, kind="stable")
    es, vecs = es[ixs], vecs[:, ixs]
    exci = basis.to(_C128).numpy() @ P.numpy() @ vecs
    return es, exci[:, es.real > 0.0], exci[:, es.real < 0.0]


def correlation_TM(ts, direction="h", N=10):
    """expectation.jl:193-220: transfer matrix of (E4, E2) or (E1, E3) and its
    eigenvalue magnitudes, descending (the full spectrum here; the reference
    takes the N largest with eigsolve)."""
    E1, E2, E3, E4 = ts.Es
    if direction == "h":
        TM = tcon([E4, E2], [[-1, -3, 1, 2], [-2, -4, 1, 2]])
    else:
        TM = tcon([E1, E3], [[-1, -3, 1, 2], [-2, -4, 1, 2]])
    d = TM.shape
    TM = freshape(TM, d[0] * d[1], -1)
    es = torch.linalg.eigvals(TM)
    es1 = torch.sort(es.abs(), descending=True).values
    return es1[:N], TM


def run_gs_h4(ts, H, A):
    """optim_gs_h4.jl:113-123: ad_max_iter iterations with the plaquette energy
    as convergence value, then get_gs_energy_4x4."""
    ts1 = ts.replace(A=A, Ad=conj(A))
    ts1, _ = run_ctm(ts1, conv_fun=lambda t: get_gs_energy_4x4(t, H))
    return get_gs_energy_4x4(ts1, H)


def energy_and_grad_h4(x, H, cfg):
    """The fg! of optim_gs_h4 (optim_gs_h4.jl:53-91): converge with the
    plaquette criterion (get_conv_boundary_h4, :100-110), then the pullback of
    run_gs_h4.  Returns (real(E), dE/dx)."""
    x = renormalize(x.detach())
    with torch.no_grad():
        ts = make_ctm_tensors(x, cfg)
        ts, _ = run_ctm(ts, conv_fun=lambda t: get_gs_energy_4x4(t, H))
    ts = _detach_ts(ts)
    p = dict(ts.Params)
    p["max_iter"] = p.get("ad_max_iter", 4)
    ts = ts.replace(Params=p)
    xv = x.clone().requires_grad_(True)
    y = run_gs_h4(ts, H, xv)
    yr = y.real if torch.is_complex(y) else y
    (g,) = torch.autograd.grad(yr, xv)
    return float(yr.item()), g.detach(), ts


def get_gs_norm(ts):
    """evaluation.jl:47-59"""
    n_dm = get_single_dm(*ts.Cs, *ts.Es)
    ndm_Ad = tcon([n_dm, ts.Ad], [[-1, -2, -3, -4, 1, 2, 3, 4], [1, 2, 3, 4, -5]])
    nrm0 = tcon([ndm_Ad, ts.A], [[1, 2, 3, 4, 5], [1, 2, 3, 4, 5]])
    return nrm0


def get_all_norm(ts):
    """evaluation.jl:61-77: returns (Nb, envB)."""
    A, Ad = get_all_A(ts), get_all_Ad(ts)
    Cs, Es = get_all_Cs(ts), get_all_Es(ts)
    n_dm = get_single_dm(*Cs, *Es)
    ndm_A = tcon([n_dm, A], [[1, 2, 3, 4, -1, -2, -3, -4], [1, 2, 3, 4, -5]])
    all_norm = tcon([ndm_A, Ad], [[1, 2, 3, 4, 5], [1, 2, 3, 4, 5]])
    envB = ndm_A[2] / all_norm[1]
    Nb = tcon([ndm_A[2], ts.Bd], [[1, 2, 3, 4, 5], [1, 2, 3, 4, 5]])
    Nb = Nb / all_norm[1]
    return Nb, envB


def get_single_dm(C1, C2, C3, C4, E1, E2, E3, E4):
    """evaluation.jl:110-122"""
    C1E1 = tcon([C1, E1], [[-1, 1], [1, -2, -3, -4]])
    CEC2 = tcon([C1E1, C2], [[-1, 1, -3, -4], [1, -2]])
    CECE4 = tcon([CEC2, E4], [[1, -2, -3, -5], [1, -1, -4, -6]])
    C4E3 = tcon([C4, E3], [[-1, 1], [1, -2, -3, -4]])
    CEC3 = tcon([C4E3, C3], [[-1, 1, -3, -4], [-2, 1]])
    CECE2 = tcon([CEC3, E2], [[-1, 1, -3, -5], [-2, 1, -4, -6]])
    return tcon([CECE4, CECE2], [[1, 2, -1, -2, -5, -6], [1, 2, -3, -4, -7, -8]])


def get_dms(ts, only_gs=True):
    """evaluation.jl:124-156"""
    if only_gs:
        A, Ad = ts.A, ts.Ad
        C1, C2, C3, C4 = ts.Cs
        E1, E2, E3, E4 = ts.Es
        ts_h = (C1, C2, C3, C4, E1, E1, E2, E3, E3, E4, A, A, Ad, Ad)
        ts_v = (C1, C2, C3, C4, E1, E2, E2, E3, E4, E4, A, A, Ad, Ad)
    else:
        A, Ad = get_all_A(ts), get_all_Ad(ts)
        C1, C2, C3, C4 = get_all_Cs(ts)
        E1, E2, E3, E4 = get_all_Es(ts)
        px = ts.Params.get("px", 0.0)
        py = ts.Params.get("py", 0.0)
        ts_h = (C1, shift(C2, px), shift(C3, px), C4, E1, shift(E1, px), shift(E2, px), E3,
                shift(E3, px), E4, A, shift(A, px), Ad, shift(Ad, px))
        ts_v = (C1, C2, shift(C3, py), shift(C4, py), E1, E2, shift(E2, py), shift(E3, py),
                E4, shift(E4, py), A, shift(A, py), Ad, shift(Ad, py))
    return get_dm_h(*ts_h), get_dm_v(*ts_v)


def get_dm_h(C1, C2, C3, C4, E1l, E1r, E2, E3l, E3r, E4, Al, Ar, Adl, Adr):
    """evaluation.jl:169-200"""
    C1E1 = tcon([C1, E1l], [[-1, 1], [1, -2, -3, -4]])
    LU = tcon([C1E1, Adl], [[-1, -2, -3, 1], [1, -4, -5, -6, -7]])
    C4E3 = tcon([C4, E3l], [[-1, 1], [1, -2, -3, -4]])
    CEE4 = tcon([E4, C4E3], [[-1, 1, -3, -5], [1, -2, -4, -6]])
    LB = tcon([CEE4, Al], [[-1, -2, 1, 2, -4, -5], [-3, 1, 2, -6, -7]])
    L = tcon([LB, LU], [[1, -2, 2, 3, 4, -3, -5], [1, -1, 2, 3, 4, -4, -6]])
    C2E1 = tcon([C2, E1r], [[1, -2], [-1, 1, -3, -4]])
    RU = tcon([C2E1, Ar], [[-1, -2, 1, -3], [1, -4, -5, -6, -7]])
    C3E3 = tcon([C3, E3r], [[-1, 1], [-2, 1, -3, -4]])
    CEE2 = tcon([C3E3, E2], [[1, -2, -3, -5], [-1, 1, -4, -6]])
    RB = tcon([CEE2, Adr], [[-1, -2, -3, -4, 1, 2], [-5, -6, 1, 2, -7]])
    R = tcon([RU, RB], [[-1, 1, 2, -3, 3, 4, -5], [1, -2, 3, 4, 2, -4, -6]])
    roh = tcon([L, R], [[1, 2, 3, 4, -1, -3], [1, 2, 3, 4, -2, -4]])
    d = (Al.size(5) if isinstance(Al, NestedTensor) else Al.shape[4])
    return wrap_reshape(roh, d * d, d * d)


def get_dm_v(C1, C2, C3, C4, E1, E2u, E2d, E3, E4u, E4d, Au, Ad, Adu, Add):
    """evaluation.jl:217-248"""
    C1E1 = tcon([C1, E1], [[-1, 1], [1, -2, -3, -4]])
    CEE4 = tcon([C1E1, E4u], [[1, -2, -3, -5], [1, -1, -4, -6]])
    UL = tcon([CEE4, Au], [[-1, -2, 1, 2, -3, -4], [1, 2, -5, -6, -7]])
    C2E2 = tcon([C2, E2u], [[-1, 1], [1, -2, -3, -4]])
    UR = tcon([C2E2, Adu], [[-1, -2, -3, 1], [-4, -5, -6, 1, -7]])
    U = tcon([UL, UR], [[-1, 1, 3, 4, -3, 2, -5], [1, -2, 2, 3, 4, -4, -6]])
    C4E3 = tcon([C4, E3], [[-1, 1], [1, -2, -3, -4]])
    CEE4 = tcon([C4E3, E4d], [[1, -2, -4, -6], [-1, 1, -3, -5]])
    BL = tcon([CEE4, Add], [[-1, -2, -3, -4, 1, 2], [-5, 1, 2, -6, -7]])
    C3E2 = tcon([C3, E2d], [[1, -2], [-1, 1, -3, -4]])
    BR = tcon([C3E2, Ad], [[-1, -2, 1, -3], [-4, -5, -6, 1, -7]])
    B = tcon([BL, BR], [[-1, 1, 2, 3, -4, 4, -6], [-2, 1, 4, -3, 2, 3, -5]])
    rov = tcon([U, B], [[1, 2, 3, 4, -1, -3], [1, 2, 3, 4, -2, -4]])
    d = (Au.size(5) if isinstance(Au, NestedTensor) else Au.shape[4])
    return wrap_reshape(rov, d * d, d * d)


def compute_gs_energy(A, H, cfg, log=None):
    """evaluation.jl:1-13: converge CTMRG from init_ctm1 with the energy criterion."""
    ts = make_ctm_tensors(A, cfg)
    ts, _ = run_ctm(ts, conv_fun=lambda x: get_gs_energy(x, H)[0], log=log)
    return get_gs_energy(ts, H)


# --------------------------------------------------------------------------
# E+grad unit (src/optimize/optim_gs.jl:53-143)
# --------------------------------------------------------------------------


def get_conv_boundary(x, H, cfg, log=None):
    """optim_gs.jl:120-131"""
    ts = make_ctm_tensors(x, cfg)
    ts, _ = run_ctm(ts, conv_fun=lambda t: get_gs_energy(t, H)[0], log=log)
    return ts


def run_gs(ts, H, A):
    """optim_gs.jl:133-143: ``ad_max_iter`` CTM iterations from a fixed env, then the energy."""
    ts1 = ts.replace(A=A, Ad=conj(A))
    ts1, _ = run_ctm(ts1, conv_fun=lambda t: get_gs_energy(t, H)[0])
    E, _ = get_gs_energy(ts1, H)
    return E


def energy_and_grad(x, H, cfg, log=None):
    """The body of ``fg!`` (optim_gs.jl:53-91) without the L-BFGS cache.

    Returns (real(E), dE/dx).  x is renormalised first (optim_gs.jl:55).
    """
    x = renormalize(x.detach())
    with torch.no_grad():
        ts = get_conv_boundary(x, H, cfg, log=log)
    ts = _detach_ts(ts)
    ad_cfg = dict(ts.Params)
    ad_cfg["max_iter"] = ad_cfg.get("ad_max_iter", 4)
    ts = ts.replace(Params=ad_cfg)
    xv = x.clone().requires_grad_(True)
    y = run_gs(ts, H, xv)
    yr = y.real if torch.is_complex(y) else y
    (g,) = torch.autograd.grad(yr, xv)
    return float(yr.item()), g.detach(), ts


def _detach_ts(ts):
    def d(x):
        return None if x is None else x.detach()
    return ts.replace(A=d(ts.A), Ad=d(ts.Ad), Cs=[d(c) for c in ts.Cs], Es=[d(e) for e in ts.Es],
                      B=d(ts.B), Bd=d(ts.Bd), B_Cs=[d(c) for c in ts.B_Cs], Bd_Cs=[d(c) for c in ts.Bd_Cs],
                      BB_Cs=[d(c) for c in ts.BB_Cs], B_Es=[d(c) for c in ts.B_Es],
                      Bd_Es=[d(c) for c in ts.Bd_Es], BB_Es=[d(c) for c in ts.BB_Es])


# --------------------------------------------------------------------------
# Excited states (src/optimize/optim_es.jl)
# --------------------------------------------------------------------------


def normalize_gs(ts):
    """optim_es.jl:212-222"""
    nrm = get_gs_norm(ts)
    A1 = ts.A / math.sqrt(abs(complex(nrm.item())))
    return ts.replace(A=A1, Ad=conj(A1))


def substract_gs_energy(ts, H):
    """optim_es.jl:224-234: H_i - (E0/2) I."""
    gs_E, _ = get_gs_energy(ts, H)
    e = float((gs_E / 2).real.item()) if torch.is_complex(gs_E) else float(gs_E.item() / 2)
    return [h - e * torch.eye(h.shape[0], dtype=h.dtype) for h in H]


def get_tangent_basis(ts):
    """optim_es.jl:236-258 ("default"): null space of vec(ndm_Ad)^T (D^4 d - 1 vectors)."""
    n_dm = get_single_dm(*ts.Cs, *ts.Es)
    ndm_Ad = tcon([n_dm, ts.Ad], [[-1, -2, -3, -4, 1, 2, 3, 4], [1, 2, 3, 4, -5]])
    row = freshape(ndm_Ad, 1, -1)
    # Julia nullspace: right singular vectors beyond the numerical rank (1 here).
    _, _, Vh = torch.linalg.svd(row.to(_C128), full_matrices=True)
    return Vh.mH[:, 1:]


def run_es(ts, H, B):
    """optim_es.jl:196-210"""
    ts1 = ts.replace(B=B, Bd=conj(B))
    ts1, _ = run_ctm(ts1, conv_fun=lambda t: get_es_energy(t, H) / get_all_norm(t)[0])
    E = get_es_energy(ts1, H)
    return E, ts1


def get_es_grad(ts, H, Bi, log=None):
    """optim_es.jl:167-194: returns (gH, gN) as flat complex vectors (column-major)."""
    B = freshape(Bi, *ts.A.shape)
    ts1 = ts.replace(B=B, Bd=conj(B))
    with torch.no_grad():
        ts1, _ = run_ctm(ts1, conv_fun=lambda t: get_es_energy(t, H) / get_all_norm(t)[0], log=log)
    ts1 = _detach_ts(ts1)
    p = dict(ts1.Params)
    p["max_iter"] = p.get("ad_max_iter", 4)
    ts1 = ts1.replace(Params=p)
    Bv = B.detach().clone().requires_grad_(True)
    y, ts2 = run_es(ts1, H, Bv)
    (gH,) = torch.autograd.grad(y, Bv)
    with torch.no_grad():
        Nb, gN = get_all_norm(_detach_ts(ts2))
    return freshape(gH.detach(), -1), freshape(gN.detach(), -1)


# --------------------------------------------------------------------------
# Models (src/model/basis.jl, honeycomb.jl, lee_gs.jl)
# --------------------------------------------------------------------------

Sx = torch.tensor([[0, 1], [1, 0]], dtype=_F64) / 2
Sy = torch.tensor([[0, -1j], [1j, 0]], dtype=_C128) / 2
Sz = torch.tensor([[1, 0], [0, -1]], dtype=_F64) / 2
SI = torch.eye(2, dtype=_F64)
sigmax = torch.tensor([[0, 1], [1, 0]], dtype=_F64)
sigmay = torch.tensor([[0, -1j], [1j, 0]], dtype=_C128)
sigmaz = torch.tensor([[1, 0], [0, -1]], dtype=_F64)
sI = SI


def _promote(a, b):
    dt = torch.promote_types(a.dtype, b.dtype)
    return a.to(dt), b.to(dt)


def tout(a, b):
    """basis.jl:16-21"""
    a, b = _promote(a, b)
    c = tcon([a, b], [[-1, -3], [-2, -4]])
    s = c.shape
    return freshape(c, s[0] * s[1], s[2] * s[3])


def ising(h=2.0):
    """basis.jl:23-29"""
    H = -tout(sigmax, sigmax) - h * tout(sigmaz, SI) / 2 / 2 - h * tout(SI, sigmaz) / 2 / 2
    return [H, H]


def heisenberg(Jz=1.0):
    """basis.jl:31-35 (complex dtype because Sy is complex; values are real)."""
    H = Jz * tout(Sz, Sz).to(_C128) - tout(Sx, Sx).to(_C128) - tout(Sy, Sy)
    return [H, H]


def honeycomb(Jx=1.0, Jy=1.0, Jz=1.0, dir="ZZ"):
    """honeycomb.jl:1-14"""
    if dir == "ZZ":
        hv = Jx * tout(tout(SI, sigmax), tout(sigmax, SI)) + (tout(tout(sigmaz, sigmaz), tout(SI, SI)) + tout(tout(SI, SI), tout(sigmaz, sigmaz))) / 2 / 2
        hh = Jy * tout(tout(SI, sigmay), tout(sigmay, SI)) + (tout(tout(sigmaz, sigmaz), tout(SI, SI)) + tout(tout(SI, SI), tout(sigmaz, sigmaz))) / 2 / 2
    elif dir == "XX":
        hv = Jy * tout(tout(SI, sigmay), tout(sigmay, SI)) + (tout(tout(sigmax, sigmax), tout(SI, SI)) + tout(tout(SI, SI), tout(sigmax, sigmax))) / 2 / 2
        hh = Jz * tout(tout(SI, sigmaz), tout(sigmaz, SI)) + (tout(tout(sigmax, sigmax), tout(SI, SI)) + tout(tout(SI, SI), tout(sigmax, sigmax))) / 2 / 2
    elif dir == "YY":
        hv = Jz * tout(tout(SI, sigmaz), tout(sigmaz, SI)) + (tout(tout(sigmay, sigmay), tout(SI, SI)) + tout(tout(SI, SI), tout(sigmay, sigmay))) / 2 / 2
        hh = Jx * tout(tout(SI, sigmax), tout(sigmax, SI)) + (tout(tout(sigmay, sigmay), tout(SI, SI)) + tout(tout(SI, SI), tout(sigmay, sigmay))) / 2 / 2
    else:
        raise ValueError(dir)
    hv = hv.real if hv.is_complex() else hv
    hh = hh.real if hh.is_complex() else hh
    return [-hh, -hv]


def get_Q_op():
    """lee_gs.jl:87-95"""
    Q = torch.zeros((2, 2, 2, 2, 2), dtype=_C128)
    Q[0, 0, 0] = SI.to(_C128)
    Q[0, 1, 1] = sigmax.to(_C128)
    Q[1, 0, 1] = sigmay
    Q[1, 1, 0] = sigmaz.to(_C128)
    return Q


def init_hb_gs(D=4, p1=0.24, p2=0.0, dir="ZZ"):
    """lee_gs.jl:2-28 (D=2 branch; D=4/8 apply act_R_op)."""
    Q_op = get_Q_op()
    ux = uy = uz = 1 / math.sqrt(3)
    s111 = torch.tensor([1 + uz, ux + 1j * uy], dtype=_C128) / math.sqrt(2 + 2 * uz)
    T = torch.einsum("abcdp,p->abcd", Q_op, s111)
    if dir == "ZZ":
        A = tcon([T, T], [[-1, -2, 1, -5], [-3, -4, 1, -6]])
    elif dir == "XX":
        A = tcon([T, T], [[1, -1, -2, -5], [1, -3, -4, -6]])
    elif dir == "YY":
        A = tcon([T, T], [[-2, 1, -1, -5], [-4, 1, -3, -6]])
    else:
        raise ValueError(dir)
    A = freshape(A, 2, 2, 2, 2, 4)
    if D == 4:
        A = act_R_op(A, p1=p1, dir=dir)
    if D == 8:
        A = act_R_op(act_R_op(A, p1=p1, dir=dir), p1=p2, dir=dir)
    return A


def act_R_op(A0, p1=0.24, dir="ZZ"):
    """lee_gs.jl:30-52"""
    phi = p1 * math.pi
    R = torch.zeros((2, 2, 2, 2, 2), dtype=_C128)
    R[0, 0, 0] = SI.to(_C128) * math.cos(phi)
    R[1, 0, 0] = (2 * Sx * math.sin(phi)).to(_C128)
    R[0, 1, 0] = 2 * Sy * math.sin(phi)
    R[0, 0, 1] = (2 * Sz * math.sin(phi)).to(_C128)
    if dir == "ZZ":
        RR = tcon([R, R], [[-1, -2, 1, -5, -7], [-3, -4, 1, -6, -8]])
    elif dir == "XX":
        RR = tcon([R, R], [[1, -1, -2, -5, -7], [1, -3, -4, -6, -8]])
    else:
        RR = tcon([R, R], [[-2, 1, -1, -5, -7], [-4, 1, -3, -6, -8]])
    d = RR.shape
    RR = freshape(RR, d[0], d[1], d[2], d[3], d[4] * d[5], d[6] * d[7])
    A = tcon([RR, A0], [[-1, -3, -5, -7, -9, 1], [-2, -4, -6, -8, 1]])
    D1, D2 = A.shape[0], A.shape[1]
    return freshape(A, D1 * D2, D1 * D2, D1 * D2, D1 * D2, A.shape[8])


def get_Q_ghz():
    """lee_gs.jl:119-136"""
    Q_op = get_Q_op()
    QQ = tcon([Q_op, Q_op], [[-1, -2, 1, -5, -7], [-3, -4, 1, -6, -8]])
    d = QQ.shape
    QQ = freshape(QQ, d[0], d[1], d[2], d[3], d[4] * d[5], d[6] * d[7])
    ghz = torch.zeros((2, 2, 2, 2), dtype=_C128)
    ghz[0, 0, 0, 0] = 1
    ghz[1, 1, 1, 1] = 1
    phi = math.pi / 4
    c2 = math.sqrt((1 + 1 / math.sqrt(3)) / 2)
    s2 = math.sqrt((1 - 1 / math.sqrt(3)) / 2)
    em, ep = complex(math.cos(-phi / 2), math.sin(-phi / 2)), complex(math.cos(phi / 2), math.sin(phi / 2))
    S = torch.tensor([[em * c2, -em * s2], [ep * s2, ep * c2]], dtype=_C128)
    ghz = torch.einsum("abcp,dp->abcd", ghz, S)
    gg = freshape(tcon([ghz, ghz], [[-1, -2, 1, -5], [-3, -4, 1, -6]]), 2, 2, 2, 2, 4)
    A = tcon([QQ, gg], [[-1, -3, -5, -7, -9, 1], [-2, -4, -6, -8, 1]])
    D1, D2 = A.shape[0], A.shape[1]
    return freshape(A, D1 * D2, D1 * D2, D1 * D2, D1 * D2, A.shape[8])


def default_config():
    """src/optimize/default_config.toml:1-49 (the keys the hot path reads)."""
    return {"gc": True, "dir": 0, "out_prefix": "test", "model": "test", "D": 2, "chi": 32,
            "min_iter": 4, "max_iter": 20, "ad_max_iter": 4, "rg_tol": 1e-6, "resume": False,
            "basis": False, "basis_t": "default", "basis_cut": 1e-3, "basis_name": 0,
            "es_resume": 1, "es_num": 0, "ad": True, "save": True, "part_save": False,
            "nrmB_cut": 1e-3, "wp": 1}


def random_A(D, d=2, seed=0, dtype=_F64):
    """Seeded synthetic input: i.i.d. N(0,1) (numpy default_rng), max|A| = 1, column-major order."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n = D ** 4 * d
    if dtype == _C128:
        flat = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    else:
        flat = rng.standard_normal(n)
    A = freshape(torch.tensor(flat, dtype=dtype), D, D, D, D, d)
    return A / A.abs().max()
