"""The warm-start network's kernels on the GPU against torch FP32 references.

The BF16 tensor-core GEMM rounds its operands to BF16 and accumulates in
FP32, so the references round the same operands (torch .bfloat16().float())
and multiply in FP32: the remaining difference is the FP32 summation order.
Bars: GEMM 1e-5 relative (Frobenius); the network's loss 1e-5 relative and
every parameter gradient 2e-3 relative: the activations feeding each GEMM are
themselves FP32 results that differ from the reference's at ~1e-6, which can
move a value across a BF16 rounding boundary (one BF16 ulp is 3.9e-3), and
these flips compound over the three layers of the backward pass."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def bf(x):
    return x.to(torch.bfloat16).to(torch.float32)


def ref_gemm(opA, opB, A, B):
    A = torch.from_numpy(np.ascontiguousarray(A))
    B = torch.from_numpy(np.ascontiguousarray(B))
    a = bf(A) if opA == "N" else bf(A).T
    b = bf(B) if opB == "N" else bf(B).T
    return (a.double() @ b.double()).float().numpy()


@pytest.mark.parametrize("opA,opB,m,n,k", [("N", "N", 128, 128, 64), ("T", "N", 512, 512, 200),
                                          ("N", "T", 200, 4128, 512), ("T", "T", 77, 300, 129)])
def test_gemm_bf16_matches_reference(engine, pkg, opA, opB, m, n, k):
    rng = np.random.default_rng(m + n + k)
    A = rng.standard_normal((m, k) if opA == "N" else (k, m)).astype(np.float32)
    B = rng.standard_normal((k, n) if opB == "N" else (n, k)).astype(np.float32)
    C0 = rng.standard_normal((m, n)).astype(np.float32)
    C = pkg.host.gemm_bf16(opA, opB, A, B, alpha=1.5, beta=0.5, C=C0, engine=engine)
    R = 1.5 * ref_gemm(opA, opB, A, B) + 0.5 * C0
    assert np.linalg.norm(C - R) <= 1e-5 * np.linalg.norm(R), np.linalg.norm(C - R) / np.linalg.norm(R)


def ref_loss_grad(p, X, T, n_in, nh, n_out):
    """Forward and hand-written backward with the kernel's roundings."""
    o = np.cumsum([0, n_in * nh, nh, nh * nh, nh, nh * n_out, n_out])
    P = torch.from_numpy(p)
    W1 = P[o[0]:o[1]].reshape(nh, n_in).T
    b1 = P[o[1]:o[2]]
    W2 = P[o[2]:o[3]].reshape(nh, nh).T
    b2 = P[o[3]:o[4]]
    W3 = P[o[4]:o[5]].reshape(n_out, nh).T
    b3 = P[o[5]:o[6]]
    X = torch.from_numpy(X)
    T = torch.from_numpy(T)
    mm = lambda a, b: (bf(a).double() @ bf(b).double()).float()  # noqa: E731
    c = 0.7978845608028654

    def gelu(z):
        return 0.5 * z * (1 + torch.tanh(c * (z + 0.044715 * z ** 3)))

    def dgelu(z):
        t = torch.tanh(c * (z + 0.044715 * z ** 3))
        return 0.5 * (1 + t) + 0.5 * z * (1 - t * t) * c * (1 + 3 * 0.044715 * z * z)

    Z1 = mm(X, W1) + b1
    H1 = gelu(Z1)
    Z2 = mm(H1, W2) + b2
    H2 = gelu(Z2)
    Y = mm(H2, W3) + b3
    n = Y.numel()
    loss = float(((Y - T) ** 2).double().sum() / n)
    dY = 2 * (Y - T) / n
    gW3 = mm(H2.T, dY)
    gb3 = dY.sum(0)
    dZ2 = mm(dY, W3.T) * dgelu(Z2)
    gW2 = mm(H1.T, dZ2)
    gb2 = dZ2.sum(0)
    dZ1 = mm(dZ2, W2.T) * dgelu(Z1)
    gW1 = mm(X.T, dZ1)
    gb1 = dZ1.sum(0)
    parts = [gW1.T.reshape(-1), gb1, gW2.T.reshape(-1), gb2, gW3.T.reshape(-1), gb3]
    return loss, [x.numpy() for x in parts], o


def test_mlp_grad_matches_reference(engine, pkg):
    n_in, nh, n_out, B = 512, 512, 700, 96
    net = pkg.host.Mlp(n_in, nh, n_out, max_batch=128, seed=3, engine=engine)
    try:
        rng = np.random.default_rng(0)
        X = rng.standard_normal((B, n_in)).astype(np.float32)
        T = rng.standard_normal((B, n_out)).astype(np.float32)
        loss, g = net.grad(X, T)
        rl, rg, o = ref_loss_grad(net.params(), X, T, n_in, nh, n_out)
        assert abs(loss - rl) <= 1e-5 * abs(rl), (loss, rl)
        errs = [np.linalg.norm(g[o[i]:o[i + 1]] - r) / np.linalg.norm(r) for i, r in enumerate(rg)]
        assert max(errs) <= 2e-3, errs
    finally:
        net.close()


def test_mlp_training_fits(engine, pkg):
    """Adam on a smooth synthetic regression: the loss falls by 10x."""
    n_in, nh, n_out, B = 64, 128, 32, 128
    rng = np.random.default_rng(1)
    X = rng.standard_normal((B, n_in)).astype(np.float32)
    M = rng.standard_normal((n_in, n_out)).astype(np.float32) / 8
    T = np.tanh(X @ M).astype(np.float32)
    net = pkg.host.Mlp(n_in, nh, n_out, max_batch=B, seed=5, engine=engine)
    try:
        first = net.train_step(X, T, 1e-3)
        for _ in range(300):
            last = net.train_step(X, T, 1e-3)
        assert last < 0.1 * first, (first, last)
    finally:
        net.close()
