"""Host side of the plaquette drivers (CPU): get_local_h reproduces the
reference's MPO decomposition (local_h.jl:1-31) - the factors rebuild h, and
for the subtracted Hamiltonian the reference saved (basis.jld2) the
decomposition of the rebuilt h has the same bond dimensions."""
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_get_local_h_roundtrip_and_reference_bonds(pkg):
    p = np.load(os.path.join(GOLD, "ref_pins.npz"))
    H4 = [p[f"es_H{k}"] for k in range(1, 5)]
    h = np.einsum("abx,xcdy,yefz,zgh->abcdefgh", *H4).reshape(4, 4, 4, 4, order="F")
    sl = pkg.drivers.get_local_h(h)
    assert [x.shape for x in sl] == [x.shape for x in H4]
    r = np.einsum("abx,xcdy,yefz,zgh->abcdefgh", *sl).reshape(4, 4, 4, 4, order="F")
    assert np.abs(r - h).max() <= 1e-12 * np.abs(h).max()


def test_w_op_and_its_mpo_match_the_oracle(pkg):
    """The honeycomb XX plaquette operator of optim_wp (get_w_op,
    honeycomb.jl:82-101) on the host equals the oracle's restatement, and its
    get_local_h MPO rebuilds it (1e-12)."""
    import ipeps_oracle as O
    w = pkg.drivers.get_w_op()
    wo = O.get_w_op().numpy()
    assert w.shape == (16, 16, 16, 16)
    assert np.abs(w - wo).max() <= 1e-15
    sl = pkg.drivers.get_local_h(w)
    d = 4
    r = np.einsum("abx,xcdy,yefz,zgh->abcdefgh", *sl).reshape(d * d, d * d, d * d, d * d, order="F")
    assert np.abs(r - w).max() <= 1e-12 * np.abs(w).max()


def test_get_wp_basis_splits_the_basis_by_eigenvalue_sign(pkg):
    """get_wp_basis (optim_wp.jl:25-72) on a synthetic Hermitian pair: the two
    sectors together span the basis, and each is orthogonal to the other in the
    metric N (generalised eigenvectors of distinct eigenvalues)."""
    rng = np.random.default_rng(3)
    nb = 12
    X = rng.standard_normal((nb, nb)) + 1j * rng.standard_normal((nb, nb))
    N = X @ X.conj().T + nb * np.eye(nb)
    Hm = rng.standard_normal((nb, nb)) + 1j * rng.standard_normal((nb, nb))
    Hm = Hm + Hm.conj().T
    basis = np.linalg.qr(rng.standard_normal((20, nb)) + 1j * rng.standard_normal((20, nb)))[0]
    es, bp, bm = pkg.drivers.get_wp_basis(Hm, N, basis)
    assert bp.shape[1] + bm.shape[1] == nb
    assert np.all(es.real[: bm.shape[1]] < 0) and np.all(es.real[bm.shape[1]:] > 0)
    # coefficients in the basis: c = basis^H b; N-orthogonality of the sectors
    cp, cm = basis.conj().T @ bp, basis.conj().T @ bm
    assert np.abs(cm.conj().T @ N @ cp).max() <= 1e-9 * np.abs(N).max() * max(np.abs(cp).max(), 1) * max(
        np.abs(cm).max(), 1)
