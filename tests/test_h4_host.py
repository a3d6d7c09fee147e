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


def test_evaluate_es_generalised_eigenproblem_and_cuts(pkg):
    """compute_es / evaluate_es (expectation.jl:13-56, 152-183) on a synthetic
    pair with known answers: N = X X^H, H = X diag(E) X^H has the generalised
    eigenvalues E; directions of N below nrmB_cut (a ratio to its largest
    eigenvalue) drop out, and an integer cut keeps the eigenvalues above the
    (cut+1)-th (Julia's 1-based ev_N[nrmB_cut+1])."""
    drv = pkg.drivers
    rng = np.random.default_rng(11)
    nb = 12
    X = rng.standard_normal((nb, nb)) + 1j * rng.standard_normal((nb, nb))
    E = np.sort(rng.uniform(-1.0, 2.0, nb))
    N = X @ X.conj().T
    H = X @ np.diag(E) @ X.conj().T
    es, vecs = drv.evaluate_es(H, N, 1e-12)
    assert np.allclose(es.real, E, atol=1e-9) and np.abs(es.imag).max() < 1e-9
    assert np.all(np.diff(es.real) >= 0)
    # each eigenvector solves H2 x = e N2 x on the selected subspace
    Hp, Np, P = drv._es_subspace(H, N, 1e-12)
    assert np.allclose(Hp @ vecs, (Np @ vecs) * es[None, :], atol=1e-8 * np.abs(Hp).max())
    assert np.allclose(drv.band_energies(H, N, 1e-12), E, atol=1e-9)
    # a nearly null direction of N (1e-8 of its largest eigenvalue) is cut at 1e-3
    w, Q = np.linalg.eigh(N)
    w2 = w.copy()
    w2[0] = 1e-8 * w.max()
    N2 = (Q * w2) @ Q.conj().T
    _, _, P2 = drv._es_subspace(H, N2, 1e-3)
    assert P2.shape[1] == nb - 1
    # integer cut: the 4 largest eigenvalues of N
    _, _, P4 = drv._es_subspace(H, N, 4)
    assert P4.shape[1] == 4
    top = np.sort(np.linalg.eigvalsh(N))[::-1][:4]
    assert np.allclose(np.sort(np.linalg.eigvalsh(P4.conj().T @ N @ P4))[::-1], top)
