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
