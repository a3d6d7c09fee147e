"""Heisenberg D=6 chi=144 (enlarged corners 5184 x 5184, 215 MB each): one
E+grad evaluation (3 CTMRG iterations, pullback of 2) runs within device
memory because the adjoint keeps only C/T and the projector factors per
iteration and recomputes the moves in the backward.  Checks: finite energy
and gradient, |E| within the energy bound of H, and the device memory in use
after the call (pool included) below 40 GB of the GPU's 180."""
import numpy as np
import pytest
import torch

import ipeps_oracle as O

pytestmark = pytest.mark.gpu


def test_d6_chi144_energy_grad_fits(engine, pkg):
    rng = np.random.default_rng(6)
    A = rng.standard_normal((6, 6, 6, 6, 2))
    A = np.asfortranarray(A / np.abs(A).max())
    H = [h.numpy() for h in O.heisenberg(1.0)]
    cfg = pkg.default_config()
    cfg.update(chi=144, min_iter=3, max_iter=3, rg_tol=0.0, ad_max_iter=2)
    E, g, info = pkg.fg(A, H, cfg, engine=engine)
    assert np.isfinite(E) and np.all(np.isfinite(g)) and np.linalg.norm(g) > 0
    assert abs(E) <= pkg.warmstart.energy_bound(H)
    free, total = torch.cuda.mem_get_info()
    used_gb = (total - free) / 2 ** 30
    print("D=6 chi=144: E = %.10f, device memory in use %.1f GB" % (E, used_gb))
    assert used_gb < 40.0, used_gb
