"""config.toml handling and result-file naming (CPU): load_config mirrors
TOML.parsefile with the default config as fallback (optim_gs.jl:1-12), and
the file names follow src/utility/io.jl."""
import os

import pytest

REF_TOML = "/root/reference/src/optimize/default_config.toml"


def test_default_config_when_file_missing(pkg, tmp_path):
    assert pkg.load_config(str(tmp_path / "absent.toml")) == pkg.default_config()
    assert pkg.load_config(None) == pkg.default_config()


def test_custom_toml(pkg, tmp_path):
    p = tmp_path / "cfg.toml"
    p.write_text('model = "hb"\nout_prefix = "run1"\nD = 3\nchi = 48\nmin_iter = 4\nmax_iter = 40\n'
                 'ad_max_iter = 4\nrg_tol = 1e-8\ndir = 0\nbasis_name = 0\npart_save = false\n')
    c = pkg.load_config(str(p))
    assert c["chi"] == 48 and c["rg_tol"] == 1e-8 and c["model"] == "hb"
    assert pkg.get_gs_name(c, cwd="/w") == "/w/simulation/hb_run1_D3_X48/gs.jld2"
    assert pkg.get_basis_name(c, cwd="/w") == "/w/simulation/hb_run1_D3_X48/basis.jld2"
    assert pkg.get_es_name(c, 0.1, 0, cwd="/w") == "/w/simulation/hb_run1_D3_X48/es_0.1_0.jld2"
    assert pkg.get_es_name(c, 1, 1.0, cwd="/w") == "/w/simulation/hb_run1_D3_X48/es_1_1.0.jld2"
    c["dir"] = "/data/out"
    assert pkg.get_gs_name(c) == "/data/out/gs.jld2"


@pytest.mark.skipif(not os.path.exists(REF_TOML), reason="reference tree not present")
def test_default_config_matches_reference_toml(pkg):
    assert pkg.load_config(REF_TOML) == pkg.default_config()


def test_optim_gs_resume_and_save(pkg, tmp_path):
    """resume from a gs.npz checkpoint in the run directory (its A and energy
    list are continued) and save after every step; the E+grad unit is a
    quadratic stand-in (CPU), so only the driver logic is exercised."""
    import numpy as np
    rng = np.random.default_rng(0)
    A0 = rng.standard_normal((2, 2, 2, 2, 2))
    target = rng.standard_normal(A0.shape)
    target /= np.linalg.norm(target)

    def fg(A, H, cfg, engine=None):
        a = A / np.linalg.norm(A)
        return float(-np.dot(a.ravel(), target.ravel())), -target.copy() / np.linalg.norm(A), None

    cfg = pkg.default_config()
    cfg.update(dir=str(tmp_path), resume=True, save=True)
    np.savez(tmp_path / "gs.npz", A=A0, energies=np.array([0.5, 0.25]), gradnorms=np.array([1.0, 0.5]))
    r = pkg.drivers.optim_gs(None, np.ones_like(A0), cfg, iterations=3, fg_fn=fg)
    assert r["energies"][:2] == [0.5, 0.25] and len(r["energies"]) >= 4
    saved = pkg.drivers.load_gs(str(tmp_path / "gs.npz"))
    assert saved["energies"] == r["energies"] and saved["A"].shape == A0.shape
