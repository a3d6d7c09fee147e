"""B200-native CTMRG engine for iPEPS.jl (the CTMRG hot path behind a C ABI).

Import through ``ipeps_b200`` (see ``load``): the directory name carries the
reference's ``.jl`` suffix, so it is registered under an importable name.
"""
from .host import (CTMTensors, Engine, IPEPSError, bottom_rg, compute_gs_energy, default_config,  # noqa: F401
                   get_all_norm, get_es_energy, get_gs_energy, get_gs_norm, left_rg, load_library,
                   rg_step, right_rg, run_ctm, top_rg, tcon, get_projector, energy_grad, fg, es_energy_grad, get_es_grad, LIB_PATH, EXPORTED,
                   load_config, get_dir, get_gs_name, get_basis_name, get_es_name,
                   get_gs_energy_4x4, get_es_energy_4x4, run_ctm_4x4, energy_grad_4x4, fg_h4, es_energy_grad_4x4,
                   get_es_grad_h4, get_wp_grad, orth, gemm_tf32x3)
from . import drivers, jld2, warmstart  # noqa: F401,E402
