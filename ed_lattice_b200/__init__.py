"""ed_lattice_b200 -- B200 (sm_100a) engine for the EDlattice sector-Lanczos path.

The compute lives in libedgpu.so (CUDA, C ABI in include/edgpu.h); this package is the
host-side mirror of the reference's interfaces (see edlat.py) and the ctypes binding.
Importing it loads the library and raises if it is missing: there is no CPU fallback.
"""
from ._edgpu_lib import (EDG_FORM_DIRECT, EDG_FORM_STORED, EDG_GS_E0_ONLY, EDG_GS_F32_REFINE, EDG_GS_F64,
                         EDG_LK_F32_REFINE, EDG_LK_F64, EDG_PREC_F32, EDG_PREC_F64, EdgError, lib)
from .edlat import (Hij, Model, Sector, Spectrum, chi_chain, chi_chain_block, drude_weight, eval_chi, eval_gf, eval_oc,
                    gf_chain, gf_chain_block, grids, oc_chain, poles_weights, random_vector, read_gfmatrix,
                    release_cached_memory, ring, sp_lanc_eigh, square_lattice, tridiag_eigh, tridiag_Hv_sector,
                    tridiag_lowest, write_gfmatrix)

from .diag import DiagParams, StateList, diagonalize_lattice, lanc_energy, lanc_observables, partition_function

lib()  # load now: a missing or broken libedgpu.so fails the import

__all__ = [
    "EDG_FORM_DIRECT", "EDG_FORM_STORED", "EDG_GS_E0_ONLY", "EDG_GS_F32_REFINE", "EDG_GS_F64", "EDG_LK_F32_REFINE",
    "EDG_LK_F64", "EDG_PREC_F32",
    "EDG_PREC_F64", "DiagParams", "EdgError", "Hij", "StateList", "diagonalize_lattice", "lanc_energy", "lanc_observables",
    "partition_function", "Model", "Sector", "Spectrum", "chi_chain", "chi_chain_block", "drude_weight", "eval_chi",
    "eval_gf", "eval_oc", "gf_chain", "gf_chain_block", "grids", "oc_chain", "poles_weights", "random_vector", "read_gfmatrix",
    "release_cached_memory", "ring",
    "sp_lanc_eigh", "square_lattice", "tridiag_eigh", "tridiag_Hv_sector", "tridiag_lowest", "write_gfmatrix",
]
