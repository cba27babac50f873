"""ephmc: B200-native HMC hot path of the Holstein-Peierls model (Python side).

Host-side mirror of the reference's C interface for the path
(simulation/organic_hmc.h, organic_dense_matrix.h, organic_bosons.h) over the
C ABI of libephmc_cuda.so.  PyTorch is only used as a device-memory provider;
the computation is the library's CUDA kernels.
"""
from ._lib import (FORCE_ADJOINT, FORCE_MIXED, FORCE_REFERENCE, MODES, EphmcError, Flags, load_library,
                   LIB_PATH)
from .context import Context, batch_eval, convert_params, lattice
from .trans_loc import TransLoc, contraction_matrix, conv_sigma_t, conv_sigma_w

__all__ = ["Context", "batch_eval", "TransLoc", "contraction_matrix", "conv_sigma_w", "conv_sigma_t", "convert_params", "lattice", "load_library", "EphmcError", "Flags", "FORCE_REFERENCE",
           "FORCE_ADJOINT", "FORCE_MIXED", "MODES", "LIB_PATH"]
