"""devil_b200 -- B200 (sm_100a) implementation of devil's per-gene
negative-binomial GLM path behind devil's own fit_devil / test_de surface.

The compute runs in libdevil_b200.so (hand-written CUDA for sm_100a behind
the C ABI of include/devil_b200.h); this package is the host-side mirror of
the R interface.
"""
from .api import (calculate_sf, cluster_blocks, compute_clustered_meat, compute_hessian,
                  compute_offset_vector, compute_sandwich, estimate_dispersion,
                  estimate_mom_dispersion, fit_devil, fit_devil_batch, fit_dispersion, fit_overdispersion_new, group_data,
                  init_beta,
                  nb_adjoint, normed_sum_sf, p_adjust, psinorm_sf, test_de, beta_fit)
from ._lib import Context, DevilError, context, load as load_library, LIB_PATH

__all__ = [
    "fit_devil", "fit_devil_batch", "test_de", "group_data", "calculate_sf", "normed_sum_sf", "psinorm_sf",
    "compute_offset_vector", "estimate_dispersion", "init_beta", "beta_fit",
    "estimate_mom_dispersion", "fit_dispersion", "fit_overdispersion_new", "compute_hessian", "compute_clustered_meat",
    "compute_sandwich", "cluster_blocks", "p_adjust", "nb_adjoint", "Context", "DevilError",
    "context", "load_library", "LIB_PATH",
]
