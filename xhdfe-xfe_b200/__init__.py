"""B200-native fixed-effects absorber (drop-in for the reference's CUDA absorber).

The package directory name contains a hyphen, so it is imported through
``load_package()`` from the repository root helpers as ``xhdfe_xfe_b200``.
"""

from .absorber import (  # noqa: F401
    Absorber,
    AbsorberError,
    AbsorptionResult,
    FeComponentStats,
    FeRecoveryResult,
    GroupIndividualStructure,
    HeterogeneousSlopeTerm,
    OlsResult,
    absorb_fixed_effects,
    absorb_many,
    build_group_individual,
    cuda_backend_available,
    demean_raw,
    dense_ids,
    dense_ids_device,
    drop_singletons_device,
    drop_singletons_mask,
    first_pair_component_stats,
    make_options,
    partial_out,
    recover_fixed_effects,
    run_ols,
)
from .kss import KssSolver, kss_system, max_lanes, stable_sort_u64  # noqa: F401
from . import learned  # noqa: F401

__version__ = "1.0.0"
