"""B200-native symmetry-reduced crystallographic FFT (KRFFT) and SCFT diffusion step.

Host-side mirror of CrystallographicFFT.jl's plan/execute API over the C ABI of
libcfft_b200.so (include/cfft_b200.h).  Importing the package loads the native
library; there is no CPU fallback.
"""
from ._lib import LIB, CFFTError, LIB_PATH  # noqa: F401
from .symmetry import (  # noqa: F401
    SymOp, SpectralIndexing, apply_op, auto_L, available_groups, calc_spectral_asu, check_shift_invariance,
    count_special_positions, detect_centering_type, dual_ops, find_optimal_shift, fractal_tree, get_k_vector, get_ops,
    shift_ops_half_grid, optimal_L_phase1, optimal_L, optimal_L_isotropic, recommended_N, group_order,
    detect_centering, CenteringType, CentP, CentC, CentA, CentI, CentF, convert_op,
    strip_centering, MIRROR_ADAPTATION_TABLE, MirrorAdaptationEntry, get_mirror_adaptation, needs_basis_change,
    needs_dct_path,
)
from .plans import (  # noqa: F401
    forward_plans, backward_plans, plan_centering_fold, SubgridCenteringFoldPlan,
    DiffusionSolver, KRFFTPlan, PATH_AUTO, PATH_CENTERED, PATH_M2, PATH_M2Q, PATH_M7, execute_centered_ikrfft,
    execute_centered_krfft, execute_m2_q, execute_m7_scft, plan_m2_q, plan_m7_scft, PATH_FULLGRID,
    Diagonal, apply_diffusion_operator, calc_gradient_term, calc_matrix_q,
    CenteringPreFoldPlan, plan_centering_prefold, plan_krfft_prefold, execute_prefold_krfft,
    execute_centered_scft, execute_krfft, execute_m2_backward, execute_m2_scft, fft_reconstruct,
    fft_reconstruct_centered, fullgrid_to_subgrid, ifft_unrecon_centered, plan_centered_ikrfft, plan_centered_scft,
    plan_diffusion, plan_krfft, plan_krfft_centered, plan_m2_backward, plan_m2_scft, step_diffusion,
    subgrid_to_fullgrid, update_kernel, update_m2_kernel,
)

from .variants import (  # noqa: F401
    FractalLeaf, FractalTree, G0ASUBackwardPlan, StagedPm3mPlan, VariantKRFFTPlan, build_recursive_tree,
    calc_asu_tree, collect_leaves, tree_summary, execute_fractal_krfft, execute_fractal_krfft_v2,
    execute_fractal_krfft_v3, execute_g0asu_ikrfft, execute_g0asu_krfft, execute_general_g0asu_krfft,
    execute_recursive_krfft, execute_selective_krfft, execute_sparse_krfft, execute_staged, execute_staged_full,
    lookup_full_spectrum, plan_fractal_krfft, plan_fractal_krfft_v2, plan_fractal_krfft_v3, plan_krfft_g0asu,
    plan_krfft_g0asu_backward, plan_krfft_g0asu_general, plan_krfft_recursive, plan_krfft_selective,
    plan_krfft_sparse, plan_staged_pm3m, plan_staged_pm3m_full,
)

from .asu import (  # noqa: F401
    ASUBlock, ASUPoint, CrystallographicASU, InterleavedOrbit, analyze_interleaved_orbits, calc_asu,
    compute_full_orbit, pack_asu, pack_asu_interleaved, CFFTPlan, plan_cfft, mul, ldiv,
)

from .scft import SCFTSolver, initial_fields, plan_scft  # noqa: F401
from .batch import MultiPlanStep, autotune_path, autotune_plan  # noqa: F401
from .sno import GROUP_SLOTS, SNOContext, SpectralNeuralOperator  # noqa: F401

__version__ = "0.3.0"
