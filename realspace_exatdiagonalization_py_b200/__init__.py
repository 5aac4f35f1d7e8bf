"""B200-native symmetry-resolved exact diagonalization.

Drop-in for the hot path of ``realspace_exactdiagonalization_py``
(``symmetry_resolved_ed.py``): orbit catalog, sector bases, matrix-free and
matrix-mode Hamiltonians, sector eigen-solves and scans keep the reference's
names and signatures; the work runs in the sm_100a kernels of ``librsed.so``
(C ABI in ``include/rsed.h``).  Batched multi-sector solves, FP32-matvec
solves with FP64 refinement and a continuous-batching solver service sit
beside the plain API.
"""

from .autotune import Autotuner, candidate_configs, default_tuner
from .bits import (
    as_uint64_array,
    bitmask_of_site,
    decode_bit_mask_to_configuration,
    decode_bit_mask_to_configuration_inplace,
    empty_site_for_mask,
    empty_site_iter_for_mask,
    encode_configuration_to_bit_mask,
    filled_site_iter_for_mask,
    is_site_empty,
    is_site_occupied,
    n_occupied_for_mask,
    occupy_site_for_mask,
)
from .batched import BatchedSectorSolver, SolverConfig
from .correlators import (compute_odlro_map, compute_structure_factor_manifold_average_map,
                          compute_structure_factor_map, off_diagonal_long_range_order, static_structure_factor,
                          static_structure_factor_manifold_average, structure_factor_allowed_momenta,
                          structure_factor_manifold_allowed_momenta)
from .catalog import Symmetry_Orbit_Catalog, build_symmetry_orbit_catalog, update_orbit_stabilizer_phases
from .fock import expand_sector_state_to_fock_amplitudes, expand_sector_state_to_fock_dense, fock_overlaps
from .models import (
    CHECKERBOARD_TPP_DENOMINATOR,
    build_bosonic_fci_ed_data,
    build_fermionic_checkerboard_tb_model,
    build_fermionic_fci_ed_data,
    build_heisenberg_ed_data,
    build_heisenberg_second_quantized_model,
    build_phase_explore_fermionic_checkerboard_model,
    build_spinful_hubbard_ed_data,
    build_spinful_hubbard_second_quantized_model,
    build_zero_flux_bosonic_fci_second_quantized_model,
    build_zero_flux_fermionic_fci_second_quantized_model,
    default_fci_sectors,
    default_fci_sectors_fermionic,
    my_optimal_param,
    params_DNSheng,
    params_Sun_Gu_Katsura_Sarma,
)
from .observables import flux_charge_pump, flux_spectrum_flow, many_body_chern_number, many_body_position_phases
from .ed import (
    Symmetry_Resolved_ED_Data,
    build_ed_data,
    ed_scan,
    ed_scan_at_irrep_matrix,
    ed_scan_at_irrep_matrixfree,
    ed_scan_checkpoint_filename,
    full_ed,
    load_checkpoint,
    print_spectrum,
    save_checkpoint,
    solve_sectors_batched,
)
from .hamiltonian import (
    DeviceModel,
    MatrixFreeHamiltonian,
    apply_hamiltonian,
    apply_hamiltonian_with_threads,
    build_ed_Hamiltonian_symmetry_block,
    build_matrixfree_projection_table,
    hamiltonian_linear_operator,
)
from .lanczos import (
    LanczosBatch,
    LanczosParams,
    diagonalize_block_arpack,
    diagonalize_block_dense,
    diagonalize_block_matrixfree,
    refine,
)
from .serving import (FluxContext, ServedCheckpoints, ServingModel, SolveRequest, SolveResult, SolveServer,
                      latency_summary)
from .second_quantized_model import (
    Real_Space_Second_Quantized_Model,
    update_second_quantized_model_with_twisted_phases,
)
from .sector import (
    CanonicalMap,
    SectorSet,
    Symmetry_Sector_Basis,
    build_symmetry_sector_basis,
    get_canonical,
    populate_canonical_map,
    project_to_sector,
    project_to_unnormalized_sector,
)
from .symmetry import (
    COMPLEX_ONE,
    MAX_N_SITE_UINT64,
    Finite_Symmetry_Group,
    Mask,
    OneDim_Irrep,
    Particle_Statistics,
    Symmetry_Operation,
    apply_operation_to_mask,
    build_identity_group,
    build_identity_irrep_list,
    build_irrep_list,
    build_translation_group,
    build_translation_irrep_list,
    get_canonical_representative,
    group_order,
    hopping_phase_for_stats,
    rank_combination,
)

__version__ = "0.1.0"
