"""ctypes mirrors of the C structs declared in include/ecg.h.

The field order and types must match ecg.h exactly; tests/test_abi.py checks
the sizes against the compiled library.
"""
import ctypes as C

c_double_p = C.POINTER(C.c_double)


class RunConfig(C.Structure):
    """ecg_run_config: numeric mirror of RunConfig (core/run_config.hpp:2-55)."""

    _fields_ = [
        ("n_cell", C.c_int32 * 2),
        ("is_periodic", C.c_int32 * 2),
        ("prob_lo", C.c_double * 2),
        ("prob_hi", C.c_double * 2),
        ("max_step", C.c_int32),
        ("spatial_order", C.c_int32),
        ("toro_test", C.c_int32),
        ("problem", C.c_int32),
        ("riemann", C.c_int32),
        ("method", C.c_int32),
        ("slope_limiter", C.c_int32),
        ("field_boundary", C.c_int32),
        ("stop_time", C.c_double),
        ("gamma", C.c_double),
        ("cfl", C.c_double),
        ("imex_cfl", C.c_double),
        ("imex_acoustic_cfl_cap", C.c_double),
        ("imex_solver_tol", C.c_double),
        ("velocity_x", C.c_double),
        ("velocity_y", C.c_double),
        ("density_inner", C.c_double),
        ("density_outer", C.c_double),
        ("pressure", C.c_double),
        ("mach", C.c_double),
        ("blob_cx", C.c_double),
        ("blob_cy", C.c_double),
        ("blob_radius", C.c_double),
        ("vortex_cx", C.c_double),
        ("vortex_cy", C.c_double),
        ("isentropic_vortex_strength", C.c_double),
        ("riemann_interface_x", C.c_double),
        ("riemann_interface_y", C.c_double),
        ("imex_solver_max_iter", C.c_int32),
        ("imex_acoustic_startup", C.c_int32),
        ("imex_picard_iterations", C.c_int32),
        ("imex_picard_extra_iterations", C.c_int32),
    ]

    def copy(self):
        out = RunConfig()
        C.pointer(out)[0] = self
        return out

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if hasattr(v, "__len__") else v
        return d


class GpuOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("arith", C.c_int32),
        ("imex_precision", C.c_int32),
        ("mixed_inner_max_iter", C.c_int32),
        ("mixed_inner_rtol", C.c_double),
        ("mixed_max_refinements", C.c_int32),
        ("tile_x", C.c_int32),
        ("tile_y", C.c_int32),
        ("mixed_reorth", C.c_int32),
        ("stream", C.c_void_p),
        ("deterministic", C.c_int32),
        ("mixed_min_iterations", C.c_int32),
    ]


class Diagnostics(C.Structure):
    _fields_ = [("rho_min", C.c_double), ("pressure_min", C.c_double), ("nonfinite_count", C.c_int32)]


class Admissibility(C.Structure):
    _fields_ = [
        ("rho_min", C.c_double),
        ("pressure_min", C.c_double),
        ("internal_energy_min", C.c_double),
        ("nonfinite_count", C.c_int32),
        ("density_failure_count", C.c_int32),
        ("pressure_failure_count", C.c_int32),
        ("internal_energy_failure_count", C.c_int32),
    ]


class ImexTimestepDiag(C.Structure):
    _fields_ = [
        ("material_rate_max", C.c_double),
        ("acoustic_rate_max", C.c_double),
        ("acoustic_startup_used", C.c_int32),
        ("acoustic_cap_used", C.c_int32),
    ]


IMEX_DIAG_INT_FIELDS = [
    "solver_status",
    "linear_solver_status_last",
    "solver_iterations",
    "picard_pressure_solves_used",
    "source_picard_iterations_used",
    "kinetic_lag_update_count",
    "kinetic_lag_nonfinite_count",
    "pressure_matrix_rows",
    "pressure_matrix_nonzeros",
    "pressure_matrix_max_row_width",
    "density_denominator_floor_count",
    "nonfinite_count",
    "positivity_failure_count",
    "face_enthalpy_denominator_guard_count",
    "face_enthalpy_nonfinite_count",
    "energy_flux_nonfinite_count",
    "gmres_inner_iterations",
    "gmres_refinements",
]
IMEX_DIAG_REAL_FIELDS = [
    "solver_initial_residual",
    "solver_initial_rhs_norm",
    "solver_residual",
    "solver_relative_residual",
    "pressure_linear_residual_linf",
    "pressure_linear_residual_relative_linf",
    "kinetic_jacobian_abs_max",
    "pressure_matrix_symmetry_linf",
    "pressure_picard_delta_linf",
    "source_picard_delta_l2_relative_to_pmax",
    "pressure_energy_residual_before_linf",
    "coupled_residual_l1_final",
    "coupled_residual_linf_final",
    "coupled_residual_relative_linf_final",
    "pressure_energy_residual_l1",
    "pressure_energy_residual_linf",
    "pressure_energy_residual_relative_linf",
    "rho_min",
    "pressure_min",
    "internal_energy_min",
    "trial_density_min",
    "solved_pressure_min",
    "solved_pressure_max",
    "eos_pressure_min",
    "eos_pressure_max",
    "internal_energy_max",
    "momentum_correction_linf",
    "energy_correction_linf",
    "energy_flux_linf",
    "energy_flux_divergence_linf",
    "eq78_divergence_linf",
    "eq78_divergence_scaled_linf",
    "energy_closeout_delta_l1",
    "energy_closeout_delta_linf",
    "gmres_vector_bytes",
]


# fields after the reals, not in the reference
IMEX_DIAG_TAIL_FIELDS = ["gmres_fp64_fallbacks", "gmres_fp32_basis"]


class ImexDiag(C.Structure):
    _fields_ = ([(n, C.c_int32) for n in IMEX_DIAG_INT_FIELDS] + [(n, C.c_double) for n in IMEX_DIAG_REAL_FIELDS] +
                [(n, C.c_int32) for n in IMEX_DIAG_TAIL_FIELDS])

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class RunResult(C.Structure):
    _fields_ = [
        ("steps", C.c_int32),
        ("failed", C.c_int32),
        ("failure_code", C.c_int32),
        ("hllc_degenerate_star_count", C.c_int32),
        ("imex_solver_iterations_max", C.c_int32),
        ("time", C.c_double),
        ("dt_min", C.c_double),
        ("dt_max", C.c_double),
        ("dt_sum", C.c_double),
        ("diagnostics", Diagnostics),
    ]


class PaperOptions(C.Structure):
    _fields_ = [
        ("mode", C.c_int32),
        ("max_steps", C.c_int32),
        ("epsilon", C.c_double),
        ("fixed_dt", C.c_double),
    ]


class PaperResult(C.Structure):
    _fields_ = [
        ("steps", C.c_int32),
        ("solver_failure_count", C.c_int32),
        ("gmres_iterations_max", C.c_int32),
        ("enthalpy_guard_count", C.c_int32),
        ("nonfinite_count", C.c_int32),
        ("nonpositive_count", C.c_int32),
        ("passed", C.c_int32),
        ("pad", C.c_int32),
        ("final_time", C.c_double),
        ("pressure_residual_linf_max", C.c_double),
        ("pressure_relative_residual_linf_max", C.c_double),
        ("rho_min", C.c_double),
        ("pressure_min", C.c_double),
        ("density_l1_error", C.c_double),
        ("velocity_l1_error", C.c_double),
        ("pressure_l1_error", C.c_double),
        ("density_l2_error", C.c_double),
        ("velocity_l2_error", C.c_double),
        ("pressure_l2_error", C.c_double),
        ("density_linf_error", C.c_double),
        ("pressure_linf_error", C.c_double),
    ]


class OutputInfo(C.Structure):
    _fields_ = [
        ("step", C.c_int32),
        ("pad", C.c_int32),
        ("time", C.c_double),
        ("trial_density_min", C.c_double),
        ("trial_pressure_min", C.c_double),
        ("trial_internal_energy_min", C.c_double),
    ]


class BubbleMetrics(C.Structure):
    _fields_ = [(f, C.c_double) for f in (
        "rho_min", "rho_max", "pressure_min", "pressure_max", "internal_energy_min", "density_bubble_centroid_x",
        "density_bubble_centroid_y", "density_bubble_area", "density_bubble_area_threshold", "schlieren_max")] + [
        ("nonfinite_count", C.c_int32), ("pad", C.c_int32)]


class BubbleRun(C.Structure):
    _fields_ = [
        ("steps_accepted", C.c_int32),
        ("steps_rejected", C.c_int32),
        ("time", C.c_double),
        ("wall_time_sec", C.c_double),
        ("dt_min", C.c_double),
        ("dt_max", C.c_double),
        ("dt_mean", C.c_double),
        ("status", C.c_char_p),
        ("failure_category", C.c_char_p),
        ("snapshot_status", C.c_char_p),
        ("snapshot_dir", C.c_char_p),
        ("snapshot_times", C.c_char_p),
    ]


# euler.bdltv20_paper_t1_s2 settings (ecg_paper_mode)
PAPER_MODE = {
    "off": 0,
    "toro_x_exact_dirichlet_y_periodic_2d": 1,
    "toro_xy_exact_dirichlet_2d": 2,
    "gresho_exact_dirichlet_2d": 3,
    "isentropic_vortex_periodic_2d": 4,
    "advection_blob_periodic_2d": 5,
}


class BatchResult(C.Structure):
    _fields_ = [
        ("steps", C.c_int32),
        ("failed", C.c_int32),
        ("hllc_degenerate_star_count", C.c_int32),
        ("pad", C.c_int32),
        ("time", C.c_double),
        ("diagnostics", Diagnostics),
    ]


# enum values (ecg.h)
PROBLEM = {
    "advection_blob": 0,
    "toro1": 1,
    "gresho_vortex": 2,
    "riemann_quadrant": 3,
    "isentropic_vortex": 4,
    "shock_density_bubble_2d": 5,
    "shock_density_bubble_cylindrical_clawpack": 6,
    "shock_bubble_mach122": 7,  # no counterpart in the reference (ecg.h)
}
RIEMANN = {"rusanov": 0, "hllc": 1, "lowmach_hllc": 2, "xie_am_hllc_p": 3}
METHOD = {"explicit": 0, "imex": 1}
LIMITER = {"minmod": 0, "mc": 1, "vanleer": 2}
ARITH_FAST, ARITH_EXACT = 0, 1
IMEX_FP64, IMEX_MIXED = 0, 1

SOLVER_STATUS = [
    "not_run",
    "converged_absolute",
    "converged_relative",
    "linear_solve_not_converged",
    "gmres_breakdown_not_converged",
    "linear_residual_nonfinite",
    "source_map_pressure_row_nonfinite",
    "source_map_lagged_momentum_nonfinite",
    "density_denominator_floor_used",
    "unsupported_mpi_for_host_single_level_gmres",
]
