"""ctypes binding of libfos.so (the C ABI declared in include/fos.h).

The library is built in-tree by ``fos.build`` (nvcc, sm_100a) into
``fos/_lib/libfos.so``.  There is no fallback: if the library is missing or a
call fails, a ``FosError`` is raised.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libfos.so")

MAX_NEIGHBORS = 32
MAX_PASSES = 64

STATUS = {0: "FOS_OK", 1: "FOS_E_ARG", 2: "FOS_E_CAPACITY", 3: "FOS_E_CUDA",
          4: "FOS_E_TIMEOUT", 5: "FOS_E_DEVICE", 6: "FOS_E_STATE"}


class FosError(RuntimeError):
    """Raised when a libfos entry point returns a non-zero status."""

    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        super().__init__(f"{where}: {STATUS.get(code, code)} {detail}".strip())


class FosParams(C.Structure):
    _fields_ = [
        ("domain_size", C.c_double), ("grid_res", C.c_int), ("power_beta", C.c_double),
        ("early_exit", C.c_int), ("min_jfa_passes", C.c_int), ("th_pass_delta", C.c_double),
        ("tie_lower_index", C.c_int), ("expected_face_scale", C.c_double), ("t_add", C.c_double),
        ("t_drop", C.c_double), ("ema_alpha", C.c_double), ("gap_fraction", C.c_double),
        ("max_displacement_frac", C.c_double), ("displacement_multiplier", C.c_double),
        ("eps", C.c_double), ("contact_tol", C.c_double), ("fsc_deadband", C.c_double),
    ]


class FosJfaFields(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "fsc", "fsc_ema", "face_ids", "face_counts", "neighbor_list", "neighbor_used_count",
        "neighbor_prev_scores", "labels", "label_filtered")]


class FosJfaStats(C.Structure):
    _fields_ = [
        ("num_passes", C.c_int), ("early_exit", C.c_int), ("changes", C.c_longlong * MAX_PASSES),
        ("jfa_res", C.c_int), ("voxel_size", C.c_float), ("mean_score", C.c_float),
        ("std_score", C.c_float), ("p_dir", C.c_int), ("p_und_accepted", C.c_int),
        ("overflow_count", C.c_int), ("overflow_pct", C.c_float), ("mean_fsc", C.c_float),
        ("min_fsc", C.c_int), ("max_fsc", C.c_int), ("mean_fsc_ema", C.c_float),
        ("finalize_iterations", C.c_int), ("face_pairs", C.c_int),
        ("max_row_candidates", C.c_int), ("zero_fsc_count", C.c_int),
    ]


class FosValidate(C.Structure):
    _fields_ = [("passed", C.c_int), ("asymmetric_pairs", C.c_int), ("overflow_count", C.c_int),
                ("self_loops", C.c_int)]


class FosFrameParams(C.Structure):
    _fields_ = [
        ("pbd_iters", C.c_int), ("pressure_iters", C.c_int), ("f_low", C.c_int),
        ("f_high", C.c_int), ("growth_pct", C.c_double), ("max_step_pct", C.c_double),
        ("adjustment_frames", C.c_int), ("bp_mode", C.c_int), ("warmstart_frames", C.c_int),
        ("zero_rate_thresh", C.c_double), ("r_min", C.c_double), ("r_max", C.c_double),
        ("pressure_k", C.c_double), ("pressure_exp", C.c_double),
        ("pressure_pair_cap", C.c_double), ("max_eq_nei", C.c_int),
        ("brownian_strength", C.c_double), ("seed", C.c_uint64), ("warmup_pbd", C.c_int),
        ("ou_jitter", C.c_int), ("jitter_rms", C.c_double), ("jitter_tau", C.c_double),
        ("dt", C.c_double), ("max_drift_fraction", C.c_double), ("jfa_warm_step", C.c_int),
    ]


class FosState(C.Structure):
    _fields_ = [("n", C.c_int)] + [(n, C.c_void_p) for n in (
        "pos", "rad", "rad_target", "local_max_depth", "delta_r", "cell_count", "cell_start",
        "cell_indices", "v_jit")]


class FosSkipSignals(C.Structure):
    _fields_ = [("n", C.c_int), ("out_of_band", C.c_int), ("zero_fsc", C.c_int),
                ("pad", C.c_int), ("r_mean", C.c_double), ("sigma_dr", C.c_double),
                ("vmax_dt", C.c_double), ("fsc_mean", C.c_double)]


class FosSurrogateStats(C.Structure):
    _fields_ = [("pairs", C.c_int), ("overflow", C.c_int), ("judged", C.c_int),
                ("exact", C.c_int), ("within1", C.c_int), ("stale_exact", C.c_int),
                ("stale_within1", C.c_int), ("abs_err", C.c_double),
                ("stale_abs_err", C.c_double)]


class FosEnsembleFoam(C.Structure):
    _fields_ = [("n", C.c_int), ("jfa_res", C.c_int), ("grid_res", C.c_int), ("f_low", C.c_int),
                ("f_high", C.c_int), ("r_min", C.c_double), ("r_max", C.c_double),
                ("seed", C.c_uint64)]


class FosEnsembleTuning(C.Structure):
    _fields_ = [("pass_block", C.c_int), ("voxel_block", C.c_int), ("coop_threads", C.c_int),
                ("coop_blocks_per_sm", C.c_int)]


class FosEnsembleView(C.Structure):
    _fields_ = [("nfoams", C.c_int), ("n_total", C.c_int)] + [(k, C.c_void_p) for k in (
        "pos", "rad", "rad_target", "local_max_depth", "delta_r", "fsc", "fsc_ema", "face_ids",
        "face_counts", "neighbor_list", "labels_a", "labels_b", "foam_of")]


SUR_FEATURES = 16
SUR_HIDDEN = 64
SUR_BINS = 11
SUR_PAIR_CAP = 96
SUR_NPARAM = 64 * 16 + 64 + 64 * 64 + 64 + 64 + 1
SUR_ABSOLUTE = 0
SUR_ANCHORED = 1

_P = C.c_void_p
_I = C.c_int
_F = C.c_float

# name -> argtypes (restype int unless listed in _RESTYPES)
SIGNATURES = {
    "fos_params_default": [C.POINTER(FosParams)],
    "fos_ctx_create": [C.POINTER(FosParams), _I, _I, _I, C.POINTER(_P)],
    "fos_ctx_destroy": [_P],
    "fos_set_params": [_P, C.POINTER(FosParams)],
    "fos_set_resolution": [_P, _I],
    "fos_get_resolution": [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_F)],
    "fos_jfa_fields": [_P, C.POINTER(FosJfaFields)],
    "fos_jfa_run": [_P, _P, _P, _I, _P],
    "fos_jfa_init": [_P, _P, _P, _I, _P],
    "fos_jfa_passes": [_P, _I, _P],
    "fos_jfa_majority_filter": [_P, _P],
    "fos_jfa_accumulate_faces": [_P, _I, _P],
    "fos_jfa_finalize": [_P, _P, _I, _P],
    "fos_jfa_update_ema": [_P, _I, _P],
    "fos_jfa_load_labels": [_P, _P, _P],
    "fos_jfa_stats": [_P, _I, _P, C.POINTER(FosJfaStats), _P],
    "fos_jfa_validate": [_P, _I, C.POINTER(FosValidate), _P],
    "fos_grid_clear": [_P, _P, _P],
    "fos_grid_count": [_P, _P, _P, _I, _P],
    "fos_grid_prefix_sum": [_P, _P, _P, _P],
    "fos_grid_copy_pointers": [_P, _P, _P, _P],
    "fos_grid_scatter": [_P, _P, _P, _P, _I, _P],
    "fos_grid_build": [_P, _P, _I, _P, _P, _P, _P],
    "fos_grid_build_noalloc": [_P, _I, _I, C.c_double, _P, _P, _P, _P],
    "fos_project_overlaps": [_P, _P, _P, _P, _P, _P, _I, _P],
    "fos_compute_max_overlap": [_P, _P, _P, _P, _P, _P, _P, _I, _P, C.POINTER(_F), _P],
    "fos_equilibrate_pressure": [_P, _I, _I, _P, _P, _P, _P, _F, _F, _F, _I, _F, _F, _I,
                                 C.POINTER(_F), C.POINTER(_I), _P],
    "fos_apply_brownian": [_P, _P, _I, _F, _F, C.c_uint64, C.c_uint32, _P],
    "fos_init_jitter_velocities": [_P, _P, _I, _P],
    "fos_compute_mean_radius": [_P, _P, _I, _P, _P],
    "fos_apply_jitter": [_P, _P, _P, _P, _I, _F, C.c_double, C.c_double, C.c_double, C.c_double,
                         C.c_uint64, C.c_uint32, _P],
    "fos_integrate_jitter": [_P, _P, _P, _I, _F, _P],
    "fos_set_fsc_targets": [_P, _P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _P],
    "fos_jfa_warm": [_P, _P, _P, _I, _I, _P],
    "fos_dirty_mark": [_P, _P, _P, _P, _P, _I, C.c_double, C.c_double, _I, _P, _P],
    "fos_dirty_count": [_P, _P, C.POINTER(_I), _P],
    "fos_topo_candidates": [_P, _P, _P, _P, _P, _P, _I, C.c_double, _I, _P, _P, _P, _P],
    "fos_topo_gabriel": [_P, _P, _P, _P, _P, _I, _I, C.c_double, _I, _I, C.c_double, _I, _P,
                         _P, _P, _P, _P],
    "fos_topo_batched": [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _I, C.c_double, C.c_double,
                         _I, _P, _P, _P, _P, _P],
    "fos_topo_knn": [_P, _P, _P, _P, _P, _P, _I, _I, C.c_double, _P, _P],
    "fos_topo_ema": [_P, _P, _P, _F, _I, _P],
    "fos_topo_update_radii": [_P, _P, _P, _F, _F, _F, _F, _F, _F, _I, _P],
    "fos_nudge_radii": [_P, _P, _P, _P, _I, _F, _F, _F, _F, _F, _I, _P],
    "fos_controller_stats": [_P, _P, _P, _P, _I, _I, _I, C.POINTER(_I), C.POINTER(_I),
                             C.POINTER(_I), C.POINTER(_F), C.POINTER(_F), _P],
    "fos_pressure_stats": [_P, _I, _P, C.POINTER(_F), C.POINTER(_F), _P],
    "fos_frame_params_default": [C.POINTER(FosFrameParams)],
    "fos_sim_init": [_P, C.POINTER(FosState), C.POINTER(FosFrameParams), _I, _P],
    "fos_frame": [_P, C.POINTER(FosState), C.POINTER(FosFrameParams), _I, _P],
    "fos_frame_graph": [_P, C.POINTER(FosState), C.POINTER(FosFrameParams), _I, _P],
    "fos_sim_set_counters": [_P, _I, _I, _P],
    "fos_frame_dynamics": [_P, C.POINTER(FosState), C.POINTER(FosFrameParams), _P],
    "fos_frame_measure": [_P, C.POINTER(FosState), C.POINTER(FosFrameParams), _I, _P],
    "fos_skip_signals": [_P, C.POINTER(FosState), _P, _P, _I, _I, C.POINTER(FosSkipSignals),
                         _P],
    "fos_frame_profile": [_P, C.POINTER(FosState), C.POINTER(FosFrameParams), _I,
                          C.POINTER(C.c_float), _P],
    "fos_frame_trace": [_P, C.POINTER(FosState), C.POINTER(FosFrameParams),
                        C.POINTER(C.c_longlong), _I, C.POINTER(_I), _P],
    "fos_sim_counters": [_P, C.POINTER(_I), C.POINTER(_I), _P],
    "fos_surrogate_create": [_I, _F, C.POINTER(_P)],
    "fos_surrogate_destroy": [_P],
    "fos_surrogate_set_weights": [_P, _P, _P, _P],
    "fos_surrogate_get_weights": [_P, _P, _P, _P],
    "fos_surrogate_cutoff": [_P],
    "fos_surrogate_train_step": [_P, _P, _P, _P, _I, _F, _P, _P],
    "fos_surrogate_gradient": [_P, _P, _P, _P, _I, _P, _P, _P],
    "fos_surrogate_forward": [_P, _P, _I, _P, _P],
    "fos_surrogate_pairs": [_P, _P, _P, _P, _I, _F, _P, _P, _P, _P],
    "fos_surrogate_pair_count": [_P, C.POINTER(_I), C.POINTER(_I), _P],
    "fos_surrogate_export": [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "fos_surrogate_predict": [_P, _P, _P, _P, _P, _P, _P],
    "fos_surrogate_stats": [_P, C.POINTER(FosSurrogateStats), _P],
    "fos_surrogate_set_mode": [_P, _I],
    "fos_frame_surrogate": [_P, C.POINTER(FosState), C.POINTER(FosFrameParams), _P, _I, _P],
    "fos_frame_surrogate_graph": [_P, C.POINTER(FosState), C.POINTER(FosFrameParams), _P, _I,
                                  _P],
    "fos_ensemble_create": [C.POINTER(FosParams), C.POINTER(FosFrameParams),
                            C.POINTER(FosEnsembleFoam), _I, _I, C.POINTER(_P)],
    "fos_ensemble_destroy": [_P],
    "fos_ensemble_view": [_P, C.POINTER(FosEnsembleView)],
    "fos_ensemble_offsets": [_P, _P, _P, _P],
    "fos_ensemble_init": [_P, _I, _P],
    "fos_ensemble_frame": [_P, _I, _P],
    "fos_ensemble_frame_graph": [_P, _I, _P],
    "fos_ensemble_set_tuning": [_P, C.POINTER(FosEnsembleTuning)],
    "fos_ensemble_set_multi_voxel": [_P, _I],
    "fos_ensemble_trace": [_P, C.POINTER(C.c_longlong), _I, C.POINTER(C.c_int), _P],
    "fos_ensemble_frame_surrogate": [_P, _P, _I, _P],
    "fos_ensemble_surrogate_mode": [_P, _I],
    "fos_ensemble_surrogate_stats": [_P, C.POINTER(FosSurrogateStats), _P],
    "fos_ensemble_get_tuning": [_P, C.POINTER(FosEnsembleTuning)],
    "fos_ensemble_autotune": [_P, _I, C.POINTER(FosEnsembleTuning), _P, _I, _P],
    "fos_ensemble_frame_index": [_P, C.POINTER(_I), _P],
    "fos_ensemble_launch_count": [_P],
    "fos_launch_count": [_P],
    "fos_device_error": [_P, C.POINTER(_I), _P],
    "fos_device_error_clear": [_P, _P],
    "fos_test_barrier_plan": [_P, _I, _P],
    "fos_set_jfa_staging": [_P, _I],
    "fos_surrogate_set_inference": [_P, _I],
    "fos_set_jfa_multi_voxel": [_P, _I],
    "fos_status_string": [_I],
    "fos_last_error": [],
}
_RESTYPES = {"fos_params_default": None, "fos_frame_params_default": None,
             "fos_launch_count": C.c_longlong, "fos_status_string": C.c_char_p,
             "fos_last_error": C.c_char_p, "fos_surrogate_cutoff": C.c_float,
             "fos_ensemble_launch_count": C.c_longlong}

_lib = None


def load(path: str = LIB_PATH):
    """Load libfos.so and attach signatures.  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FosError(3, "load", f"{path} not built; run fos.build.build() (nvcc, sm_100a)")
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, C.c_int)
    _lib = lib
    return lib


def check(rc: int, where: str):
    if rc != 0:
        detail = load().fos_last_error()
        raise FosError(rc, where, detail.decode() if detail else "")


def call(name: str, *args):
    rc = getattr(load(), name)(*args)
    check(rc, name)
    return rc
