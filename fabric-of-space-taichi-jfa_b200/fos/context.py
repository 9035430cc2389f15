"""Owner of one libfos context: the B200 counterpart of jfa.py's module fields.

A ``Context`` wraps the C handle (``fos_ctx_create``), exposes the context's
device fields as torch tensor views and calls every stage through the C ABI
on torch's current CUDA stream.  Caller tensors must be CUDA, contiguous and of
the reference's dtypes (pos [n,3] float32, rad [n] float32, cell arrays int32).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import FosJfaFields, FosJfaStats, FosValidate, call
from .config import FosConfig

S = _lib.MAX_NEIGHBORS


class _DevArray:
    """__cuda_array_interface__ shim so torch can view context-owned memory."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None, "stream": None}


def _view(ptr, shape, dtype: torch.dtype) -> torch.Tensor:
    typestr = {torch.int32: "<i4", torch.float32: "<f4"}[dtype]
    return torch.as_tensor(_DevArray(ptr, shape, typestr), device="cuda")


def ptr(t: torch.Tensor | None, dtype: torch.dtype | None = None, name: str = "tensor"):
    """Device pointer of a CUDA tensor (checked), or None."""
    if t is None:
        return None
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA torch tensor")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return C.c_void_p(t.data_ptr())


def stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class Context:
    def __init__(self, cfg: FosConfig, max_n: int | None = None, max_res: int | None = None,
                 device: int | None = None):
        lib = _lib.load()
        if not torch.cuda.is_available():
            raise _lib.FosError(3, "Context", "no CUDA device: libfos has no CPU path")
        self.cfg = cfg
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.max_n = int(max_n if max_n is not None else cfg.MAX_PARTICLES)
        self.max_res = int(max_res if max_res is not None else max(cfg.JFA_RES, 2))
        self._p = cfg.params()
        h = C.c_void_p()
        call("fos_ctx_create", C.byref(self._p), self.max_n, self.max_res, self.device, C.byref(h))
        self.h = h
        self._lib = lib
        self.set_resolution(cfg.JFA_RES)
        f = FosJfaFields()
        call("fos_jfa_fields", self.h, C.byref(f))
        n = self.max_n
        self.fsc = _view(f.fsc, (n,), torch.int32)
        self.fsc_ema = _view(f.fsc_ema, (n,), torch.float32)
        self.face_ids = _view(f.face_ids, (n, S), torch.int32)
        self.face_counts = _view(f.face_counts, (n, S), torch.int32)
        self.neighbor_list = _view(f.neighbor_list, (n, S), torch.int32)
        self.neighbor_used_count = _view(f.neighbor_used_count, (n,), torch.int32)
        self.neighbor_prev_scores = _view(f.neighbor_prev_scores, (n, S), torch.float32)

    # ------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "h", None):
            self._lib.fos_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, cfg: FosConfig):
        self.cfg = cfg
        self._p = cfg.params()
        call("fos_set_params", self.h, C.byref(self._p))

    def set_resolution(self, res: int):
        call("fos_set_resolution", self.h, int(res))
        r, p, v = C.c_int(), C.c_int(), C.c_float()
        call("fos_get_resolution", self.h, C.byref(r), C.byref(p), C.byref(v))
        self.res, self.num_passes, self.voxel_size = r.value, p.value, v.value

    def launch_count(self) -> int:
        return int(self._lib.fos_launch_count(self.h))

    def device_error(self) -> int:
        w = C.c_int()
        call("fos_device_error", self.h, C.byref(w), stream())
        return w.value

    def clear_device_error(self):
        """Clear the device error word after a failed launch has ended."""
        call("fos_device_error_clear", self.h, stream())

    def test_barrier_plan(self, leave_at_barrier: int):
        """For failure-path tests: later cooperative launches lose one block at
        grid barrier `leave_at_barrier` (>= 2) and their waits give up after
        ~1 ms with FOS_E_TIMEOUT; 0 turns it off."""
        call("fos_test_barrier_plan", self.h, int(leave_at_barrier), stream())

    def set_jfa_staging(self, on: bool):
        """JFA passes with record rows staged in shared memory by TMA copies, or
        read from global memory (the default); the labels are the same."""
        call("fos_set_jfa_staging", self.h, int(bool(on)))

    def set_jfa_multi_voxel(self, mode: int):
        """JFA record passes: 0 one voxel a thread, 1 four along x where the
        grid fills the GPU (default), 2 always four; the labels are the same."""
        call("fos_set_jfa_multi_voxel", self.h, int(mode))

    # ----------------------------------------------------------------- JFA
    def labels(self) -> torch.Tensor:
        """Final owner grid of the last run, [R, R, R] int32 (view)."""
        f = FosJfaFields()
        call("fos_jfa_fields", self.h, C.byref(f))
        r = self.res
        return _view(f.labels, (r, r, r), torch.int32)

    def label_filtered(self) -> torch.Tensor:
        f = FosJfaFields()
        call("fos_jfa_fields", self.h, C.byref(f))
        r = self.res
        return _view(f.label_filtered, (r, r, r), torch.int32)

    def jfa_run(self, pos, rad, n: int):
        call("fos_jfa_run", self.h, ptr(pos, torch.float32, "pos"), ptr(rad, torch.float32, "rad"),
             int(n), stream())

    def jfa_init(self, pos, rad, n):
        call("fos_jfa_init", self.h, ptr(pos, torch.float32, "pos"), ptr(rad, torch.float32, "rad"),
             int(n), stream())

    def jfa_passes(self, n):
        call("fos_jfa_passes", self.h, int(n), stream())

    def majority_filter(self):
        call("fos_jfa_majority_filter", self.h, stream())

    def accumulate_faces(self, n):
        call("fos_jfa_accumulate_faces", self.h, int(n), stream())

    def finalize(self, rad, n):
        call("fos_jfa_finalize", self.h, ptr(rad, torch.float32, "rad"), int(n), stream())

    def update_ema(self, n):
        call("fos_jfa_update_ema", self.h, int(n), stream())

    def load_labels(self, labels: torch.Tensor):
        call("fos_jfa_load_labels", self.h, ptr(labels, torch.int32, "labels"), stream())

    def jfa_stats(self, n: int, rad) -> dict:
        st = FosJfaStats()
        call("fos_jfa_stats", self.h, int(n), ptr(rad, torch.float32, "rad"), C.byref(st), stream())
        V = float(self.res ** 3)
        hist = [st.changes[p] / max(1.0, V) for p in range(st.num_passes)]
        return {
            "num_passes": st.num_passes, "early_exit": bool(st.early_exit),
            "delta_history": hist, "jfa_res": st.jfa_res, "voxel_size": st.voxel_size,
            "mean_score": st.mean_score, "std_score": st.std_score, "valid_pairs_pct": 100.0,
            "p_dir": st.p_dir, "p_und_accepted": st.p_und_accepted,
            "overflow_count": st.overflow_count, "overflow_pct": st.overflow_pct,
            "mean_fsc": st.mean_fsc, "min_fsc": st.min_fsc, "max_fsc": st.max_fsc,
            "mean_fsc_ema": st.mean_fsc_ema,
            "finalize_iterations": st.finalize_iterations, "face_pairs": st.face_pairs,
            "max_row_candidates": st.max_row_candidates, "zero_fsc_count": st.zero_fsc_count,
            "label_changes": [int(st.changes[p]) for p in range(st.num_passes)],
        }

    def validate(self, n: int) -> dict:
        v = FosValidate()
        call("fos_jfa_validate", self.h, int(n), C.byref(v), stream())
        return {"passed": bool(v.passed), "asymmetric_pairs": v.asymmetric_pairs,
                "overflow_count": v.overflow_count, "self_loops": v.self_loops}

    # ---------------------------------------------------------------- grid
    def grid_clear(self, cell_count):
        call("fos_grid_clear", self.h, ptr(cell_count, torch.int32, "cell_count"), stream())

    def grid_count(self, pos, cell_count, n):
        call("fos_grid_count", self.h, ptr(pos, torch.float32, "pos"),
             ptr(cell_count, torch.int32, "cell_count"), int(n), stream())

    def grid_prefix_sum(self, cell_count, cell_start):
        call("fos_grid_prefix_sum", self.h, ptr(cell_count, torch.int32, "cell_count"),
             ptr(cell_start, torch.int32, "cell_start"), stream())

    def grid_copy_pointers(self, cell_start, cell_write):
        call("fos_grid_copy_pointers", self.h, ptr(cell_start, torch.int32, "cell_start"),
             ptr(cell_write, torch.int32, "cell_write"), stream())

    def grid_scatter(self, pos, cell_write, cell_indices, n):
        call("fos_grid_scatter", self.h, ptr(pos, torch.float32, "pos"),
             ptr(cell_write, torch.int32, "cell_write"),
             ptr(cell_indices, torch.int32, "cell_indices"), int(n), stream())

    def grid_build(self, pos, n, cell_count, cell_start, cell_indices):
        call("fos_grid_build", self.h, ptr(pos, torch.float32, "pos"), int(n),
             ptr(cell_count, torch.int32, "cell_count"), ptr(cell_start, torch.int32, "cell_start"),
             ptr(cell_indices, torch.int32, "cell_indices"), stream())

    # ------------------------------------------------------------ dynamics
    def project_overlaps(self, pos, rad, cell_start, cell_count, cell_indices, n):
        call("fos_project_overlaps", self.h, ptr(pos, torch.float32, "pos"),
             ptr(rad, torch.float32, "rad"), ptr(cell_start, torch.int32, "cell_start"),
             ptr(cell_count, torch.int32, "cell_count"),
             ptr(cell_indices, torch.int32, "cell_indices"), int(n), stream())

    def compute_max_overlap(self, pos, rad, cell_start, cell_count, cell_indices,
                            local_max_depth, n, sync: bool = True):
        out = C.c_float(0.0)
        call("fos_compute_max_overlap", self.h, ptr(pos, torch.float32, "pos"),
             ptr(rad, torch.float32, "rad"), ptr(cell_start, torch.int32, "cell_start"),
             ptr(cell_count, torch.int32, "cell_count"),
             ptr(cell_indices, torch.int32, "cell_indices"),
             ptr(local_max_depth, torch.float32, "local_max_depth"), int(n), None,
             C.byref(out) if sync else None, stream())
        return float(out.value) if sync else None

    def equilibrate_pressure(self, n, frame, rad, delta_r, face_ids, fsc, k, P_exp, pair_cap,
                             max_nei, r_min, r_max, sweeps: int = 1, sync: bool = True):
        mx, ch = C.c_float(0.0), C.c_int(0)
        call("fos_equilibrate_pressure", self.h, int(n), int(frame),
             ptr(rad, torch.float32, "rad"), ptr(delta_r, torch.float32, "delta_r"),
             ptr(face_ids, torch.int32, "face_ids"), ptr(fsc, torch.int32, "fsc"), float(k),
             float(P_exp), float(pair_cap), int(max_nei), float(r_min), float(r_max), int(sweeps),
             C.byref(mx) if sync else None, C.byref(ch) if sync else None, stream())
        return (float(mx.value), int(ch.value)) if sync else None

    def apply_brownian(self, pos, n, strength, domain_size, seed, frame):
        call("fos_apply_brownian", self.h, ptr(pos, torch.float32, "pos"), int(n), float(strength),
             float(domain_size), int(seed) & 0xFFFFFFFFFFFFFFFF, int(frame) & 0xFFFFFFFF, stream())

    def init_jitter_velocities(self, v_jit, n):
        call("fos_init_jitter_velocities", self.h, ptr(v_jit, torch.float32, "v_jit"), int(n),
             stream())

    def compute_mean_radius(self, rad, n, mean_radius):
        call("fos_compute_mean_radius", self.h, ptr(rad, torch.float32, "rad"), int(n),
             ptr(mean_radius, torch.float32, "mean_radius"), stream())

    def apply_jitter(self, v_jit, rad, mean_radius, n, dt, rms, tau, max_drift, gap, seed, frame):
        call("fos_apply_jitter", self.h, ptr(v_jit, torch.float32, "v_jit"),
             ptr(rad, torch.float32, "rad"), ptr(mean_radius, torch.float32, "mean_radius"),
             int(n), float(dt), float(rms), float(tau), float(max_drift), float(gap),
             int(seed) & 0xFFFFFFFFFFFFFFFF, int(frame) & 0xFFFFFFFF, stream())

    def integrate_jitter(self, pos, v_jit, n, dt):
        call("fos_integrate_jitter", self.h, ptr(pos, torch.float32, "pos"),
             ptr(v_jit, torch.float32, "v_jit"), int(n), float(dt), stream())

    def set_fsc_targets(self, rad, rad_target, fsc, fsc_ema, n, f_low, f_high, growth_pct,
                        r_min, r_max):
        call("fos_set_fsc_targets", self.h, ptr(rad, torch.float32, "rad"),
             ptr(rad_target, torch.float32, "rad_target"), ptr(fsc, torch.int32, "fsc"),
             ptr(fsc_ema, torch.float32, "fsc_ema"), int(n), int(f_low), int(f_high),
             float(growth_pct), float(r_min), float(r_max), stream())

    def nudge_radii(self, rad, rad_target, local_max_depth, n, alpha, max_step_pct, r_min, r_max,
                    back_global, mode):
        call("fos_nudge_radii", self.h, ptr(rad, torch.float32, "rad"),
             ptr(rad_target, torch.float32, "rad_target"),
             ptr(local_max_depth, torch.float32, "local_max_depth"), int(n), float(alpha),
             float(max_step_pct), float(r_min), float(r_max), float(back_global), int(mode),
             stream())

    def controller_stats(self, rad, rad_target, fsc_ema, n, f_low, f_high):
        g, s_, i = C.c_int(), C.c_int(), C.c_int()
        md, mx = C.c_float(), C.c_float()
        call("fos_controller_stats", self.h, ptr(rad, torch.float32, "rad"),
             ptr(rad_target, torch.float32, "rad_target"), ptr(fsc_ema, torch.float32, "fsc_ema"),
             int(n), int(f_low), int(f_high), C.byref(g), C.byref(s_), C.byref(i), C.byref(md),
             C.byref(mx), stream())
        return g.value, s_.value, i.value, md.value, mx.value

    def pressure_stats(self, n, rad):
        a, b = C.c_float(), C.c_float()
        call("fos_pressure_stats", self.h, int(n), ptr(rad, torch.float32, "rad"), C.byref(a),
             C.byref(b), stream())
        return a.value, b.value


def to_numpy(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().numpy()
