"""Headless frame driver: run.py's per-frame order (run.py:699-1261) on one GPU.

``FoamSim`` owns the particle state (pos, rad, rad_target, local_max_depth,
delta_r, hash-grid arrays) as torch CUDA tensors and a libfos ``Context``
holding the JFA/FSC fields.  ``step()`` issues one frame through
``fos_frame_graph``: the frame is captured once per kind (JFA frame /
non-JFA frame) and replayed as a CUDA graph; the frame index, settle counter
and warm-start gate live on the device, so no frame synchronises the host.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._lib import FosState, call
from .config import FosConfig
from .context import Context, stream


class FoamSim:
    def __init__(self, cfg: FosConfig, pos: np.ndarray, rad: np.ndarray, use_graph: bool = True,
                 ctx: Context | None = None, device: int | None = None, surrogate=None,
                 policy=None, surrogate_mode: str = "anchored", jfa_warm: bool = False,
                 warm_refresh: int = 0):
        n = int(rad.shape[0])
        self.cfg = cfg
        # learned FSC between JFA runs (fos.surrogate); None = the reference's stale reuse
        self.surrogate = surrogate
        if surrogate is not None and policy is None:
            from .surrogate import RefreshPolicy
            policy = RefreshPolicy(every=2 * cfg.JFA_CADENCE, warm_frames=cfg.JFA_WARM_FRAMES)
        self.policy = policy
        self.surrogate_mode = surrogate_mode
        # warm-started JFA (fos_jfa_warm) on JFA frames after the first; with
        # warm_refresh = k > 0 every k-th JFA frame is exact again
        self.jfa_warm = bool(jfa_warm)
        self.warm_refresh = int(warm_refresh)
        self._jfa_runs = 0
        self.n = n
        self.use_graph = use_graph
        self.ctx = ctx or Context(cfg, max_n=n, max_res=cfg.JFA_RES, device=device)
        self.ctx.set_resolution(cfg.JFA_RES)
        dev = torch.device("cuda", self.ctx.device)
        G3 = cfg.grid_res() ** 3
        self.pos = torch.as_tensor(np.ascontiguousarray(pos, np.float32).reshape(n, 3)).to(dev)
        self.rad = torch.as_tensor(np.ascontiguousarray(rad, np.float32)).to(dev)
        self.rad_target = self.rad.clone()
        self.local_max_depth = torch.zeros(n, dtype=torch.float32, device=dev)
        self.delta_r = torch.zeros(n, dtype=torch.float32, device=dev)
        self.cell_count = torch.zeros(G3, dtype=torch.int32, device=dev)
        self.cell_start = torch.zeros(G3, dtype=torch.int32, device=dev)
        self.cell_indices = torch.zeros(n, dtype=torch.int32, device=dev)
        self.v_jit = torch.zeros(n, 3, dtype=torch.float32, device=dev)  # run.py:151
        self.state = FosState(n, self.pos.data_ptr(), self.rad.data_ptr(),
                              self.rad_target.data_ptr(), self.local_max_depth.data_ptr(),
                              self.delta_r.data_ptr(), self.cell_count.data_ptr(),
                              self.cell_start.data_ptr(), self.cell_indices.data_ptr(),
                              self.v_jit.data_ptr())
        self.fp = cfg.frame_params()
        self.frame = 0
        if surrogate is not None:
            from .surrogate import set_mode
            set_mode(self.ctx, surrogate_mode)

    @classmethod
    def from_foam(cls, foam, use_graph: bool = True, surrogate=None, policy=None,
                  surrogate_mode: str = "anchored", jfa_warm: bool = False, warm_refresh: int = 0,
                  **over) -> "FoamSim":
        return cls(FosConfig.for_foam(foam, **over), foam.pos, foam.rad, use_graph=use_graph,
                   surrogate=surrogate, policy=policy, surrogate_mode=surrogate_mode,
                   jfa_warm=jfa_warm, warm_refresh=warm_refresh)

    def _jfa_kind(self, jfa: bool) -> int:
        """0 no JFA, 1 the exact JFA, 2 the warm-started one."""
        if not jfa:
            return 0
        k = self._jfa_runs
        self._jfa_runs += 1
        if not self.jfa_warm or k == 0 or (self.warm_refresh and k % self.warm_refresh == 0):
            return 1
        return 2

    def initialize(self, frame0: int = 0):
        """initialize_simulation's device part (run.py:320-382)."""
        call("fos_sim_init", self.ctx.h, C.byref(self.state), C.byref(self.fp), int(frame0),
             stream())
        self.frame = int(frame0)
        self._jfa_runs = 0

    def step(self):
        if self.surrogate is not None:
            return self._step_surrogate()
        jfa = self._jfa_kind(self.cfg.is_jfa_frame(self.frame))
        fn = "fos_frame_graph" if self.use_graph else "fos_frame"
        call(fn, self.ctx.h, C.byref(self.state), C.byref(self.fp), jfa, stream())
        self.frame += 1
        return bool(jfa)

    def _step_surrogate(self):
        """A frame with the surrogate's FSC between JFA runs.  Every JFA frame
        (warm start included) also evaluates the surrogate, which sets the
        anchor of the anchored mode; after the warm start each JFA frame is
        judged (one host sync to read the counters) and drift forces
        refreshes.  Non-JFA frames that the policy gives no surrogate update
        keep the controller's last FSC."""
        f = self.frame
        pol = self.policy
        jfa = pol.is_jfa(f)
        if jfa or pol.is_surrogate(f):
            fn = "fos_frame_surrogate_graph" if self.use_graph else "fos_frame_surrogate"
            call(fn, self.ctx.h, C.byref(self.state), C.byref(self.fp), self.surrogate.h,
                 int(jfa), stream())
        else:
            fn = "fos_frame_graph" if self.use_graph else "fos_frame"
            call(fn, self.ctx.h, C.byref(self.state), C.byref(self.fp), 0, stream())
        pol.ran(f, jfa)
        if jfa and f >= pol.warm_frames:
            from .surrogate import stats
            pol.observe(stats(self.ctx) | {"frame": f})
        self.frame += 1
        return bool(jfa)

    STAGES = ("grid", "max_overlap", "nudge", "pressure", "brownian", "pbd", "jfa_passes",
              "filter_faces", "finalize_ema", "targets_end", "ou_jitter")

    def step_profiled(self) -> dict:
        """One frame (no graph) with CUDA events between stages -> ms per stage."""
        jfa = self._jfa_kind(self.cfg.is_jfa_frame(self.frame))
        ms = (C.c_float * len(self.STAGES))()
        call("fos_frame_profile", self.ctx.h, C.byref(self.state), C.byref(self.fp), jfa, ms,
             stream())
        self.frame += 1
        return {k: float(v) for k, v in zip(self.STAGES, ms)} | {"jfa": bool(jfa)}

    def trace_dynamics(self, cap: int = 256) -> list:
        """ns between the phases of one cooperative plain-frame kernel (block 0's
        view; the frame counter is not advanced, positions and radii are)."""
        buf = (C.c_longlong * cap)()
        cnt = C.c_int()
        call("fos_frame_trace", self.ctx.h, C.byref(self.state), C.byref(self.fp), buf, cap,
             C.byref(cnt), stream())
        t = [buf[i] for i in range(cnt.value)]
        return [t[i + 1] - t[i] for i in range(len(t) - 1)]

    def run(self, frames: int):
        for _ in range(frames):
            self.step()

    def counters(self):
        f, s = C.c_int(), C.c_int()
        call("fos_sim_counters", self.ctx.h, C.byref(f), C.byref(s), stream())
        return f.value, s.value

    # convenience views
    @property
    def fsc(self) -> torch.Tensor:
        return self.ctx.fsc[: self.n]

    @property
    def fsc_ema(self) -> torch.Tensor:
        return self.ctx.fsc_ema[: self.n]

    @property
    def face_ids(self) -> torch.Tensor:
        return self.ctx.face_ids[: self.n]

    @property
    def neighbor_list(self) -> torch.Tensor:
        return self.ctx.neighbor_list[: self.n]
