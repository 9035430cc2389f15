"""Batched ensembles: many independent periodic foams advanced together.

There is no counterpart in the reference, which runs one foam per process.
``Ensemble`` packs the foams into one libfos ensemble (``fos_ensemble_*``).
Every stage of a frame is one launch over all foams: the dynamics are one
persistent cooperative kernel, and the JFA and FSC stages are one launch each.
The frame is replayed from a CUDA graph, and each foam's result is
bit-identical to the same foam run alone in ``FoamSim``.

Launch shapes (JFA pass block, voxel-stage block, dynamics kernel shape) are
picked by ``Ensemble.autotune``, which times the candidates on the ensemble's
own state and caches the choice in a JSON file keyed by device and ensemble
shape.

``partition`` splits foams over ranks for multi-GPU runs, with no exchange
during a frame.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os

import numpy as np
import torch

from . import _lib
from ._lib import FosEnsembleFoam, FosEnsembleTuning, FosEnsembleView, call
from .config import FosConfig
from .context import _view, stream

S = _lib.MAX_NEIGHBORS
FIXED = {"pass_block": 256, "voxel_block": 256, "coop_threads": 1024, "coop_blocks_per_sm": 1}
REPORT_KEYS = ["pass_block=128", "pass_block=256", "pass_block=512", "voxel_block=128",
               "voxel_block=256", "voxel_block=512", "coop=512x1", "coop=512x2", "coop=1024x1",
               "coop=1024x2"]
_SHARED_FRAME_FIELDS = ("pbd_iters", "pressure_iters", "growth_pct", "max_step_pct",
                        "adjustment_frames", "bp_mode", "warmstart_frames", "zero_rate_thresh",
                        "pressure_k", "pressure_exp", "pressure_pair_cap", "max_eq_nei",
                        "brownian_strength", "warmup_pbd")


def frame_cost(foam) -> float:
    """Relative per-frame cost of a foam for load balancing.

    Measured on one B200 for the headline foam: the dynamics cost about 40 ns
    per particle per frame; the JFA and FSC stages cost about 0.45 ns per voxel
    per JFA frame, run every 5th frame.  So the cost is N + R^3 / 450, in
    units of one particle's dynamics."""
    return float(foam.n) + float(foam.res) ** 3 / 450.0


def partition(foams, world: int) -> list[list[int]]:
    """Foam indices per rank: longest-processing-time greedy on frame_cost, so
    the most loaded rank carries at most 4/3 of the optimum.  Ties go to the
    lowest rank; each rank's indices come back ascending."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(foams)), key=lambda k: (-frame_cost(foams[k]), k))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += frame_cost(foams[k])
    return [sorted(v) for v in out]


class Ensemble:
    """fos_ensemble_* over a list of ``inputs.Foam`` (one shared configuration,
    per-foam band, radius bounds, resolutions and seed)."""

    def __init__(self, foams, device: int | None = None, **cfg_over):
        lib = _lib.load()
        if not torch.cuda.is_available():
            raise _lib.FosError(3, "Ensemble", "no CUDA device: libfos has no CPU path")
        if not foams:
            raise ValueError("an ensemble needs at least one foam")
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.foams = list(foams)
        self.cfgs = [FosConfig.for_foam(f, **cfg_over) for f in self.foams]
        self.cfg = self.cfgs[0]
        fp0 = self.cfg.frame_params()
        for cfg in self.cfgs[1:]:
            fp = cfg.frame_params()
            for k in _SHARED_FRAME_FIELDS:
                if getattr(fp, k) != getattr(fp0, k):
                    raise ValueError(f"foams disagree on shared frame parameter {k}")
            if (cfg.JFA_WARM_FRAMES, cfg.JFA_CADENCE) != (self.cfg.JFA_WARM_FRAMES,
                                                          self.cfg.JFA_CADENCE):
                raise ValueError("foams disagree on the JFA cadence")
        arr = (FosEnsembleFoam * len(self.foams))()
        for k, (foam, cfg) in enumerate(zip(self.foams, self.cfgs)):
            fp = cfg.frame_params()
            arr[k] = FosEnsembleFoam(foam.n, int(cfg.JFA_RES), int(cfg.grid_res()), fp.f_low,
                                     fp.f_high, fp.r_min, fp.r_max, fp.seed)
        self._lib = lib
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            call("fos_ensemble_create", C.byref(self.cfg.params()), C.byref(fp0), arr,
                 len(self.foams), self.device, C.byref(h))
        self.h = h
        v = FosEnsembleView()
        call("fos_ensemble_view", h, C.byref(v))
        self.n_total = v.n_total
        nf = len(self.foams)
        po = (C.c_int * (nf + 1))()
        vo = (C.c_longlong * (nf + 1))()
        co = (C.c_int * (nf + 1))()
        call("fos_ensemble_offsets", h, po, vo, co)
        self.part_off = list(po)
        self.vox_off = list(vo)
        self.cell_off = list(co)
        n = self.n_total
        self.pos = _view(v.pos, (n, 3), torch.float32)
        self.rad = _view(v.rad, (n,), torch.float32)
        self.rad_target = _view(v.rad_target, (n,), torch.float32)
        self.local_max_depth = _view(v.local_max_depth, (n,), torch.float32)
        self.fsc = _view(v.fsc, (n,), torch.int32)
        self.fsc_ema = _view(v.fsc_ema, (n,), torch.float32)
        self.face_ids = _view(v.face_ids, (n, S), torch.int32)
        self.face_counts = _view(v.face_counts, (n, S), torch.int32)
        self.neighbor_list = _view(v.neighbor_list, (n, S), torch.int32)
        self.foam_of = _view(v.foam_of, (n,), torch.int32)
        pos = np.concatenate([np.ascontiguousarray(f.pos, np.float32) for f in self.foams])
        rad = np.concatenate([np.ascontiguousarray(f.rad, np.float32) for f in self.foams])
        self.pos.copy_(torch.as_tensor(pos.reshape(n, 3)))
        self.rad.copy_(torch.as_tensor(rad))
        torch.cuda.synchronize(self.device)
        self.frame = 0
        self.use_graph = True
        self.surrogate = None
        self.policy = None

    def close(self):
        if getattr(self, "h", None):
            self._lib.fos_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- frames
    def initialize(self, frame0: int = 0):
        call("fos_ensemble_init", self.h, int(frame0), stream())
        self.frame = int(frame0)

    def is_jfa_frame(self, frame: int) -> bool:
        return self.cfg.is_jfa_frame(frame)

    def attach_surrogate(self, surrogate, policy=None, mode: str = "anchored"):
        """Run the learned FSC surrogate between JFA frames, as FoamSim does for
        one foam: the policy (fos.surrogate.RefreshPolicy; default a refresh
        every 2 cadences after the warm start) picks the JFA frames, every JFA
        frame after the warm start is judged over all foams, and drift forces
        refreshes.  Each foam's pairs come from its own grid, so every foam
        gets the FSC it gets alone."""
        from .surrogate import MODES, RefreshPolicy
        if policy is None:
            c = self.cfg
            policy = RefreshPolicy(every=2 * c.JFA_CADENCE, warm_frames=c.JFA_WARM_FRAMES)
        self.surrogate, self.policy = surrogate, policy
        call("fos_ensemble_surrogate_mode", self.h, MODES[mode])

    def surrogate_stats(self) -> dict:
        """Counters of the last pair build and judged JFA frame, all foams."""
        from ._lib import FosSurrogateStats
        st = FosSurrogateStats()
        call("fos_ensemble_surrogate_stats", self.h, C.byref(st), stream())
        d = {k: getattr(st, k) for k, _ in FosSurrogateStats._fields_}
        j = max(d["judged"], 1)
        d.update(exact_frac=d["exact"] / j, within1_frac=d["within1"] / j,
                 stale_exact_frac=d["stale_exact"] / j, stale_within1_frac=d["stale_within1"] / j,
                 mean_abs_err=d["abs_err"] / j, stale_mean_abs_err=d["stale_abs_err"] / j)
        return d

    def step(self) -> bool:
        if self.surrogate is not None:
            return self._step_surrogate()
        jfa = 1 if self.is_jfa_frame(self.frame) else 0
        fn = "fos_ensemble_frame_graph" if self.use_graph else "fos_ensemble_frame"
        call(fn, self.h, jfa, stream())
        self.frame += 1
        return bool(jfa)

    def _step_surrogate(self) -> bool:
        f, pol = self.frame, self.policy
        jfa = pol.is_jfa(f)
        if jfa or pol.is_surrogate(f):
            call("fos_ensemble_frame_surrogate", self.h, self.surrogate.h, int(jfa), stream())
        else:
            fn = "fos_ensemble_frame_graph" if self.use_graph else "fos_ensemble_frame"
            call(fn, self.h, 0, stream())
        pol.ran(f, jfa)
        if jfa and f >= pol.warm_frames:
            pol.observe(self.surrogate_stats() | {"frame": f})
        self.frame += 1
        return bool(jfa)

    def run(self, frames: int):
        for _ in range(frames):
            self.step()

    def launch_count(self) -> int:
        return int(self._lib.fos_ensemble_launch_count(self.h))

    # ---------------------------------------------------------------- views
    def foam(self, k: int) -> dict:
        """Foam k's slices; face_ids / neighbor_list renumbered to the foam's
        own indices (-1 and unused slots kept)."""
        a, b = self.part_off[k], self.part_off[k + 1]

        def local(t):
            t = t[a:b]
            return torch.where(t >= 0, t - a, t)

        return {"pos": self.pos[a:b], "rad": self.rad[a:b], "rad_target": self.rad_target[a:b],
                "fsc": self.fsc[a:b], "fsc_ema": self.fsc_ema[a:b],
                "face_ids": local(self.face_ids), "face_counts": self.face_counts[a:b],
                "neighbor_list": local(self.neighbor_list)}

    # ---------------------------------------------------------------- tuning
    @property
    def tuning(self) -> dict:
        t = FosEnsembleTuning()
        call("fos_ensemble_get_tuning", self.h, C.byref(t))
        return {k: getattr(t, k) for k, _ in FosEnsembleTuning._fields_}

    @tuning.setter
    def tuning(self, d: dict):
        t = FosEnsembleTuning(**{k: int(d[k]) for k, _ in FosEnsembleTuning._fields_})
        call("fos_ensemble_set_tuning", self.h, C.byref(t))

    def set_multi_voxel(self, on: bool):
        """Record passes with four voxels a thread (default) or one; the labels
        are the same."""
        call("fos_ensemble_set_multi_voxel", self.h, int(bool(on)))

    def trace_dynamics(self, cap: int = 512) -> list:
        """ns between the phases of one dynamics kernel over every foam (block
        0's view; positions and radii advance, the frame index does not)."""
        buf = (C.c_longlong * cap)()
        cnt = C.c_int()
        call("fos_ensemble_trace", self.h, buf, cap, C.byref(cnt), stream())
        t = [buf[i] for i in range(cnt.value)]
        return [t[i + 1] - t[i] for i in range(len(t) - 1)]

    def signature(self) -> str:
        """Device name + shape of the ensemble (counts, JFA res, hash res)."""
        shape = [(f.n, c.JFA_RES, c.grid_res()) for f, c in zip(self.foams, self.cfgs)]
        dig = hashlib.sha1(json.dumps(shape).encode()).hexdigest()[:16]
        return f"{torch.cuda.get_device_name(self.device)}|{len(shape)}|{dig}"

    def autotune(self, reps: int = 3, cache: str | None = None) -> tuple[dict, dict]:
        """Pick the launch shapes by timing (fos_ensemble_autotune); with a
        cache path, reuse a stored choice for the same device and ensemble
        shape, or store the new one.  Returns (tuning, {candidate: ms})."""
        key = self.signature()
        if cache and os.path.exists(cache):
            try:
                db = json.load(open(cache))
            except (OSError, ValueError):
                db = {}
            if key in db:
                self.tuning = db[key]["tuning"]
                return self.tuning, db[key].get("report_ms", {})
        best = FosEnsembleTuning()
        rep = (C.c_float * len(REPORT_KEYS))()
        call("fos_ensemble_autotune", self.h, int(reps), C.byref(best), rep, len(REPORT_KEYS),
             stream())
        report = {k: round(float(v), 4) for k, v in zip(REPORT_KEYS, rep)}
        tuning = self.tuning
        if cache:
            db = {}
            if os.path.exists(cache):
                try:
                    db = json.load(open(cache))
                except (OSError, ValueError):
                    db = {}
            db[key] = {"tuning": tuning, "report_ms": report}
            tmp = cache + ".tmp"
            with open(tmp, "w") as fh:
                json.dump(db, fh, indent=1, sort_keys=True)
            os.replace(tmp, cache)
        return tuning, report
