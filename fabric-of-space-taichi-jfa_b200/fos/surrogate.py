"""Learned face-sharing-count (FSC) surrogate.

There is no counterpart in the reference. Its run.py measures FSC with the JFA
only on measurement frames (run.py:1230-1261) and keeps using that stale
``fsc`` / ``fsc_ema`` on the frames between.  The surrogate estimates FSC on
those frames from the particle geometry alone:

* candidate pairs with ``|d| < cutoff * (r_i + r_j)``, found on the hash grid,
  each kept once by its owner (balanced ownership, ``include/fos.h``);
* a 16-feature vector per pair, defined in ``include/fos.h``;
* a 16 -> 64 -> 64 -> 1 MLP (ReLU, sigmoid) giving P(pair shares a face).
  Inference uses BF16 weights on the tensor cores with FP32 accumulation;
  training uses FP32 master weights and Adam;
* per-particle FSC = the sum of the pair probabilities at both ends.

Two modes turn the estimate into the FSC the controller sees.  In
``absolute`` mode it is the estimate itself.  In ``anchored`` mode it is the
last JFA's exact fsc plus the change in the estimate since that JFA, which
cancels the estimate's per-cell bias.

The exact JFA still runs every ``RefreshPolicy.every`` frames.  On those
frames it judges the surrogate per cell.  If the surrogate's error exceeds
the policy's thresholds, the next frames run the JFA instead: a drift-forced
refresh.

All arithmetic runs in libfos (CUDA, sm_100a).  This module only owns buffers
and drives the calls.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import FosSurrogateStats, call
from .context import Context, ptr, stream

NF = _lib.SUR_FEATURES
NH = _lib.SUR_HIDDEN
NPARAM = _lib.SUR_NPARAM
OFF_W1, OFF_B1 = 0, NH * NF
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH


def init_params(seed: int = 0) -> np.ndarray:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases (the
    default initialisation of a dense layer), FP32, in the ABI layout."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)

    def u(n, fan_in):
        b = 1.0 / math.sqrt(fan_in)
        return rng.uniform(-b, b, n).astype(np.float32)

    p[OFF_W1:OFF_B1] = u(NH * NF, NF)
    p[OFF_B1:OFF_W2] = u(NH, NF)
    p[OFF_W2:OFF_B2] = u(NH * NH, NH)
    p[OFF_B2:OFF_W3] = u(NH, NH)
    p[OFF_W3:OFF_B3] = u(NH, NH)
    p[OFF_B3] = u(1, NH)[0]
    return p


def unpack(params: np.ndarray) -> dict:
    """ABI parameter vector -> named arrays (W[out][in])."""
    p = np.asarray(params, np.float32)
    return {"W1": p[OFF_W1:OFF_B1].reshape(NH, NF), "b1": p[OFF_B1:OFF_W2],
            "W2": p[OFF_W2:OFF_B2].reshape(NH, NH), "b2": p[OFF_B2:OFF_W3],
            "w3": p[OFF_W3:OFF_B3], "b3": p[OFF_B3:OFF_B3 + 1]}


class Surrogate:
    """One MLP on one device (``fos_surrogate_create``)."""

    def __init__(self, cutoff: float = 2.5, device: int | None = None, seed: int = 0):
        _lib.load()
        if not torch.cuda.is_available():
            raise _lib.FosError(3, "Surrogate", "no CUDA device: libfos has no CPU path")
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.cutoff = float(cutoff)
        h = C.c_void_p()
        call("fos_surrogate_create", self.device, C.c_float(self.cutoff), C.byref(h))
        self.h = h
        self._loss = torch.zeros(1, dtype=torch.float32, device=f"cuda:{self.device}")
        self.set_weights(init_params(seed), np.zeros(NF, np.float32), np.ones(NF, np.float32))

    def close(self):
        if getattr(self, "h", None):
            _lib.load().fos_surrogate_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- weights
    def set_weights(self, params, mu, sd):
        p = np.ascontiguousarray(params, np.float32).reshape(NPARAM)
        m = np.ascontiguousarray(mu, np.float32).reshape(NF)
        s = np.ascontiguousarray(sd, np.float32).reshape(NF)
        call("fos_surrogate_set_weights", self.h, p.ctypes.data, m.ctypes.data, s.ctypes.data)

    def get_weights(self):
        p = np.zeros(NPARAM, np.float32)
        m = np.zeros(NF, np.float32)
        s = np.zeros(NF, np.float32)
        call("fos_surrogate_get_weights", self.h, p.ctypes.data, m.ctypes.data, s.ctypes.data)
        return p, m, s

    def standardize_from(self, X: torch.Tensor):
        """Feature mean / std of X (FP32, on the device) as the model's input
        standardisation; resets Adam."""
        p, _, _ = self.get_weights()
        mu = X.double().mean(0)
        sd = X.double().std(0).clamp_min(1e-3)
        self.set_weights(p, mu.float().cpu().numpy(), sd.float().cpu().numpy())

    def save(self, path: str):
        p, m, s = self.get_weights()
        np.savez(path, params=p, mu=m, sd=s, cutoff=np.float32(self.cutoff))

    @classmethod
    def load(cls, path: str, device: int | None = None) -> "Surrogate":
        z = np.load(path)
        sur = cls(cutoff=float(z["cutoff"]), device=device)
        sur.set_weights(z["params"], z["mu"], z["sd"])
        return sur

    # ---------------------------------------------------------------- training
    def train_step(self, X, y, rows, lr: float = 1e-3) -> torch.Tensor:
        """One Adam step on the rows ``rows`` of (X, y); returns the batch loss
        as a device tensor (no host sync)."""
        call("fos_surrogate_train_step", self.h, ptr(X, torch.float32, "X"),
             ptr(y, torch.float32, "y"), ptr(rows, torch.int32, "rows"), int(rows.numel()),
             C.c_float(lr), ptr(self._loss), stream())
        return self._loss

    def gradient(self, X, y, rows):
        grad = torch.zeros(NPARAM, dtype=torch.float32, device=X.device)
        loss = torch.zeros(1, dtype=torch.float32, device=X.device)
        call("fos_surrogate_gradient", self.h, ptr(X, torch.float32, "X"),
             ptr(y, torch.float32, "y"), ptr(rows, torch.int32, "rows"), int(rows.numel()),
             ptr(grad), ptr(loss), stream())
        return grad, loss

    def fit(self, X, y, epochs: int = 20, batch: int = 65536, lr: float = 1e-3,
            seed: int = 0) -> list:
        """Adam over shuffled batches; returns the mean loss of each epoch."""
        P = int(X.shape[0])
        g = torch.Generator(device=X.device)
        g.manual_seed(seed)
        out = []
        for _ in range(epochs):
            perm = torch.randperm(P, generator=g, device=X.device).to(torch.int32)
            tot = torch.zeros(1, dtype=torch.float32, device=X.device)
            nb = 0
            for k in range(0, P, batch):
                tot += self.train_step(X, y, perm[k:k + batch], lr)
                nb += 1
            out.append(float(tot.item()) / max(nb, 1))
        return out

    # ---------------------------------------------------------------- inference
    def forward(self, X: torch.Tensor) -> torch.Tensor:
        """Pair probabilities for raw features X [P, 16] (tensor cores)."""
        P = int(X.shape[0])
        prob = torch.empty(P, dtype=torch.float32, device=X.device)
        call("fos_surrogate_forward", self.h, ptr(X, torch.float32, "X"), P, ptr(prob),
             stream())
        return prob


# -------------------------------------------------------------------- pairs
def build_pairs(ctx: Context, sur: Surrogate, pos, rad, n: int, r_max: float, cell_start,
                cell_count, cell_indices):
    call("fos_surrogate_pairs", ctx.h, sur.h, ptr(pos, torch.float32, "pos"),
         ptr(rad, torch.float32, "rad"), int(n), C.c_float(r_max),
         ptr(cell_start, torch.int32, "cell_start"), ptr(cell_count, torch.int32, "cell_count"),
         ptr(cell_indices, torch.int32, "cell_indices"), stream())


def pair_count(ctx: Context):
    p, o = C.c_int(), C.c_int()
    call("fos_surrogate_pair_count", ctx.h, C.byref(p), C.byref(o), stream())
    return p.value, o.value


def export(ctx: Context, rad, labels: bool = True, memory=None) -> dict:
    """Features, labels (pair in the last JFA neighbour list) and pair indices
    of the last pair build.  memory = (neighbor_list, neighbor_used_count,
    fsc) of an earlier JFA frame for the memory features 14-15 (None: the
    context's current ones, as inference sees them)."""
    P, overflow = pair_count(ctx)
    dev = rad.device
    X = torch.empty((P, NF), dtype=torch.float32, device=dev)
    y = torch.empty(P, dtype=torch.float32, device=dev) if labels else None
    pi = torch.empty(P, dtype=torch.int32, device=dev)
    pj = torch.empty(P, dtype=torch.int32, device=dev)
    if P > 0:
        mem = [None, None, None] if memory is None else list(memory)
        call("fos_surrogate_export", ctx.h, ptr(rad, torch.float32, "rad"), ptr(X), ptr(y),
             ptr(pi), ptr(pj), ptr(mem[0]), ptr(mem[1]), ptr(mem[2]), stream())
    return {"X": X, "y": y, "i": pi, "j": pj, "overflow": overflow}


def predict(ctx: Context, sur: Surrogate, rad, n: int, with_pairs: bool = False) -> dict:
    dev = rad.device
    fs = torch.empty(n, dtype=torch.float32, device=dev)
    fi = torch.empty(n, dtype=torch.int32, device=dev)
    prob = None
    if with_pairs:
        P, _ = pair_count(ctx)
        prob = torch.empty(max(P, 1), dtype=torch.float32, device=dev)
    call("fos_surrogate_predict", ctx.h, sur.h, ptr(rad, torch.float32, "rad"), ptr(fs),
         ptr(fi), ptr(prob), stream())
    return {"fsc_float": fs, "fsc": fi, "prob": prob}


MODES = {"absolute": _lib.SUR_ABSOLUTE, "anchored": _lib.SUR_ANCHORED}


def set_mode(ctx: Context, mode: str):
    """absolute: the controller sees the model's estimate s; anchored: the last
    JFA fsc moved by the change of s since that JFA (include/fos.h)."""
    if mode not in MODES:
        raise ValueError(f"mode must be one of {sorted(MODES)}")
    call("fos_surrogate_set_mode", ctx.h, MODES[mode])


def stats(ctx: Context) -> dict:
    st = FosSurrogateStats()
    call("fos_surrogate_stats", ctx.h, C.byref(st), stream())
    d = {k: getattr(st, k) for k, _ in FosSurrogateStats._fields_}
    j = max(d["judged"], 1)
    d.update(exact_frac=d["exact"] / j, within1_frac=d["within1"] / j,
             stale_exact_frac=d["stale_exact"] / j, stale_within1_frac=d["stale_within1"] / j,
             mean_abs_err=d["abs_err"] / j, stale_mean_abs_err=d["stale_abs_err"] / j)
    return d


# -------------------------------------------------------------------- policy
@dataclass
class RefreshPolicy:
    """When the exact JFA runs while the surrogate supplies FSC.

    * Frames below ``warm_frames`` always run the JFA (the reference's warm
      start).
    * After that, the JFA runs when ``every`` frames have passed since the
      last JFA frame.
    * After a judged JFA frame, drift is ``exact_frac < min_exact`` or
      ``mean_abs_err > max_mean_abs_err``.  Drift makes the next
      ``force_frames`` frames JFA frames too.  The defaults are the target's:
      at least 99 % of cells with the JFA's FSC, and a mean absolute error of
      at most 0.05 faces per cell.  ``min_exact=0.0`` with
      ``max_mean_abs_err=math.inf`` switches the guard off.
    * Between JFA frames the surrogate runs on every ``surrogate_every``-th
      frame; on the others the controller keeps its last FSC, as the
      reference does on every non-JFA frame.
    """
    every: int = 10
    surrogate_every: int = 1
    warm_frames: int = 20
    min_exact: float = 0.99
    max_mean_abs_err: float = 0.05
    force_frames: int = 1
    last_jfa: int = -10**9
    forced_left: int = 0
    forced_total: int = 0
    judged: list = field(default_factory=list)

    def is_jfa(self, frame: int) -> bool:
        if frame < self.warm_frames or self.forced_left > 0:
            return True
        return frame - self.last_jfa >= self.every

    def is_surrogate(self, frame: int) -> bool:
        """On a non-JFA frame: whether the surrogate updates the FSC."""
        return (frame - self.last_jfa) % max(1, self.surrogate_every) == 0

    def ran(self, frame: int, jfa: bool):
        if jfa:
            self.last_jfa = frame
            if self.forced_left > 0 and frame >= self.warm_frames:
                self.forced_left -= 1

    def observe(self, s: dict) -> bool:
        """Record a judged frame's stats; returns True when drift forces a refresh."""
        self.judged.append(s)
        drift = s["exact_frac"] < self.min_exact or s["mean_abs_err"] > self.max_mean_abs_err
        if drift:
            self.forced_left = self.force_frames
            self.forced_total += 1
        return drift


# -------------------------------------------------------------------- data
def collect(foams, sur: Surrogate, export_frames=(15, 25), max_rows: int | None = None,
            seed: int = 0) -> dict:
    """Labelled pairs from JFA frames of plain simulations.  For each foam,
    the plain frame loop runs up to the last export frame; at every export
    frame (which must be a JFA frame) the pairs of the post-frame positions
    are built and labelled by that frame's JFA neighbour lists, and their
    memory features come from the JFA frame before it (the lists a surrogate
    frame would see).  With max_rows, a seeded uniform subset of that many
    rows is kept."""
    from .driver import FoamSim
    Xs, ys = [], []
    for foam in foams:
        sim = FoamSim.from_foam(foam)
        sim.initialize()
        last = max(export_frames)
        mem = None
        for f in range(last + 1):
            if f in export_frames:
                n = sim.n
                mem = (sim.neighbor_list[:n].clone(), sim.ctx.neighbor_used_count[:n].clone(),
                       sim.fsc[:n].clone())
            jfa = sim.step()
            if f in export_frames:
                if not jfa:
                    raise ValueError(f"export frame {f} is not a JFA frame")
                build_pairs(sim.ctx, sur, sim.pos, sim.rad, sim.n, float(sim.cfg.R_MAX),
                            sim.cell_start, sim.cell_count, sim.cell_indices)
                d = export(sim.ctx, sim.rad, memory=mem)
                Xs.append(d["X"])
                ys.append(d["y"])
        sim.ctx.close()
    X, y = torch.cat(Xs), torch.cat(ys)
    if max_rows is not None and X.shape[0] > max_rows:
        g = torch.Generator(device=X.device)
        g.manual_seed(seed)
        keep = torch.randperm(X.shape[0], generator=g, device=X.device)[:max_rows]
        X, y = X[keep].contiguous(), y[keep].contiguous()
    return {"X": X, "y": y}


def train_default(foams=None, cutoff: float = 2.5, frames=(20, 40, 60, 80, 100, 140, 200),
                  max_rows: int = 3_000_000, epochs: int = 30, lr: float = 1e-3) -> Surrogate:
    """The model the benchmarks use: labelled pairs from JFA frames 20-200 of
    the headline law with seeds 10-19 (about 2-3 M pairs kept), standardised,
    30 epochs of Adam at lr 1e-3 with 65,536-pair batches."""
    from . import inputs
    foams = foams if foams is not None else [inputs.surrogate_variant(s) for s in range(10, 20)]
    sur = Surrogate(cutoff=cutoff)
    data = collect(foams, sur, export_frames=frames, max_rows=max_rows)
    sur.standardize_from(data["X"])
    sur.fit(data["X"], data["y"], epochs=epochs, batch=65536, lr=lr)
    return sur
