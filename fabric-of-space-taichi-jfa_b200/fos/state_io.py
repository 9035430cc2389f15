"""State I/O: run.py's CSV export and a checkpoint that resumes bit for bit.

``export_csv`` writes the file run.py's 'S' key writes (run.py:608-629):
``particle_data_frame_{frame}.csv`` with header ``ID,X,Y,Z,Radius,FSC`` and
one row per particle, the values formatted as Python's csv module formats
numpy float32 / int32 scalars.

``save_checkpoint`` / ``load_checkpoint`` have no reference counterpart.  They
write one ``.npz`` holding every field a later frame reads, the device frame
and settle counters, the configuration, and for a ``HeadlessRun`` the
temporal-skip state and previous-frame copies.  A run resumed from it
continues exactly as the uninterrupted run would.  A surrogate model is not
part of a checkpoint: its weights have their own get/set calls.
"""
from __future__ import annotations

import csv
import dataclasses
import json
import os

import numpy as np
import torch

from ._lib import call
from .config import FosConfig
from .context import stream

CSV_HEADER = ["ID", "X", "Y", "Z", "Radius", "FSC"]
_STATE = ("pos", "rad", "rad_target", "local_max_depth", "v_jit", "cell_count", "cell_start",
          "cell_indices")
_JFA = ("fsc", "fsc_ema", "face_ids", "face_counts", "neighbor_list", "neighbor_used_count",
        "neighbor_prev_scores")
FORMAT = "fos-checkpoint"
VERSION = 1


def _host(x, n=None):
    a = x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)
    return a[:n] if n is not None else a


def export_csv(path: str, pos, rad, fsc, n: int | None = None) -> str:
    """Write run.py's particle CSV.  pos [n,3] float32, rad [n] float32, fsc
    [n] int32 (tensors or arrays); n = active particle count."""
    n = int(rad.shape[0]) if n is None else int(n)
    p = np.ascontiguousarray(_host(pos, n), np.float32)
    r = np.ascontiguousarray(_host(rad, n), np.float32)
    f = np.ascontiguousarray(_host(fsc, n), np.int32)
    with open(path, "w", newline="") as fh:
        w = csv.writer(fh)
        w.writerow(CSV_HEADER)
        for i in range(n):
            w.writerow([i, p[i][0], p[i][1], p[i][2], r[i], f[i]])
    return path


def export_frame_csv(sim, directory: str = ".") -> str:
    """export_csv of a FoamSim / HeadlessRun under run.py's file name."""
    s = getattr(sim, "sim", sim)
    name = os.path.join(directory, f"particle_data_frame_{sim.frame}.csv")
    return export_csv(name, s.pos, s.rad, s.fsc, s.n)


def read_csv(path: str) -> dict:
    """Parse a particle CSV back into arrays (float32 values round-trip)."""
    with open(path, newline="") as fh:
        rows = list(csv.reader(fh))
    if rows[0] != CSV_HEADER:
        raise ValueError(f"{path}: header {rows[0]} is not {CSV_HEADER}")
    body = rows[1:]
    return {"id": np.array([int(r[0]) for r in body], np.int64),
            "pos": np.array([[np.float32(v) for v in r[1:4]] for r in body],
                            np.float32).reshape(-1, 3),
            "rad": np.array([np.float32(r[4]) for r in body], np.float32),
            "fsc": np.array([int(r[5]) for r in body], np.int32)}


# ---------------------------------------------------------------- checkpoint
def save_checkpoint(path: str, sim) -> str:
    """Write sim (FoamSim or fos.headless.HeadlessRun) to an .npz file."""
    from .headless import HeadlessRun
    head = sim if isinstance(sim, HeadlessRun) else None
    fs = head.sim if head else sim
    if getattr(fs, "surrogate", None) is not None:
        raise ValueError("checkpoints cover the exact path; save the surrogate's weights apart")
    n = fs.n
    dev_frame, settle = fs.counters()
    arrays = {k: _host(getattr(fs, k)) for k in _STATE}
    for k in _JFA:
        arrays[k] = _host(getattr(fs.ctx, k), n)
    meta = {"format": FORMAT, "version": VERSION, "kind": "HeadlessRun" if head else "FoamSim",
            "n": n, "frame": int(sim.frame), "device_frame": dev_frame, "settle": settle,
            "res": int(fs.ctx.res), "config": dataclasses.asdict(fs.cfg)}
    if head:
        arrays["pos_prev"] = _host(head.pos_prev)
        arrays["rad_prev"] = _host(head.rad_prev)
        sk = head.skip
        meta["headless"] = {"have_prev": head.have_prev, "res": head.res,
                            "counter": sk.counter, "since": sk.since, "lockout": sk.lockout,
                            "last_fsc_mu": sk.last_fsc_mu,
                            "baseline_pending": sk._baseline_pending}
    blob = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    with open(path, "wb") as fh:
        np.savez(fh, meta=blob, **arrays)
    return path


def load_checkpoint(path: str, device: int | None = None, use_graph: bool = True):
    """Rebuild the FoamSim / HeadlessRun a checkpoint was written from."""
    from .driver import FoamSim
    from .headless import HeadlessRun
    with np.load(path) as z:
        meta = json.loads(bytes(z["meta"]).decode())
        if meta.get("format") != FORMAT or meta.get("version") != VERSION:
            raise ValueError(f"{path}: not a {FORMAT} v{VERSION} file")
        arrays = {k: z[k] for k in z.files if k != "meta"}
    cfg = FosConfig(**meta["config"])
    if meta["kind"] == "HeadlessRun":
        out = HeadlessRun(cfg, arrays["pos"], arrays["rad"], device=device)
        fs = out.sim
    else:
        out = fs = FoamSim(cfg, arrays["pos"], arrays["rad"], use_graph=use_graph, device=device)
    n = fs.n
    if n != meta["n"]:
        raise ValueError(f"{path}: {meta['n']} particles, arrays hold {n}")
    for k in _STATE:
        getattr(fs, k).copy_(torch.as_tensor(arrays[k]))
    for k in _JFA:
        getattr(fs.ctx, k)[:n].copy_(torch.as_tensor(arrays[k]))
    fs.ctx.set_resolution(meta["res"])
    call("fos_sim_set_counters", fs.ctx.h, int(meta["device_frame"]), int(meta["settle"]),
         stream())
    fs.frame = int(meta["frame"])
    if meta["kind"] == "HeadlessRun":
        h = meta["headless"]
        out.pos_prev.copy_(torch.as_tensor(arrays["pos_prev"]))
        out.rad_prev.copy_(torch.as_tensor(arrays["rad_prev"]))
        out.have_prev = bool(h["have_prev"])
        out.res = int(h["res"])
        out.frame = int(meta["frame"])
        sk = out.skip
        sk.counter, sk.since, sk.lockout = int(h["counter"]), int(h["since"]), int(h["lockout"])
        sk.last_fsc_mu = h["last_fsc_mu"]
        sk._baseline_pending = bool(h["baseline_pending"])
    torch.cuda.synchronize(fs.ctx.device)
    return out
