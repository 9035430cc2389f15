"""The oracle's topology.py restatement against a line-by-line Python
transcription (numpy float32 scalars, serial loops) and known answers.

The reference ships no topology tests or vectors; these pin the C restatement
on small seeded foams: candidate lists (serial scan order, 28-slot cap and
truncation flag), Gabriel degrees (with subsampling and early exit), the
batched variant, the k-NN proxy, the EMA and the radius rule.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

f32 = np.float32


def wrapP(x, L):
    return f32(x - f32(L) * np.floor(f32(x * f32(1.0 / L)) + f32(0.5)))


def pdelta(a, b, L):
    return [wrapP(f32(b[k] - a[k]), L) for k in range(3)]


def dot(d):
    return f32(f32(f32(d[0] * d[0]) + f32(d[1] * d[1])) + f32(d[2] * d[2]))


def home(p, L, G):
    out = []
    for k in range(3):
        w = wrapP(p[k], L)
        q = f32(f32(w + f32(0.5 * L)) * f32(1.0 / L))
        out.append(int(f32(q * f32(G))))
    return out


def cells27(h, G):
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                yield (((h[0] + dx) % G) * G + (h[1] + dy) % G) * G + (h[2] + dz) % G


def py_candidates(pos, rad, grid, L, G, mult, cap):
    cc, cs, ci = grid
    n = len(rad)
    pairs = [[] for _ in range(n)]
    trunc = [0] * n
    for i in range(n):
        for c in cells27(home(pos[i], L, G), G):
            for k in range(cs[c], cs[c] + cc[c]):
                j = int(ci[k])
                if j <= i:
                    continue
                th = f32(f32(mult) * f32(rad[i] + rad[j]))
                if dot(pdelta(pos[i], pos[j], L)) <= f32(th * th):
                    if len(pairs[i]) < cap:
                        pairs[i].append(j)
                    else:
                        trunc[i] = 1
                        break
    return pairs, trunc


def py_gabriel_pair(pos, grid, i, j, d2, L, G, cell, rev):
    cc, cs, ci = grid
    d = pdelta(pos[i], pos[j], L)
    m = [wrapP(f32(pos[i][k] + f32(f32(0.5) * d[k])), L) for k in range(3)]
    r_sq = f32(f32(0.25) * d2)
    mc = [int(f32(f32(f32(m[k] + f32(0.5 * L)) * f32(1.0 / L)) * f32(G))) % G for k in range(3)]
    s = int(math.ceil(f32(f32(f32(np.sqrt(d2)) * f32(0.5)) / f32(cell))))
    s = min(max(1, min(s, 3)), G // 2)
    eps = max(f32(1e-12), f32(f32(1e-6) * r_sq))
    for dx in range(-s, s + 1):
        for dy in range(-s, s + 1):
            for dz in range(-s, s + 1):
                c = (((mc[0] + dx) % G) * G + (mc[1] + dy) % G) * G + (mc[2] + dz) % G
                for q in range(cs[c], cs[c] + cc[c]):
                    k = int(ci[q])
                    if k in (i, j):
                        continue
                    e = pdelta(m, pos[k], L) if rev else pdelta(pos[k], m, L)
                    if dot(e) < f32(r_sq - eps):
                        return False
    return True


def keep(i, j, frame, q):
    h = ((i * 73856093) & 0xFFFFFFFF) ^ ((j * 19349663) & 0xFFFFFFFF) ^ ((frame * 83492791) & 0xFFFFFFFF)
    h = h - (1 << 32) if h >= (1 << 31) else h
    return q <= 1 or int(math.fmod(h, q)) == 0


def _foam(n, seed, G=5):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-0.5, 0.5, (n, 3)).astype(np.float32)
    rad = rng.uniform(0.04, 0.09, n).astype(np.float32)
    p = O.OracleParams(n=n, L=1.0, r_max_cell=0.5 / G)
    assert p.G == G
    grid = O.grid_build(pos, p)
    return pos, rad, grid, p


@pytest.mark.parametrize("seed,cap", [(1, 28), (2, 6)])
def test_candidates_match_transcription(seed, cap):
    pos, rad, grid, p = _foam(180, seed)
    tp = O.TopoParams(cap=cap, cell_size=1.0 / p.G)
    pairs, pc, tr = O.topo_candidates(pos, rad, grid, p, tp)
    want, wtr = py_candidates(pos, rad, grid, 1.0, p.G, tp.mult, cap)
    for i in range(p.n):
        assert list(pairs[i, :pc[i]]) == want[i], i
    assert list(tr) == wtr
    if cap == 6:
        assert tr.sum() > 0  # the cap binds


@pytest.mark.parametrize("stride,early", [(1, False), (3, True)])
def test_gabriel_matches_transcription(stride, early):
    pos, rad, grid, p = _foam(160, 3)
    tp = O.TopoParams(stride=stride, early_exit=early, deg_high=9.0, cell_size=1.0 / p.G)
    pairs, pc, _ = O.topo_candidates(pos, rad, grid, p, tp)
    ema = np.random.default_rng(4).uniform(5, 14, p.n).astype(np.float32)
    frame = 7
    deg = O.topo_gabriel(pos, grid, pairs, pc, ema, frame, p, tp)
    want = np.zeros(p.n, np.int64)
    for i in range(p.n):
        for j in pairs[i, :pc[i]]:
            j = int(j)
            if not keep(i, j, frame, stride):
                continue
            if early and ema[i] >= f32(9.0) and ema[j] >= f32(9.0):
                continue
            d2 = dot(pdelta(pos[i], pos[j], 1.0))
            if d2 < f32(1e-16):
                continue
            if py_gabriel_pair(pos, grid, i, j, d2, 1.0, p.G, tp.cell_size, False):
                want[i] += 1
                want[j] += 1
    assert np.array_equal(deg, want)
    assert deg.sum() > 0


def test_batched_and_knn_match_transcription():
    pos, rad, grid, p = _foam(150, 5)
    tp = O.TopoParams(cap=28, cell_size=1.0 / p.G)
    pairs = np.zeros((p.n, tp.cap), np.int32)
    pc = np.zeros(p.n, np.int32)
    tr = np.zeros(p.n, np.int32)
    deg = np.zeros(p.n, np.int32)
    for b in range(3):
        O.topo_batched(pos, rad, grid, b, 3, 2, 11, pairs, pc, tr, deg, p, tp)
    want = np.zeros(p.n, np.int64)
    cc, cs, ci = grid
    for i in range(p.n):
        cand = []
        for c in cells27(home(pos[i], 1.0, p.G), p.G):
            for k in range(cs[c], cs[c] + cc[c]):
                j = int(ci[k])
                if j <= i or not keep(i, j, 11, 2):
                    continue
                th = f32(f32(tp.mult) * f32(rad[i] + rad[j]))
                if dot(pdelta(pos[i], pos[j], 1.0)) <= f32(th * th):
                    cand.append(j)
        assert pc[i] == len(cand)
        for j in cand[:tp.cap]:
            d2 = dot(pdelta(pos[i], pos[j], 1.0))
            if d2 >= f32(1e-16) and py_gabriel_pair(pos, grid, i, j, d2, 1.0, p.G, tp.cell_size,
                                                      True):
                want[i] += 1
                want[j] += 1
    assert np.array_equal(deg, want)
    knn = O.topo_knn(pos, rad, grid, 5, p, tp)
    for i in range(p.n):
        lim = f32(f32(tp.mult) * rad[i])
        cnt = sum(1 for c in cells27(home(pos[i], 1.0, p.G), p.G)
                  for k in range(cs[c], cs[c] + cc[c])
                  if int(ci[k]) != i and dot(pdelta(pos[i], pos[int(ci[k])], 1.0)) <= f32(lim * lim))
        assert knn[i] == min(cnt, 5)


def test_known_answers():
    # B at the midpoint of A-C is a witness for A-C; A-B and B-C are Gabriel edges
    pos = np.array([[-0.1, 0.0, 0.0], [0.0, 0.001, 0.0], [0.1, 0.0, 0.0]], np.float32)
    rad = np.full(3, 0.05, np.float32)
    p = O.OracleParams(n=3, L=1.0, r_max_cell=0.1)
    grid = O.grid_build(pos, p)
    tp = O.TopoParams(stride=1, early_exit=False, cell_size=0.2)
    pairs, pc, tr = O.topo_candidates(pos, rad, grid, p, tp)
    assert list(pc) == [2, 1, 0] and list(tr) == [0, 0, 0]
    deg = O.topo_gabriel(pos, grid, pairs, pc, np.zeros(3, np.float32), 0, p, tp)
    assert list(deg) == [1, 2, 1]


def test_ema_and_radius_rule():
    deg = np.array([0, 10, 20], np.int32)
    ema = np.array([5.0, 5.0, 5.0], np.float32)
    O.topo_ema(deg, ema, 0.1)
    want = [f32(f32(f32(0.1) * f32(d)) + f32(f32(f32(1.0) - f32(0.1)) * f32(5.0))) for d in deg]
    assert list(ema) == want
    rad = np.array([0.01, 0.01, 0.01, 0.029], np.float32)
    deff = np.array([5.0, 12.0, 25.0, 5.0], np.float32)
    O.topo_radii(rad, deff, 10, 18, 0.02, 0.03, 0.005, 0.0295)
    assert rad[0] == f32(f32(0.01) * f32(1.02))
    assert rad[1] == f32(0.01)
    assert rad[2] == f32(f32(0.01) * f32(0.97))
    assert rad[3] == f32(0.0295)  # clamped
