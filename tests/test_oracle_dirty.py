"""The oracle's dirty-tile marking (jfa.py:966-1024) against a numpy float32
transcription: thresholds in VOXEL_SIZE units, tile crossings, the PBC halo
and the count."""
import numpy as np

from oracle import oracle as O

f32 = np.float32


def _np_mark(pos, rad, pp, rp, R, L=1.0, pos_frac=0.5, rad_frac=0.25, halo=1):
    t = (R + 15) // 16
    vs = L / R
    d = (pos - pp).astype(np.float32)
    dpos = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
    drad = np.abs(rad - rp)

    def tile(x):
        v = np.floor(((x + f32(0.5 * L)) / f32(L)) * f32(R)).astype(np.int64) % R
        return v // 16

    tc, tp = tile(pos), tile(pp)
    dirty_p = (dpos > f32(pos_frac * vs)) | (drad > f32(rad_frac * vs)) | (tc != tp).any(1)
    out = np.zeros((t, t, t), np.uint8)
    for c in tc[dirty_p]:
        for ox in range(-halo, halo + 1):
            for oy in range(-halo, halo + 1):
                for oz in range(-halo, halo + 1):
                    out[(c[0] + ox) % t, (c[1] + oy) % t, (c[2] + oz) % t] = 1
    return out


def test_dirty_marking_matches_transcription():
    rng = np.random.default_rng(0)
    n, R = 3000, 128
    pp = rng.uniform(-0.5, 0.5, (n, 3)).astype(np.float32)
    rp = rng.uniform(0.005, 0.02, n).astype(np.float32)
    pos = pp.copy()
    rad = rp.copy()
    mv = rng.random(n) < 0.003
    pos[mv] += rng.normal(0, 0.01, (mv.sum(), 3)).astype(np.float32)   # some move > 0.5 voxel
    rz = rng.random(n) < 0.002
    rad[rz] *= f32(1.5)
    p = O.OracleParams(n=n, R=R)
    t = (R + 15) // 16
    dirty = np.zeros(t ** 3, np.uint8)
    O.dirty_mark(pos, rad, pp, rp, dirty, p)
    want = _np_mark(pos, rad, pp, rp, R)
    assert np.array_equal(dirty.reshape(t, t, t), want)
    assert O.dirty_count(dirty, R) == int(want.sum())
    assert 0 < want.sum() < t ** 3
    # nothing moved: nothing marked
    none = np.zeros(t ** 3, np.uint8)
    O.dirty_mark(pp, rp, pp, rp, none, p)
    assert O.dirty_count(none, R) == 0
