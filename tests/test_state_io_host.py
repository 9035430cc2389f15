"""run.py's particle CSV (run.py:608-629) written from host arrays: header,
row layout, value formatting and an exact float32 round trip."""
import csv

import numpy as np

from fos.state_io import CSV_HEADER, export_csv, read_csv


def test_csv_layout_and_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    n = 500
    pos = rng.uniform(-0.5, 0.5, (n, 3)).astype(np.float32)
    rad = rng.uniform(0.002, 0.03, n).astype(np.float32)
    fsc = rng.integers(0, 32, n).astype(np.int32)
    pos[0] = np.float32([0.1, -0.25, 0.5])
    rad[0] = np.float32(0.0125)
    fsc[0] = 12
    path = export_csv(str(tmp_path / "particle_data_frame_7.csv"), pos, rad, fsc)
    lines = open(path).read().splitlines()
    assert lines[0] == ",".join(CSV_HEADER)
    assert lines[1] == "0,0.1,-0.25,0.5,0.0125,12"
    assert len(lines) == n + 1
    # the same rows a csv.writer over numpy scalars writes (run.py's loop)
    with open(tmp_path / "ref.csv", "w", newline="") as fh:
        w = csv.writer(fh)
        w.writerow(CSV_HEADER)
        for i in range(n):
            w.writerow([i, pos[i][0], pos[i][1], pos[i][2], rad[i], fsc[i]])
    assert open(tmp_path / "ref.csv").read() == open(path).read()
    back = read_csv(path)
    assert np.array_equal(back["pos"], pos) and np.array_equal(back["rad"], rad)
    assert np.array_equal(back["fsc"], fsc) and np.array_equal(back["id"], np.arange(n))


def test_csv_active_prefix_only(tmp_path):
    pos = np.zeros((10, 3), np.float32)
    rad = np.full(10, 0.01, np.float32)
    fsc = np.zeros(10, np.int32)
    path = export_csv(str(tmp_path / "a.csv"), pos, rad, fsc, n=4)
    assert len(open(path).read().splitlines()) == 5
