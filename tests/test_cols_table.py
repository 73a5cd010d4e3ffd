"""Columns-per-lane choice per length bucket (ragged.cols_table, bucket_of):
host logic, on CPU."""

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_buckets():
    from orihime_b200 import ragged

    assert ragged.bucket_of(32, 32) == "0:0"
    assert ragged.bucket_of(300, 63) == "0:256"
    assert ragged.bucket_of(255, 64) == "64:0"
    assert ragged.bucket_of(2048, 2048) == "1024:256"
    assert ragged.bucket_of(256, 1023) == "512:256"
    # every bucket has a default
    for a2 in ragged.L2_EDGES:
        for a1 in ragged.L1_EDGES:
            assert ragged.DEFAULT_COLS[f"{a2}:{a1}"] in (2, 4, 8)


def test_table_overrides(monkeypatch, tmp_path):
    from orihime_b200 import ragged

    monkeypatch.setenv("ORIHIME_B200_CACHE", str(tmp_path))
    monkeypatch.delenv("ORIHIME_B200_COLS", raising=False)
    assert ragged.cols_table() == ragged.DEFAULT_COLS
    monkeypatch.setenv("ORIHIME_B200_COLS", "0:0=4,1024:256=2")
    t = ragged.cols_table()
    assert t["0:0"] == 4 and t["1024:256"] == 2 and t["512:0"] == ragged.DEFAULT_COLS["512:0"]
    monkeypatch.setenv("ORIHIME_B200_COLS", json.dumps({"64:0": 8}))
    assert ragged.cols_table()["64:0"] == 8
    p = tmp_path / "t.json"
    p.write_text(json.dumps({"128:256": 4}))
    monkeypatch.setenv("ORIHIME_B200_COLS", str(p))
    assert ragged.cols_table()["128:256"] == 4


def test_bench_batch_computed_cells_reported():
    """Cells the bands compute per useful cell on the bench batch (dead
    columns of each pair's last band, 31 fill and drain steps per band) at 4
    columns per lane for all pairs and with the bucket table.  The table is
    chosen for time, not for this count: 8 columns per lane computes more
    dead cells on wide pairs but halves the per-step work of the bands."""
    import bench
    from orihime_b200 import ragged

    ln = bench.workload_lengths(3)
    useful = float((ln[:, 0] * ln[:, 1]).sum())
    r4 = ragged.pair_cost(ln, 4).sum() / useful
    cols = np.array([ragged.DEFAULT_COLS[ragged.bucket_of(int(a), int(b))] for a, b in ln])
    w = 32 * cols
    nb = np.maximum(1, (ln[:, 1] + w - 1) // w)
    mixed = (nb * (ln[:, 0] + 31) * w).sum() / useful
    print(f"  computed / useful cells: 4 columns per lane {r4:.3f}, bucket table {mixed:.3f}")
    assert 1.0 < r4 < 1.3 and 1.0 < mixed < 1.4


def test_bench_traffic_profile_per_cols():
    """The bench's roofline traffic comes from the committed DRAM capture of
    the adjoint it launched: one per columns-per-lane choice."""
    import bench

    for cols in (4, 8):
        v, src = bench.profile_traffic(cols)
        assert v is not None and 8.0 <= v <= 20.0, (cols, v)
        assert os.path.exists(os.path.join(ROOT, src))
    assert bench.profile_traffic(2) == (None, None)
