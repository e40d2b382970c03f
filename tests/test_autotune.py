"""Launch-shape tuning: the table the tuner writes and the library reads, the
library's lookup of it (host only), and on the GPU that a tuned shape is
never slower than the default and that uploads pick it up."""
import ctypes

import numpy as np
import pytest

from vlasiator_b200 import autotune


def _lookup(path, device, mean_blocks):
    from vlasiator_b200 import vlgpu
    lib = vlgpu.load()
    cfg = vlgpu.CLaunchT()
    code = lib.vlgpu_launch_table_lookup(path.encode(), device.encode(), float(mean_blocks), ctypes.byref(cfg))
    return code, cfg.as_tuple()


def test_table_round_trip_and_library_lookup(tmp_path):
    path = str(tmp_path / "launch_table.tsv")
    autotune.update_table(path, "NVIDIA B200", 0.0, (4, 2, 3, 0))
    autotune.update_table(path, "NVIDIA B200", 600.0, (3, 2, 2, 0))
    autotune.update_table(path, "NVIDIA B200", 2400.0, (4, 1, 3, 5))
    autotune.update_table(path, "Other GPU", 0.0, (1, 1, 1, 1))
    autotune.update_table(path, "NVIDIA B200", 600.0, (2, 2, 2, 0))  # replaces the bucket's entry
    rows = autotune.read_table(path)
    assert len(rows) == 4
    assert ("NVIDIA B200", 600.0, (2, 2, 2, 0)) in rows
    # the library's own parser: the bucket with the largest lower bound <= mean blocks
    assert _lookup(path, "NVIDIA B200", 100) == (0, (4, 2, 3, 0))
    assert _lookup(path, "NVIDIA B200", 600) == (0, (2, 2, 2, 0))
    assert _lookup(path, "NVIDIA B200", 1e5) == (0, (4, 1, 3, 5))
    assert _lookup(path, "Other GPU", 5000) == (0, (1, 1, 1, 1))
    assert _lookup(path, "NVIDIA H100", 100)[0] == 9  # VLGPU_ENOENT
    assert _lookup(str(tmp_path / "missing.tsv"), "NVIDIA B200", 100)[0] == 9


def test_buckets_and_candidates():
    assert autotune.bucket_of(10) == 0.0
    assert autotune.bucket_of(1423) == 600.0
    assert autotune.bucket_of(9000) == 2400.0
    c = autotune.candidates((4, 2, 3))
    assert len(c) == 24 and (4, 2, 3, 0) in c and (1, 1, 1, 0) in c


@pytest.mark.gpu
def test_tuned_shape_is_not_slower_and_uploads_use_it(tmp_path, monkeypatch):
    from vlasiator_b200 import vlgpu
    from vlasiator_b200.mesh import CHARGE, MASS_PROTON, VelocityMesh
    from vlasiator_b200.projects import random_drifting_cells
    import torch
    mesh = VelocityMesh()
    cells = random_drifting_cells(256, seed=5, mesh=mesh)
    total = sum(c.n_blocks for c in cells)
    B = np.stack([c.B for c in cells])
    dt = 0.01 * 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(B, axis=1))
    orders = [0, 1, 2]
    path = str(tmp_path / "launch_table.tsv")
    monkeypatch.setenv("VLGPU_LAUNCH_TABLE", path)
    with vlgpu.Batch(mesh, len(cells), 3 * total + 65536) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        assert b.launch()[0] >= 1  # no table yet: the defaults
        default = b.launch()
        b.accelerate(B, dt, 0)
        maxima = default[:3]
        shapes = [(r, m, a, 0) for r in sorted({1, maxima[0] // 2 or 1, maxima[0]})
                  for m in sorted({1, maxima[1]}) for a in sorted({1, maxima[2]})]
        best, times = autotune.tune_batch(b, orders, steps=2, shapes=shapes)
        # the choice against the default on fresh timings
        b.set_launch(best)
        t_best = min(autotune.time_steps(b, orders, 3) for _ in range(2))
        b.set_launch((0, 0, 0, 0))
        t_def = min(autotune.time_steps(b, orders, 3) for _ in range(2))
        assert t_best <= 1.05 * t_def, (best, t_best, t_def)
    # the table is consulted at upload, and a pinned shape is kept
    device = torch.cuda.get_device_name(0)
    bucket = autotune.bucket_of(total / len(cells))
    autotune.update_table(path, device, bucket, (1, 1, 1, 0))
    with vlgpu.Batch(mesh, len(cells), 3 * total + 65536) as b:
        b.upload([c.gids for c in cells], [c.data for c in cells])
        assert b.launch()[:3] == (1, 1, 1)
        b.accelerate(B, dt, 1)  # runs with the table's shapes
        assert not b.status().any()
        b.set_launch((2, 1, 1, 0))
        b.upload([c.gids for c in cells], [c.data for c in cells])
        assert b.launch()[:3] == (min(2, default[0]), 1, 1)
        b.set_launch(None)
        b.upload([c.gids for c in cells], [c.data for c in cells])
        assert b.launch()[:3] == (1, 1, 1)
