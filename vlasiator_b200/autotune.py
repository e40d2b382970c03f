"""Launch-shape tuning of the batched acceleration step.

The persistent kernels of a batch run with a number of CTAs per SM (the
acceleration remap, whose CTAs each keep 16 column sets in flight; the
moments; the block adjustment; the translation walk).  Which numbers are
fastest depends on the device and on the cells' sizes: few large cells favour
full occupancy, many small ones can favour fewer resident CTAs.  This module
times whole acceleration steps (CUDA events on the batch's stream) for every
candidate shape on a workload of one bucket of mean blocks per cell, and
writes the fastest shapes to the launch table that every batch consults when
cells are uploaded (include/vlgpu.h, vlgpu_batch_set_launch).

    python -m vlasiator_b200.autotune [--table PATH] [--cells N] [--steps K]

tunes the three buckets on cells drawn from the batched-acceleration workload
(drifting Maxwellians sorted by size) and writes the table for this GPU.
"""
from __future__ import annotations

import argparse
import itertools
import os

import numpy as np

# lowest mean blocks per cell of each bucket
BUCKETS = (0.0, 600.0, 2400.0)


def table_path() -> str:
    """The launch table the library reads: $VLGPU_LAUNCH_TABLE, else
    $XDG_CACHE_HOME/vlgpu/launch_table.tsv (~/.cache when unset)."""
    if os.environ.get("VLGPU_LAUNCH_TABLE"):
        return os.environ["VLGPU_LAUNCH_TABLE"]
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "vlgpu", "launch_table.tsv")


def bucket_of(mean_blocks: float) -> float:
    """The bucket (its lowest mean block count) a workload falls in."""
    return max(b for b in BUCKETS if b <= mean_blocks)


def read_table(path: str) -> list:
    """Entries (device, lowest mean blocks, (remap, moments, adjust, translate))."""
    rows = []
    if not os.path.exists(path):
        return rows
    with open(path) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            parts = line.rstrip("\n").split("\t")
            if len(parts) != 6:
                continue
            rows.append((parts[0], float(parts[1]), tuple(int(x) for x in parts[2:])))
    return rows


def write_table(path: str, rows: list) -> None:
    """Writes the entries, one per line, in the format the library parses."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write("# device\tlowest mean blocks per cell\tremap\tmoments\tadjust\ttranslate (CTAs per SM)\n")
        for dev, lo, shape in sorted(rows, key=lambda r: (r[0], r[1])):
            f.write(f"{dev}\t{lo:g}\t" + "\t".join(str(int(x)) for x in shape) + "\n")


def update_table(path: str, device: str, bucket: float, shape) -> None:
    """Replaces (or adds) the entry of one device and bucket, keeping the rest."""
    rows = [r for r in read_table(path) if not (r[0] == device and r[1] == bucket)]
    rows.append((device, float(bucket), tuple(int(x) for x in shape)))
    write_table(path, rows)


def candidates(maxima) -> list:
    """Every shape from 1 CTA per SM up to each kernel's occupancy maximum
    (remap, moments, adjust; translation left at its maximum)."""
    r, m, a = maxima
    return [(x, y, z, 0) for x, y, z in itertools.product(range(1, r + 1), range(1, m + 1), range(1, a + 1))]


def time_steps(batch, orders, steps: int) -> float:
    """Device time (ms) of `steps` acceleration steps, CUDA events on the batch's stream."""
    import torch
    stream = torch.cuda.ExternalStream(batch.stream_handle())
    batch.sync()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for s in range(steps):
        batch.accelerate_device(orders[s % len(orders)])
    end.record(stream)
    batch.sync()
    return start.elapsed_time(end) / steps


def tune_batch(batch, orders, steps: int = 3, shapes=None) -> tuple:
    """Times every candidate shape on the batch (its cells uploaded and one
    step taken, so the fields are staged) and returns (best shape, {shape: ms}).
    The default shape (every kernel at its maximum) is among the candidates,
    so the choice is never slower than it on the timed steps."""
    batch.set_launch((0, 0, 0, 0))
    maxima = batch.launch()[:3]
    shapes = shapes or candidates(maxima)
    times = {}
    time_steps(batch, orders, 1)  # warm the default once more
    for shape in shapes:
        batch.set_launch(shape)
        times[tuple(shape)] = time_steps(batch, orders, steps)
    best = min(times, key=times.get)
    batch.set_launch(None)
    return best, times


def bucket_workloads(n_cells: int, seed: int = 2026):
    """Cells of the batched-acceleration workload sorted by size and cut into
    one workload per bucket (mean blocks per cell in the bucket's range)."""
    from vlasiator_b200.mesh import VelocityMesh
    from vlasiator_b200.projects import random_drifting_cells
    mesh = VelocityMesh()
    cells = sorted(random_drifting_cells(4 * n_cells, seed=seed, mesh=mesh), key=lambda c: c.n_blocks)
    out = {}
    for k, lo in enumerate(BUCKETS):
        hi = BUCKETS[k + 1] if k + 1 < len(BUCKETS) else float("inf")
        pick = [c for c in cells if lo <= c.n_blocks < hi][:n_cells]
        if pick:
            out[lo] = pick
    return mesh, out


def tune_and_save(path: str | None = None, n_cells: int = 1024, steps: int = 3, seed: int = 2026) -> dict:
    """Tunes every bucket on this GPU and writes its entries; returns
    {bucket: (best shape, default ms, best ms)}."""
    import torch

    from vlasiator_b200 import vlgpu
    from vlasiator_b200.mesh import CHARGE, MASS_PROTON
    path = path or table_path()
    device = torch.cuda.get_device_name(0)
    mesh, work = bucket_workloads(n_cells, seed)
    rng = np.random.default_rng(seed)
    orders = [int(x) for x in rng.integers(0, 3, size=8)]
    result = {}
    for lo, cells in work.items():
        total = sum(c.n_blocks for c in cells)
        B = np.stack([c.B for c in cells])
        dt = 0.01 * 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(B, axis=1))
        with vlgpu.Batch(mesh, len(cells), 3 * total + 65536) as b:
            b.upload([c.gids for c in cells], [c.data for c in cells])
            b.accelerate(B, dt, orders[0])
            best, times = tune_batch(b, orders, steps)
        default = max(times, key=lambda s: sum(s[:3]))  # every kernel at its maximum
        update_table(path, device, lo, best)
        result[lo] = (best, times[default], times[best], times, len(cells), total / len(cells))
    return result


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--table", default=None, help="launch table to write (default: the library's)")
    ap.add_argument("--cells", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=3)
    args = ap.parse_args()
    res = tune_and_save(args.table, args.cells, args.steps)
    for lo, (best, t_def, t_best, times, n, mean) in sorted(res.items()):
        print(f"bucket >= {lo:g} blocks/cell ({n} cells, mean {mean:.0f} blocks): best {best} "
              f"{t_best:.3f} ms/step (default {t_def:.3f})")
        ranked = sorted(times.items(), key=lambda kv: kv[1])
        for shape, ms in ranked[:4] + ranked[-2:]:
            print(f"    {shape}: {ms:.3f} ms/step")
    print("table:", args.table or table_path())


if __name__ == "__main__":
    main()
