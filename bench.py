"""Benchmark of the B200 Vlasov acceleration hot path.

Workload (batched acceleration): 4096 independent spatial cells, each a
drifting Maxwellian with n log-uniform in [1e5, 1e7] m^-3, T log-uniform in
[1e5, 1e7] K, |V| uniform in [0, 800] km/s along a random direction, B of
random direction with |B| uniform in [5, 50] nT, on the +-4020 km/s mesh with
dv = 30 km/s (67^3 blocks of 4^3 cells), fp32 VDF, minValue 1e-15.  One step =
one SLICE-3D acceleration step of every cell (FP64 moments for the pivot,
FP64 gyration geometry, three 1D remaps in a random dimension order) with
dt = 0.01 gyroperiod per cell.

Metric: phase-space cell-updates/s, one update = one of the 64 cells of a
block existing before the step advanced through the three sweeps.  `value`
is device time with the batch resident in HBM; `e2e` runs the same step
through the C ABI from pinned host buffers, the cells split into 32 batches
whose uploads, steps and downloads overlap; `cpu_baseline` and
`--impl reference` time the reference's own map_1d built from its sources.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --workload vlasov     # full Vlasov step, 64x64x16 sine-wave grid
    python bench.py --workload serve      # Poisson stream of requests

Prints one JSON line (rank 0).  Under torchrun each rank runs its own batch
(independent cells, weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from vlasiator_b200.mesh import CHARGE, MASS_PROTON, WID3, VelocityMesh  # noqa: E402
from vlasiator_b200.projects import random_drifting_cells  # noqa: E402

METRIC = "phase-space cell-updates/s (batched vs plain, same GPU); p50/p99 solve latency"
UNIT = "cell-updates/s"
WORKLOAD = "batched acceleration, 4096 drifting Maxwellian cells, 1 SLICE-3D step (PPM), dt=0.01 gyroperiod"
BYTES_PER_CELL_SWEEP = 8  # read + write one fp32 phase-space cell per 1D sweep
# DRAM bytes (read + write) of one remap_walk_kernel launch per source block,
# from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum = 203.8 +
# 175.9 MB) of the 512-cell case of this workload (705,499 blocks at the step's
# start), fused arithmetic; scaled by the source blocks of a launch to give the
# full-size traffic per launch.
REMAP_DRAM_BYTES_PER_BLOCK = 379.7e6 / 705499
DEFAULT_SEED = 2026  # the workload's seed unless --seed says otherwise


def workload(n_cells: int, seed: int):
    mesh = VelocityMesh()
    cells = random_drifting_cells(n_cells, seed=seed, mesh=mesh)
    offs = np.zeros(n_cells + 1, np.uint64)
    offs[1:] = np.cumsum([c.n_blocks for c in cells])
    gids = np.concatenate([c.gids for c in cells]).astype(np.uint32)
    data = np.concatenate([c.data for c in cells]).astype(np.float32)
    B = np.stack([c.B for c in cells])
    Tg = 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(B, axis=1))
    dt = 0.01 * Tg
    return mesh, offs, gids, data, B, dt


def map_orders(steps: int, seed: int):
    rng = np.random.default_rng(seed + 7919)
    return [int(x) for x in rng.integers(0, 3, size=steps)]


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for s in self.samples for q in range(4) if len(s) > 5 + q and "Active" in s[5 + q]
                          and "Not" not in s[5 + q]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def allreduce_max(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own map_1d (oracle/_ref) on host cores
# ---------------------------------------------------------------------------
def cpu_reference_rate(mesh, offs, gids, data, B, dt, orders, sample_cells, target_s=12.0):
    """Times the reference's full acceleration step (pivot moments, geometry,
    map_1d x3, adjustVelocityBlocks, moments with pressure) on the workload's
    cells with all host threads, as many steps as fit in about target_s;
    returns (cell-updates/s, cores, sample description, kind) or None."""
    from oracle.oracle import ReferenceBuild, reference_available  # CPU baseline leg only
    if not reference_available("sp"):
        return None
    n = min(sample_cells, len(offs) - 1)
    glist = [gids[offs[c]:offs[c + 1]] for c in range(n)]
    dlist = [data[offs[c]:offs[c + 1]] for c in range(n)]
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    cores = ref.max_threads()
    h = ref.create(glist, dlist, [1e-15] * n)
    updates, elapsed, reps = 0, 0.0, 0
    while elapsed < target_s and reps < 64:
        blocks = sum(ref.lib.ref_cells_block_count(h, c) for c in range(n))
        t0 = time.perf_counter()
        ref.full_step(h, B[:n], dt[:n], orders[reps % len(orders)], CHARGE, MASS_PROTON)
        elapsed += time.perf_counter() - t0
        updates += WID3 * blocks
        reps += 1
    ref.destroy(h)
    what = "all" if n == len(offs) - 1 else f"the first {n} of the"
    return (updates / elapsed, cores,
            f"{what} {len(offs) - 1} cells of the workload x {reps} full acceleration steps ({updates} "
            f"cell-updates): the reference's map_1d, adjust_velocity_blocks and moment templates", "reference")


def cpu_vlasov_rate(dims, target_s=12.0):
    """Times the reference's full Vlasov step (trans_map_1d_amr z, x, y, the _R
    moments, the full acceleration step with spatial neighbours in the
    adjustment) on a smaller periodic grid of the same sine-wave workload with
    all host threads; returns (cell-updates/s, cores, sample description, kind)
    or None."""
    from oracle.oracle import ReferenceBuild, reference_available  # CPU baseline leg only
    from vlasiator_b200.grid import grid_neighbors
    from vlasiator_b200.projects import sinewave_grid
    if not reference_available("sp"):
        return None
    mesh = VelocityMesh()
    cells = sinewave_grid(dims, mesh)
    B = np.stack([c.B for c in cells])
    nbrs = grid_neighbors(dims)
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    cores = ref.max_threads()
    h = ref.create([c.gids for c in cells], [c.data for c in cells], [1e-15] * len(cells))
    dt = 0.2
    updates, elapsed, steps = 0, 0.0, 0
    while elapsed < target_s and steps < 50:
        blocks = sum(ref.lib.ref_cells_block_count(h, c) for c in range(len(cells)))
        t0 = time.perf_counter()
        ref.vlasov_step(h, dims, (3e5, 3e5, 3e5), B, dt, steps % 3, CHARGE, MASS_PROTON, nbrs)
        elapsed += time.perf_counter() - t0
        updates += WID3 * blocks
        steps += 1
    ref.destroy(h)
    return (updates / elapsed, cores,
            f"{dims[0]}x{dims[1]}x{dims[2]} periodic grid of the same workload x {steps} full Vlasov steps "
            f"({updates} cell-updates): the reference's trans_map_1d_amr, map_1d, adjust_velocity_blocks and "
            f"moment templates", "reference")


def run_reference_arm(args):
    """The reference's own CPU code for the same workload and metric: its full
    acceleration step (ReferenceBuild.full_step) on every cell of the
    workload, all host threads, W untimed and K timed steps."""
    world, rank, local, pg = dist_setup()
    if rank != 0:
        return 0
    from oracle.oracle import reference_available
    mesh, offs, gids, data, B, dt = workload(args.cells, args.seed)
    orders = map_orders(max(args.steps, 1), args.seed)
    if not reference_available("sp"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (reference tree absent)"}))
        return 0
    from oracle.oracle import ReferenceBuild
    ref = ReferenceBuild("sp")
    ref.init(mesh)
    cores = ref.max_threads()
    n = min(args.ref_sample, args.cells) if args.ref_sample > 0 else args.cells
    glist = [gids[offs[c]:offs[c + 1]] for c in range(n)]
    dlist = [data[offs[c]:offs[c + 1]] for c in range(n)]
    total = int(offs[n])
    h = ref.create(glist, dlist, [1e-15] * n)
    for w in range(args.warmup):
        ref.full_step(h, B[:n], dt[:n], orders[w % len(orders)], CHARGE, MASS_PROTON)
    upd = 0
    t_total = 0.0
    for s in range(args.steps):
        blocks = sum(ref.lib.ref_cells_block_count(h, c) for c in range(n))
        t0 = time.perf_counter()
        ref.full_step(h, B[:n], dt[:n], orders[s], CHARGE, MASS_PROTON)
        t_total += time.perf_counter() - t0
        upd += WID3 * blocks
    ref.destroy(h)
    rate = upd / t_total
    config = {"workload": WORKLOAD, "cells_per_gpu": args.cells, "blocks_per_gpu": total,
              "mean_blocks_per_cell": total / n, "l2": "inputs larger than L2 (126 MB)",
              "parallelism": "host threads (OpenMP over cells, as cpu_accelerate_cells)"}
    if n < args.cells:
        config["sampled_cells"] = n
    line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_total / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded drifting Maxwellians)",
            "config": config,
            "impl": "reference",
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": (f"{'all' if n == args.cells else f'the first {n} of the'} {args.cells} "
                                        f"cells, {args.steps} full acceleration steps (map_1d x3, "
                                        f"adjust_velocity_blocks, moments)")},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    world, rank, local, pg = dist_setup()
    from vlasiator_b200 import vlgpu
    vlgpu.load()
    import torch
    torch.cuda.set_device(local)
    mesh, offs, gids, data, B, dt = workload(args.cells, args.seed + 1000 * rank)
    orders = map_orders(args.warmup + args.steps, args.seed)
    total = int(offs[-1])
    cap = int(total * 1.6) + 262144
    batch = vlgpu.Batch(mesh, args.cells, cap, device=local, exact=args.exact)
    batch.upload_packed(offs, gids, data)
    stream = torch.cuda.ExternalStream(batch.stream_handle(), device=local)

    # first call uploads the per-cell fields; later steps reuse them on the device
    batch.accelerate(B, dt, orders[0])
    for w in range(1, args.warmup):
        batch.accelerate_device(orders[w])
    batch.sync()
    st0 = batch.stats()
    batch.profile(True)
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    if args.graph:
        # CUDA graphs of two steps each; dimension orders (0,1), (2,0), (1,2) repeat
        if args.steps % 2:
            raise SystemExit("--graph times pairs of steps: --steps must be even")
        batch.profile(False)
        for g, pair in enumerate([(0, 1), (2, 0), (1, 2)]):
            batch.capture(g, "accel", list(pair))
        st0 = batch.stats()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local) as clk:
        evs[0].record(stream)
        if args.graph:
            for q in range(args.steps // 2):
                batch.replay(q % 3)
                evs[2 * q + 1].record(stream)
                evs[2 * q + 2].record(stream)
        else:
            for s in range(args.steps):
                batch.accelerate_device(orders[args.warmup + s])
                evs[s + 1].record(stream)
        evs[-1].synchronize()
    torch.cuda.synchronize()
    ms = evs[0].elapsed_time(evs[-1])
    step_ms = np.array([evs[q].elapsed_time(evs[q + 1]) for q in range(args.steps)])
    if args.graph:  # a replay covers two steps: split its time evenly
        step_ms = np.repeat(step_ms[0::2] / 2.0, 2)
    st1 = batch.stats()
    status = batch.status()
    updates = WID3 * (st1["step_blocks"] - st0["step_blocks"])
    src_blocks = st1["src_blocks"] - st0["src_blocks"]
    launches = st1["launches"] - st0["launches"]
    remap_ms = st1["remap_ns"] * 1e-6
    remap_n = st1["remap_profiled"]
    ms_max = allreduce_max(pg, ms)
    updates_all = allreduce_sum(pg, float(updates))
    value = updates_all / (ms_max * 1e-3)
    peak, peak_kind = measured_peak()
    achieved = (BYTES_PER_CELL_SWEEP * WID3 * src_blocks / remap_n) / (remap_ms * 1e-3 / remap_n) / 1e9 \
        if remap_n else None
    if args.graph:
        # no per-launch events inside graphs: the remap's share of the step
        # comes from the eager timing of the warm-up steps instead
        achieved = None

    # the plain per-cell launch path (the drop-in baseline) on the same batch
    plain = None
    if args.plain_steps > 0:
        batch.profile(False)
        batch.upload_packed(offs, gids, data)
        p_steps = max(1, min(args.steps, args.plain_steps))
        pst0 = batch.stats()
        pe0 = torch.cuda.Event(enable_timing=True)
        pe1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        pe0.record(stream)
        for s in range(p_steps):
            batch.accelerate_device(orders[args.warmup + s], per_cell=True)
        pe1.record(stream)
        pe1.synchronize()
        p_ms = allreduce_max(pg, pe0.elapsed_time(pe1))
        p_upd = allreduce_sum(pg, float(WID3 * (batch.stats()["step_blocks"] - pst0["step_blocks"])))
        p_value = p_upd / (p_ms * 1e-3)
        plain = {"value": p_value, "unit": UNIT, "steps": p_steps, "ms_per_step": p_ms / p_steps,
                 "batched_over_plain": value / p_value,
                 "path": "vlgpu_accelerate_per_cell: one columnize + remap launch sequence per cell and sweep"}

    batch.close()

    # end to end through the C ABI: host -> device copy of the step's input,
    # the step, device -> host copy of the result (pinned host buffers).  The
    # cells are split into chunks, one batch (and CUDA stream) each, issued
    # with the asynchronous upload / two-phase download so that one chunk's
    # copies overlap the others' steps and copies in the other direction.
    h_gids = torch.from_numpy(gids).pin_memory()
    h_data = torch.from_numpy(data).pin_memory()
    n_chunks = max(1, min(args.e2e_chunks, args.cells))
    bounds = np.linspace(0, args.cells, n_chunks + 1).astype(np.int64)
    chunks = []
    for k in range(n_chunks):
        c0, c1 = int(bounds[k]), int(bounds[k + 1])
        b0, b1 = int(offs[c0]), int(offs[c1])
        cap_k = int((b1 - b0) * 1.6) + 65536
        bk = vlgpu.Batch(mesh, c1 - c0, cap_k, device=local, exact=args.exact)
        chunks.append({"batch": bk, "offs": (offs[c0:c1 + 1] - offs[c0]).astype(np.uint64),
                       "gids": h_gids[b0:b1].numpy(), "data": h_data[b0:b1].numpy(),
                       "B": B[c0:c1], "dt": dt[c0:c1] if np.ndim(dt) else dt,
                       "out_g": torch.empty(cap_k, dtype=torch.int32).pin_memory().numpy().view(np.uint32),
                       "out_d": torch.empty((cap_k, WID3), dtype=torch.float32).pin_memory().numpy()})
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    t_e2e = 0.0
    h2d = d2h = 0
    e2e_updates = 0
    for s in range(e2e_steps + 1):
        t0 = time.perf_counter()
        # every chunk's upload, step and slot read-back is queued first (the
        # host-to-device engine never waits on the host); each download then
        # follows as soon as its chunk's step is done
        for ch in chunks:
            ch["batch"].upload_async(ch["offs"], ch["gids"], ch["data"])
            ch["batch"].accelerate(ch["B"], ch["dt"], orders[s % len(orders)])
            ch["batch"].download_begin()
        outs = [ch["batch"].download_end(ch["out_g"], ch["out_d"]) for ch in chunks]
        for ch in chunks:
            ch["batch"].sync()
        el = time.perf_counter() - t0
        if s > 0:  # the first pass warms the host paths
            t_e2e += el
            e2e_updates += WID3 * total
            for ch, (c_off, c_cnt, g_out, _) in zip(chunks, outs):
                h2d += ch["offs"].nbytes + ch["gids"].nbytes + ch["data"].nbytes
                d2h += c_off.nbytes + c_cnt.nbytes + len(g_out) * (4 + WID3 * 4)
    for ch in chunks:
        ch["batch"].close()
    t_e2e = allreduce_max(pg, t_e2e)
    e2e_value = allreduce_sum(pg, float(e2e_updates)) / t_e2e

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_rate(mesh, offs, gids, data, B, dt, orders, args.cpu_sample)
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded drifting Maxwellians)",
        "config": {"workload": WORKLOAD, "cells_per_gpu": args.cells, "blocks_per_gpu": total,
                   "mean_blocks_per_cell": total / args.cells, "l2": "inputs larger than L2 (126 MB)",
                   "parallelism": f"{world} independent batches (no data-path collective)"},
        "gpu_launches": launches,
        "cuda_graph": bool(args.graph),
        "arithmetic": "exact (bit-identical to the reference's map_1d)" if args.exact else
                      "fused (the remap walk: PPM face values once per face, target edges with the "
                      "reference's rounding; 1e-5 of peak per sweep)",
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                       "what": "device time of one batched acceleration step of all cells"},
        "plain_per_cell": plain,
        "status_cells_flagged": int((status != 0).sum()),
        "roofline": {"bound": "hbm", "kernel": "remap_kernel" if args.exact else "remap_walk_kernel", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": (REMAP_DRAM_BYTES_PER_BLOCK * src_blocks / remap_n) if remap_n else None,
                     "traffic_note": "bytes per launch, ncu capture of the 512-cell case scaled by source blocks",
                     "algorithmic_bytes": "8 B per source phase-space cell per sweep"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // max(e2e_steps, 1),
                "d2h_bytes_per_step": d2h // max(e2e_steps, 1), "steps": e2e_steps,
                "chunks": n_chunks,
                "path": "per chunk of cells: vlgpu_batch_upload_async + vlgpu_accelerate + "
                        "vlgpu_batch_download_begin / _end, pinned host buffers, chunks overlapped"},
        "clocks": clk.summary(),
    }
    if cpu is not None:
        rate, cores, sample, kind = cpu
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# full Vlasov step on a periodic grid
# ---------------------------------------------------------------------------
VLASOV_WORKLOAD = ("full Vlasov step, periodic sine-wave grid {nx}x{ny}x{nz}, dx=300 km, n=1e6(1+0.5 sin 2pi x/Lx), "
                   "T=1 MK, V=(400,0,0) km/s, B=(0,0,5 nT); translation z,x,y + R moments + acceleration (PPM) + "
                   "adjust with spatial neighbours + V moments; dt = 0.8 x the r-space CFL limit")
BYTES_PER_CELL_VLASOV = 60  # 24 acceleration + 24 translation + 4 adjust + 8 moments (unfused count)


def run_vlasov(args):
    world, rank, local, pg = dist_setup()
    from vlasiator_b200 import vlgpu
    vlgpu.load()
    import torch
    torch.cuda.set_device(local)
    from vlasiator_b200.projects import sinewave_grid
    dims = tuple(int(v) for v in args.grid)
    mesh = VelocityMesh()
    cells = sinewave_grid(dims, mesh)
    n = len(cells)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum([c.n_blocks for c in cells])
    total = int(offs[-1])
    gids = np.concatenate([c.gids for c in cells]).astype(np.uint32)
    data = np.concatenate([c.data for c in cells]).astype(np.float32)
    B = np.stack([c.B for c in cells])
    dx = 3e5
    cap = int(total * 1.5) + 262144
    batch = vlgpu.Batch(mesh, n, cap, device=local, exact=args.exact)
    batch.upload_packed(offs, gids, data)
    del data
    batch.set_grid(dims, dx)
    batch.compute_intersections(B, 1.0, 0)  # stages the fields for the time-step limits
    r_dt, v_dt = batch.max_dt(22.0)
    dt = 0.8 * float(r_dt.min())
    orders = map_orders(args.warmup + args.steps, args.seed)
    stream = torch.cuda.ExternalStream(batch.stream_handle(), device=local)
    batch.vlasov_step(B, dt, orders[0])
    for w in range(1, args.warmup):
        batch.vlasov_step_device(dt, orders[w])
    batch.sync()
    st0 = batch.stats()
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local) as clk:
        evs[0].record(stream)
        for s in range(args.steps):
            batch.vlasov_step_device(dt, orders[args.warmup + s])
            evs[s + 1].record(stream)
        evs[-1].synchronize()
    torch.cuda.synchronize()
    ms = evs[0].elapsed_time(evs[-1])
    step_ms = np.array([evs[q].elapsed_time(evs[q + 1]) for q in range(args.steps)])
    st1 = batch.stats()
    status = batch.status()
    batch.sync()
    updates = WID3 * (st1["step_blocks"] - st0["step_blocks"])
    launches = st1["launches"] - st0["launches"]
    ms_max = allreduce_max(pg, ms)
    value = allreduce_sum(pg, float(updates)) / (ms_max * 1e-3)
    peak, peak_kind = measured_peak()
    achieved = value * BYTES_PER_CELL_VLASOV / 1e9
    blocks_now = int(batch.block_counts().astype(np.uint64).sum())

    # end to end through the C ABI: host -> device copy of the grid's blocks
    # (pinned), one Vlasov step with the fields staged from the host, device
    # -> host copy of the result.  Translation couples all cells, so the grid
    # is one batch (no chunk pipeline).
    h_gids = torch.from_numpy(gids).pin_memory().numpy()
    h_data = torch.from_numpy(np.concatenate([c.data for c in cells]).astype(np.float32)).pin_memory().numpy()
    out_g = torch.empty(cap, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    out_d = torch.empty((cap, WID3), dtype=torch.float32).pin_memory().numpy()
    e_steps = max(1, min(args.steps, args.e2e_steps))
    t_e2e, h2d, d2h, e_upd = 0.0, 0, 0, 0
    for s in range(e_steps + 1):
        t0 = time.perf_counter()
        batch.upload_async(offs, h_gids, h_data)
        batch.vlasov_step(B, dt, orders[s % len(orders)])
        batch.download_begin()
        c_off, c_cnt, g_out, _ = batch.download_end(out_g, out_d)
        batch.sync()
        el = time.perf_counter() - t0
        if s > 0:  # the first pass warms the host paths
            t_e2e += el
            e_upd += WID3 * total
            h2d += offs.nbytes + h_gids.nbytes + h_data.nbytes
            d2h += c_off.nbytes + c_cnt.nbytes + len(g_out) * (4 + WID3 * 4)
    t_e2e = allreduce_max(pg, t_e2e)
    e2e_value = allreduce_sum(pg, float(e_upd)) / t_e2e
    batch.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_vlasov_rate((16, 16, 8))
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded sine-wave Maxwellian grid)",
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // e_steps,
                "d2h_bytes_per_step": d2h // e_steps, "steps": e_steps,
                "path": "vlgpu_batch_upload_async + vlgpu_vlasov_step + vlgpu_batch_download_begin / _end, "
                        "pinned host buffers"},
        "config": {"workload": VLASOV_WORKLOAD.format(nx=dims[0], ny=dims[1], nz=dims[2]), "cells_per_gpu": n,
                   "blocks_at_start": total, "blocks_at_end": blocks_now, "dt_s": dt,
                   "l2": "inputs larger than L2 (126 MB)",
                   "parallelism": f"{world} independent grids (no data-path collective)"},
        "gpu_launches": launches,
        "arithmetic": "exact (the reference's operation order)" if args.exact else
        "fused acceleration remap and fused translation (1e-5 of peak per sweep)",
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                       "what": "device time of one full Vlasov step of the grid"},
        "status_cells_flagged": int((status != 0).sum()),
        "roofline": {"bound": "hbm", "kernel": "whole step", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                     "algorithmic_bytes": "60 B per phase-space cell per step (24 acc + 24 trans + 4 adjust + 8 "
                                          "moments)"},
        "clocks": clk.summary(),
    }
    if cpu is not None:
        rate, cores, sample, kind = cpu
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# serving: a Poisson stream of independent VDF-advance requests
# ---------------------------------------------------------------------------
SERVE_WORKLOAD = ("serving: Poisson stream of {n} independent requests ({distinct} distinct drifting bi-Maxwellian "
                  "VDFs, T_par/T_perp U(0.5,3), blocks log-normal median 5k clipped 500..60k; own B 5-50 nT, "
                  "E=-VxB, dt=0.01 gyroperiod, steps U(1,{max_steps})); {budget} GB HBM budget, state device-resident")


def run_serve(args):
    world, rank, local, pg = dist_setup()
    from vlasiator_b200 import vlgpu
    vlgpu.load()
    import torch
    torch.cuda.set_device(local)
    from vlasiator_b200.projects import serving_requests
    from vlasiator_b200.serve import Server, run_plain, run_stream
    mesh = VelocityMesh()
    base = serving_requests(args.distinct, seed=args.seed + rank, mesh=mesh, max_steps=args.max_steps)
    rng = np.random.default_rng(args.seed + 17 + rank)
    reqs = []
    for k in range(args.requests):
        q = dict(base[k % len(base)])
        q["steps"] = int(rng.integers(1, args.max_steps + 1))
        reqs.append(q)
    work = sum(WID3 * q["cell"].n_blocks * q["steps"] for q in reqs)  # nominal, blocks at submission
    budget = int(args.budget_gb * 1e9)
    with Server(mesh, args.max_cells, budget, device=local) as srv:
        # warm-up: a few requests through the whole path
        run_stream(srv, reqs[: min(8, len(reqs))], rate_per_s=1e6)
        st0 = srv.stats()
        if pg is not None:
            pg.barrier()
        with ClockSampler(local) as clk:
            latency, wall, _ = run_stream(srv, reqs, rate_per_s=args.rate, seed=args.seed)
        st1 = srv.stats()
    updates = st1["cell_updates"] - st0["cell_updates"]
    wall_max = allreduce_max(pg, wall)
    value = allreduce_sum(pg, float(updates)) / wall_max
    # the plain per-request launch path on a bounded sample of the same requests
    plain = None
    if args.plain_requests > 0:
        sample = reqs[: args.plain_requests]
        times, _ = run_plain(mesh, sample)
        p_work = sum(WID3 * q["cell"].n_blocks * q["steps"] for q in sample)
        p_value = p_work / float(times.sum())
        plain = {"value": p_value, "unit": UNIT, "requests": len(sample), "seconds": float(times.sum()),
                 "latency_p50_ms": float(np.percentile(times, 50) * 1e3),
                 "served_over_plain": value / p_value,
                 "path": "one request at a time: vlgpu_batch_upload + vlgpu_accelerate_per_cell x steps + download"}
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": len(reqs), "warmup": 8,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded bi-Maxwellian requests)",
        "config": {"workload": SERVE_WORKLOAD.format(n=len(reqs), distinct=len(base), max_steps=args.max_steps,
                                                     budget=args.budget_gb),
                   "arrival_rate_per_s": args.rate, "max_cells": args.max_cells,
                   "nominal_cell_updates": work, "wall_s": wall_max},
        "latency_ms": {"p50": float(np.percentile(latency, 50) * 1e3),
                       "p99": float(np.percentile(latency, 99) * 1e3),
                       "what": "request arrival to its result on the host (wall clock)"},
        "plain_per_request": plain,
        "clocks": clk.summary(),
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=DEFAULT_SEED)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-chunks", type=int, default=32, help="accel e2e: batches the cells are split into")
    ap.add_argument("--cpu-sample", type=int, default=4096, help="cpu_baseline: cells timed (default all)")
    ap.add_argument("--ref-sample", type=int, default=0, help="reference arm: cells timed (0: all)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--exact", action="store_true", help="remap in the reference's exact operation order")
    ap.add_argument("--plain-steps", type=int, default=2, help="steps of the plain per-cell path (0: skip)")
    ap.add_argument("--graph", action="store_true", help="accel: replay CUDA graphs of two steps")
    ap.add_argument("--workload", default="accel", choices=["accel", "vlasov", "serve"],
                    help="accel: batched acceleration of independent cells; vlasov: full step of a periodic grid")
    ap.add_argument("--grid", type=int, nargs=3, default=[64, 64, 16], help="grid of the vlasov workload")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests in the stream")
    ap.add_argument("--distinct", type=int, default=100, help="serve: distinct generated VDFs")
    ap.add_argument("--max-steps", type=int, default=100, help="serve: steps per request U(1, max)")
    ap.add_argument("--rate", type=float, default=400.0, help="serve: mean arrival rate (requests/s)")
    ap.add_argument("--max-cells", type=int, default=4096, help="serve: cells of the server's batch")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serve: HBM budget (GB)")
    ap.add_argument("--plain-requests", type=int, default=8, help="serve: requests timed on the plain path")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "vlasov":
        return run_vlasov(args)
    if args.workload == "serve":
        return run_serve(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
