"""The serving engine (vlgpu_server_*): requests of different sizes and step
counts, admitted by block budget and between ticks, give results bit-identical
to the same request run alone and to the plain per-cell launch path with the
same dimension orders (step s uses order s mod 3)."""
import numpy as np
import pytest

from vlasiator_b200.mesh import CHARGE, MASS_PROTON, VelocityMesh
from vlasiator_b200.projects import random_drifting_cells

pytestmark = pytest.mark.gpu


def make_requests(n, seed):
    rng = np.random.default_rng(seed)
    cells = random_drifting_cells(n, seed=seed)
    out = []
    for c in cells:
        Tg = 2 * np.pi * MASS_PROTON / (CHARGE * np.linalg.norm(c.B))
        out.append({"cell": c, "B": c.B, "dt": 0.01 * Tg, "steps": int(rng.integers(1, 8))})
    return out


def same(a, b, what):
    np.testing.assert_array_equal(a[0], b[0], err_msg=what)
    assert np.array_equal(a[1], b[1]), f"{what}: max |diff| {np.abs(a[1] - b[1]).max()}"


def run_all(server, reqs, stagger=False):
    ids = []
    results = {}
    half = len(reqs) // 2 if stagger else len(reqs)
    for q in reqs[:half]:
        ids.append(server.submit(q["cell"].gids, q["cell"].data, q["B"], q["dt"], q["steps"]))
    ticks = 0
    while len(results) < len(reqs):
        if stagger and ticks == 4:
            for q in reqs[half:]:
                ids.append(server.submit(q["cell"].gids, q["cell"].data, q["B"], q["dt"], q["steps"]))
        server.tick()
        ticks += 1
        for k, rid in enumerate(ids):
            if k not in results:
                r = server.result(rid)
                if r is not None:
                    results[k] = r
        assert ticks < 500
    return [results[k] for k in range(len(reqs))]


def test_results_independent_of_the_mix(mesh=VelocityMesh()):
    from vlasiator_b200.serve import Server, run_plain
    reqs = make_requests(10, seed=3)
    with Server(mesh, 16, 2 << 30) as s:
        mixed = run_all(s, reqs, stagger=True)
        st = s.stats()
        assert st["completed"] == len(reqs)
    for k, q in enumerate(reqs):
        with Server(mesh, 2, 1 << 30) as s:
            alone, = run_all(s, [q])
        same(mixed[k], alone, f"request {k}: mix vs alone")
        assert mixed[k][2] == 0
    _, plain = run_plain(mesh, reqs)
    for k in range(len(reqs)):
        same(mixed[k][:2], plain[k][:2], f"request {k}: server vs plain per-cell path")


def test_budget_admission_queues_requests(mesh=VelocityMesh()):
    """A block budget far below the requests' total: they wait and still
    finish with the same results."""
    from vlasiator_b200.serve import Server
    reqs = make_requests(8, seed=9)
    biggest = max(q["cell"].n_blocks for q in reqs)
    budget = int(600 * biggest / 0.6 * 1.2)  # room for about one largest request at a time
    with Server(mesh, 8, max(budget, 600 * 4096)) as s:
        queued = run_all(s, reqs)
    with Server(mesh, 8, 2 << 30) as s:
        free = run_all(s, reqs)
    for k in range(len(reqs)):
        same(queued[k], free[k], f"request {k}")
