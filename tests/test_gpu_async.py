"""The asynchronous upload and two-phase download (vlgpu_batch_upload_async,
vlgpu_batch_download_begin / _end) give the same blocks as the blocking
calls, over several steps and with the batch's work overlapping another
batch's."""
import numpy as np
import pytest

from vlasiator_b200.projects import random_drifting_cells

pytestmark = pytest.mark.gpu


def _packed(cells):
    offs = np.zeros(len(cells) + 1, np.uint64)
    offs[1:] = np.cumsum([c.n_blocks for c in cells])
    return offs, np.concatenate([c.gids for c in cells]), np.concatenate([c.data for c in cells])


def test_async_upload_and_download_match_blocking(mesh):
    from vlasiator_b200 import vlgpu
    vlgpu.load()
    import torch
    cells = random_drifting_cells(24, seed=71, mesh=mesh)
    offs, gids, data = _packed(cells)
    B = np.stack([c.B for c in cells])
    dt = np.full(len(cells), 0.05)
    cap = 2 * int(offs[-1]) + 65536
    h_gids = torch.from_numpy(gids).pin_memory().numpy()
    h_data = torch.from_numpy(data).pin_memory().numpy()
    with vlgpu.Batch(mesh, len(cells), cap) as ref, vlgpu.Batch(mesh, len(cells), cap) as a, \
            vlgpu.Batch(mesh, len(cells), cap) as other:
        other.upload_packed(offs, gids, data)
        for step in range(3):
            ref.upload_packed(offs, gids, data)
            ref.accelerate(B, dt, step)
            r_off, r_cnt, r_g, r_d = ref.download_raw()
            other.accelerate(B, dt, step)  # other work in flight on another stream
            a.upload_async(offs, h_gids, h_data)
            a.accelerate(B, dt, step)
            a.download_begin()
            out_g = np.zeros(cap, np.uint32)
            out_d = np.zeros((cap, 64), np.float32)
            off, cnt, g, d = a.download_end(out_g, out_d)
            a.sync()
            # cell regions are placed by a device-side allocator, so the
            # offsets may differ; counts and contents may not
            np.testing.assert_array_equal(cnt, r_cnt)
            for c in range(len(cells)):
                s1 = slice(int(r_off[c]), int(r_off[c] + r_cnt[c]))
                s2 = slice(int(off[c]), int(off[c] + cnt[c]))
                o1, o2 = np.argsort(r_g[s1]), np.argsort(g[s2])
                np.testing.assert_array_equal(r_g[s1][o1], g[s2][o2])
                assert np.array_equal(r_d[s1][o1], d[s2][o2])
        assert not a.status().any()
