"""The block-index decomposition the kernels use (block_xyz,
vlasiator_b200/csrc/vlgpu_common.cuh): floor(n / d) as the high word of
n * (floor(2^32 / d) + 1), enabled only when every n it sees is below
2^32 / d.  Checked exhaustively, on the CPU, for the velocity meshes of the
tests and benchmarks and for meshes at the edge of the enabling condition."""
import numpy as np
import pytest


def reciprocals(L0, L1, L2):
    """set_block_reciprocals: (m0, m1), or (0, 0) when the kernels divide."""
    two32 = 1 << 32
    if L0 < 2 or L1 < 2 or L0 * L1 * L2 * L0 >= two32 or L1 * L2 * L1 >= two32:
        return 0, 0
    return two32 // L0 + 1, two32 // L1 + 1


def umulhi(a, m):
    return (a.astype(np.uint64) * np.uint64(m)) >> np.uint64(32)


@pytest.mark.parametrize("dims", [(67, 67, 67), (8, 8, 8), (100, 37, 3), (2, 2, 2), (200, 200, 200),
                                  (1000, 60, 60)])
def test_multiply_high_division_is_exact(dims):
    L0, L1, L2 = dims
    m0, m1 = reciprocals(L0, L1, L2)
    if m0 == 0:
        # the kernels divide; the condition must really be violated or trivial
        assert L0 < 2 or L1 < 2 or L0 * L1 * L2 * L0 >= 1 << 32 or L1 * L2 * L1 >= 1 << 32
        return
    g = np.arange(L0 * L1 * L2, dtype=np.uint64)
    q0 = umulhi(g, m0)
    np.testing.assert_array_equal(q0, g // L0)
    z = umulhi(q0, m1)
    np.testing.assert_array_equal(z, q0 // L1)
    x = g - q0 * np.uint64(L0)
    y = q0 - z * np.uint64(L1)
    np.testing.assert_array_equal(x, g % L0)
    np.testing.assert_array_equal(y, (g // L0) % L1)
    np.testing.assert_array_equal(z, g // (L0 * L1))


def test_reciprocals_disabled_past_the_bound():
    assert reciprocals(1000, 1000, 1000) == (0, 0)  # 1e9 * 1000 >= 2^32
    assert reciprocals(1, 67, 67) == (0, 0)
    assert reciprocals(67, 67, 67) != (0, 0)
