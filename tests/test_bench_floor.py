"""The shared-memory wavefront floor that bench.py reports beside the roofline
of the FP64 alpha-beta kernel (CPU only: plain arithmetic on table sizes)."""
import numpy as np

import bench


def test_default_group_follows_the_shared_memory_budget():
    # 144M workload: 12,000 beta strings, norb 36 (666 pairs): a row of C
    # (96 KB) and 16 integral rows fit in the 227 KB opt-in limit
    assert bench.ab_default_group(12000, 666, 232448) == 16
    # 400M workload: 20,000 strings, norb 48 (1,176 pairs): only groups of 4
    assert bench.ab_default_group(20000, 1176, 232448) == 4
    # nothing fits: no floor
    assert bench.ab_default_group(40000, 2080, 232448) is None


def test_floor_counts_ctas_slices_and_wavefronts():
    # 3 alpha strings with 16, 17 and 0 singles: 1 + 2 + 0 CTAs of 16
    # 40 beta strings: a slice of 32 (longest list 5) and a padded one of 8 (longest 7)
    st = {("singles", 0): np.array([16, 17, 0]),
          ("singles", 1): np.array([5] * 32 + [7] * 8)}
    f = bench.ab_smem_floor(st, 16, sm_count=2, sm_mhz=1000.0)
    assert f["ctas"] == 3
    assert f["warp_steps"] == 3 * (5 + 7)
    assert f["wavefronts_per_step"] == 4 * 8 + 2
    # cycles / SMs / (MHz * 1e3) = ms
    assert abs(f["floor_ms"] - 3 * 12 * 34 / 2 / 1e6) < 1e-15
