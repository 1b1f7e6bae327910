"""bench.py's host-side arithmetic: the V-cycle's algorithmic bytes
(the per-level formula N w [8 (nu1 + nu2) + 6 + rho + 2 + rho + 3] plus 11
FP64 words per finest cell), checked against a hand count on the bench grid."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402
import mgpoisson2d_b200.api as M  # noqa: E402
from mgpoisson2d_b200.types import Box  # noqa: E402


def _by_hand(sides, bottom, mixed):
    per = 8 * 16 + 6 + 0.25 + 2 + 0.25 + 3   # nu = 8/8, full coarsening
    total = 11 * 8 * sides[0] ** 2
    for d in range(bottom):
        n = sides[d] ** 2
        w = 4 if (mixed and n > 1024) else 8
        total += n * w * per
    return total


def test_vcycle_bytes_bench_grid():
    v = Box.of_size(1024, 1024)
    sides = [1024 >> d for d in range(9)]   # 1024 .. 4: levels 0-8
    # exact bottom on the first level of at most 64 cells (8 x 8, level 7)
    assert bench.vcycle_bytes(M, v, True, True) == _by_hand(sides, 7, True)
    # the reference bottom (4 x 4, level 8) in plain FP64
    assert bench.vcycle_bytes(M, v, False, False) == _by_hand(sides, 8, False)
    # exact bottom on the first level of at most 1024 cells (32 x 32, level
    # 5), plus one read of its 1024 x 1024 inverse and of r and e
    assert bench.vcycle_bytes(M, v, True, True, large=True) == _by_hand(sides, 5, True) + 8 * 1024 * 1026


def test_vcycle_bytes_scales_with_word_size():
    v = Box.of_size(512, 512)
    b64 = bench.vcycle_bytes(M, v, False, False)
    b32 = bench.vcycle_bytes(M, v, True, False)
    assert b32 < b64 < 2 * b32 + 11 * 8 * 512 * 512
