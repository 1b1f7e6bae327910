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


def test_solve_fraction():
    # a sample of 4 V-cycles of 1 s each after a 0.5 s set-up, in a solve of 100 V-cycles
    f = bench.solve_fraction(4.5, 4, 0.5, 100)
    assert abs(f - 4.5 / 100.5) < 1e-12
    # a whole solve is one solve
    assert abs(bench.solve_fraction(0.5 + 100 * 0.2, 100, 0.5, 100) - 1.0) < 1e-12


def test_reference_arm_is_measured_not_projected():
    """--impl reference on a small grid: one JSON line whose ms_per_step times
    the steps fits inside the run's own wall time (the steps' time is measured,
    not a projection of a whole solve), with the solve fractions it counted."""
    import json
    import subprocess
    import time
    t0 = time.time()
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "64",
                          "--steps", "2", "--warmup", "1", "--cpu-vcycles", "2"],
                         capture_output=True, text=True, check=True, timeout=300).stdout
    wall = time.time() - t0
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "solves/s"
    assert line["ms_per_step"] * line["steps"] / 1e3 <= wall
    assert abs(line["value"] - line["solves_per_step"] / (line["ms_per_step"] / 1e3)) <= 1e-9 * line["value"]
    assert line["cpu_baseline"]["cores"] >= 1 and line["e2e"]["h2d_bytes_per_step"] == 0
