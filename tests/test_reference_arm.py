"""The reference arm's CPU baseline (CPU): the FP64 oracle in several spawned processes, one simulation
each, with the work balanced so that every process runs until the end of the timed region."""
import numpy as np

import bench


def test_oracle_parallel_rate_balances_processes():
    rate, wall, cells = bench.oracle_parallel_rate(np.array([12, 16]), np.array([100.0, 400.0]), [0.04, 0.03], 1, 2)
    assert rate > 0 and wall > 0
    # the 16^2 cavity takes one step, the 12^2 one round(256 / 144) = 2 steps
    assert cells == 16 * 16 + 2 * 12 * 12
    assert abs(rate - cells / wall) <= 1e-9 * rate
