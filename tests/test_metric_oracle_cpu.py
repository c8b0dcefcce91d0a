"""The numpy restatement of the reference's metric (oracle/metric_oracle.py),
which builds the workloads' geometry for the CPU baseline and the reference
arm of bench.py without loading the product library, against the library's
ostc_metric_from_grid (itself pinned to the reference's compute_jac_metric
by tests/test_metric_cpu.py)."""
import sys
from pathlib import Path

import numpy as np

import ostc

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import metric_oracle  # noqa: E402


def test_numpy_metric_restatement_matches_library_helper():
    """oracle/metric_oracle.py (the geometry of the CPU baseline, which must
    not load the product library) is bit-identical to ostc_metric_from_grid
    on warped 3-D, 2-D and three-ghost grids"""
    for mx, my, mz, g in ((20, 16, 10, 2), (24, 20, 1, 2), (16, 12, 8, 3)):
        x, y, z = ostc.grid_coordinates(mx, my, mz, g + 1, 1e-3, warp=0.02)
        a = ostc.HostBlock.allocate(mx, my, mz, g, 5, 0)
        ostc.fill_metric(a, x, y, z)
        jac, met = metric_oracle.metric(mx, my, mz, g, x, y, z)
        assert np.array_equal(a.arrays["jac"], jac)
        assert np.array_equal(a.arrays["metric"]["m"], met["m"])
        assert np.array_equal(a.arrays["metric"]["bias"], met["bias"])
