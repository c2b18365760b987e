"""The reference's polar solves/min is estimated, not run: each point's
iterations x cells at the reference's measured per-core rate, scheduled
longest first over the host cores. Checked here on hand-made numbers."""
import pytest

import bench


def test_one_point_per_core_takes_the_longest_point():
    points = [{"iterations": 100, "cells": 1000}, {"iterations": 300, "cells": 1000}]
    est = bench.reference_polar_estimate(points, {"value": 2.0e5, "cores": 2})
    # 1e5 cell-iterations/s per core: the longer point takes 3 s
    assert est["wall_s"] == pytest.approx(3.0)
    assert est["solves_per_min"] == pytest.approx(60.0 * 2 / 3.0)
    assert est["cores"] == 2
    assert "estimate" in est["basis"]


def test_points_are_packed_longest_first():
    # loads 4, 3, 3, 2 on two cores: longest first gives 4+2 and 3+3, so 6 s
    points = [{"iterations": n, "cells": 1} for n in (4, 3, 3, 2)]
    est = bench.reference_polar_estimate(points, {"value": 2.0, "cores": 2})
    assert est["wall_s"] == pytest.approx(6.0)
    assert est["solves_per_min"] == pytest.approx(40.0)
