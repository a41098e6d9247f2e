"""The host arithmetic behind bench.py's baselines and work counts (no GPU).

The plain per-instance baseline's sample covers every (incidence angle, order
count) stratum of the sweep; the CPU baseline's representatives and its
scaling to the whole sweep; the field workload's wave-evaluation count
against an explicit count over the grid points.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_plain_sample_covers_every_stratum():
    inst = bench.sweep_instances()
    strata = bench.plain_strata(inst)
    assert set(strata) == {(a, m) for a in bench.ANGLES for m in bench.ORDERS}
    assert all(len(v) == bench.PLAIN_PER_STRATUM for v in strata.values())
    for (a, m), idx in strata.items():
        assert all(inst[i].angle_deg == a and inst[i].orders == m for i in idx)


def test_cpu_representatives_and_scaling():
    inst = bench.sweep_instances()
    reps = bench.representatives(inst)
    assert [r.orders for r in reps] == list(bench.ORDERS)
    # the scaled estimate is the per-instance sum of t_rep (L_i + f) / (L_rep + f)
    per = {m: (0.5 * (j + 1), 2) for j, m in enumerate(bench.ORDERS)}
    f = bench.FIXED_LAYERS
    want = sum(per[it.orders][0] * (it.maps.shape[0] + f) / (2 + f) for it in inst)
    assert abs(bench.cpu_sweep_estimate(inst, per) - want) <= 1e-12 * want


def test_wave_evals_count_matches_the_points_regions():
    class Table:
        z_layers = np.array([-1.0, 0.5, 2.0])
        begin = np.array([0, 10, 25, 40])
        end = np.array([7, 21, 33, 52])
    grid = {"origin": (0.0, 0.0, -3.0), "step": (0.1, 0.2, 0.37), "counts": (4, 3, 17)}
    pts = bench.grid_points(grid)
    assert pts.shape == (4 * 3 * 17, 3)
    count = 0
    for z in pts[:, 2]:
        l = int(np.sum(z >= Table.z_layers - 0.001))
        count += int(Table.end[l] - Table.begin[l])
    assert bench.wave_evals(Table, grid) == count
