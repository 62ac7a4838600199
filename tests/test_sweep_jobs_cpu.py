"""The sweep runner's handling of the reference's job list (compose_config.py
format) and of run_sim.py's grids and file names; no GPU needed."""
from __future__ import annotations

import numpy as np
import pytest

from henon_map_cpp_b200 import sweep


def test_read_jobs_of_a_composed_list(tmp_path):
    path = tmp_path / "all_jobs.txt"
    # written the way compose_config.py writes it
    jobs = [((0.168, 0.201, 0.75), 0.0, 0.25), ((0.31, 0.32, 0.25), 64.0, 1.0)]
    with open(path, "w") as f:
        for (ox, oy, rmax), eps, mu in jobs:
            f.write(f"{ox} {oy} {eps} {mu} {rmax}\n")
        f.write("\n")
    got = sweep.read_jobs(path)
    assert got == [dict(omega_x=0.168, omega_y=0.201, epsilon=0.0, mu=0.25, max_radius=0.75),
                   dict(omega_x=0.31, omega_y=0.32, epsilon=64.0, mu=1.0, max_radius=0.25)]
    bad = tmp_path / "bad.txt"
    bad.write_text("0.1 0.2 0.3\n")
    with pytest.raises(ValueError):
        sweep.read_jobs(bad)


def test_grid_and_file_name_follow_run_sim():
    x, px, y, py = sweep.job_grid(0.75, 5)
    v = np.linspace(0, 0.75, 5)
    xx, yy = np.meshgrid(v, v)
    np.testing.assert_array_equal(x, xx.flatten())
    np.testing.assert_array_equal(y, yy.flatten())
    assert not px.any() and not py.any()
    job = dict(omega_x=0.168, omega_y=0.201, epsilon=16.0, mu=0.25, max_radius=0.75)
    assert sweep.job_file_name(job) == "stability_henon_0d168_0d201_16d0_0d25_0d75"
