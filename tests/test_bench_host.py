"""bench.py's reference arm (the CPU port of the operator, no GPU) prints one
well-formed JSON line with a finite positive value and the keys the
measurement contract asks for."""
import json
import math
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("workload", ["poly3d"])
def test_reference_arm_prints_contract_line(workload):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1",
                        "--workload", workload], cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "cpu_baseline", "e2e", "config", "dtype"):
        assert k in line, k
    assert math.isfinite(line["value"]) and line["value"] > 0
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["unit"] == "solves/s" and line["higher_is_better"] is True


def test_sixteen_system_workload_is_well_formed():
    """The uneven 16-system workload: sizes within [1k, 64k] summing to about
    250k, no two spheres overlapping (periodic minimum image), every box
    edge above twice the real-space cutoff of tol 1e-6, xi 0.5."""
    sys.path.insert(0, ROOT)
    import numpy as np
    from scipy.spatial import cKDTree

    import bench

    syst = bench.c5_systems()
    n = [s.num_particles for s in syst]
    assert len(syst) == 16 and min(n) >= 1000 and max(n) <= 64000
    assert abs(sum(n) - 250_000) < 2_000
    rc = math.sqrt(-math.log(bench.TOL)) / bench.XI * bench.RADIUS   # nm
    for s in syst:
        p = np.asarray(s.positions)
        box = np.asarray(s.box)
        assert np.all(box > 2 * rc)
        q = np.mod(p, box)
        d, _ = cKDTree(q, boxsize=box).query(q, k=2)
        assert d[:, 1].min() >= 2 * bench.RADIUS - 1e-9
        assert s.quadrupoles is True and s.options == {"batch_all": True, "refine": True}
