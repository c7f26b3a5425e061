"""bench.py's reference arm (the reference's CPU path on a bounded sample of
the workload), run here on the CPU: one JSON line with the contract's keys;
under several ranks only rank 0 runs and prints."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *map(str, args)], capture_output=True,
                       text=True, timeout=600, env=e, cwd=ROOT)
    return r.returncode, r.stdout, r.stderr


def test_reference_arm_prints_one_contract_line():
    rc, out, err = run_bench("--impl", "reference", "--steps", 2, "--warmup", 1, "--cpu-sample-scale", 10)
    assert rc == 0, err
    lines = [l for l in out.splitlines() if l.strip()]
    assert len(lines) == 1
    j = json.loads(lines[0])
    assert j["impl"] == "reference"
    assert j["metric"] == "triangles peeled/sec" and j["unit"] == "triangles/s"
    assert j["higher_is_better"] is True and j["scaling"] == "weak"
    assert j["steps"] == 2 and j["warmup"] == 1 and j["n_gpus"] == 1
    assert j["value"] > 0 and j["ms_per_step"] > 0
    assert j["vs_baseline"] is None and j["data"] == "synthetic"
    assert j["config"]["workload"].startswith("R-MAT scale 20 ef 16")
    cb = j["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    assert cb["value"] == j["value"] and cb["unit"] == j["unit"]
    assert "R-MAT scale 10" in cb["sample"]
    assert j["e2e"] == {"value": j["value"], "unit": j["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_zero_only():
    rc, out, err = run_bench("--impl", "reference", "--gpus", 2, "--steps", 1, "--warmup", 0,
                             "--cpu-sample-scale", 10, env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert rc == 0, err
    assert out.strip() == ""


def test_reference_arm_sample_generator_equals_the_library_generator(n34):
    """The reference arm generates its sample in numpy (no library of this
    project in that process); it must be the library's R-MAT edge for edge."""
    sys.path.insert(0, ROOT)
    import bench
    for scale, ef, seed in ((6, 8, 1), (10, 16, 2), (12, 16, 5)):
        s, d = n34.gen_rmat(scale, ef, seed)
        bs, bd = bench.rmat_edges_numpy(scale, ef, seed)
        assert np.array_equal(s, bs) and np.array_equal(d, bd), (scale, ef, seed)


def test_reference_arm_sample_file_equals_the_library_writer(n34, tmp_path):
    sys.path.insert(0, ROOT)
    import bench
    s, d = n34.gen_rmat(9, 8, 3)
    n34.write_edges(s, d, str(tmp_path / "lib.edges"))
    bench.write_edges_text(s, d, str(tmp_path / "np.edges"))
    assert (tmp_path / "lib.edges").read_bytes() == (tmp_path / "np.edges").read_bytes()


def test_reference_arm_loads_no_library_of_this_project():
    """The reference arm's process maps none of this project's shared
    libraries (only the reference's own program runs, as a child)."""
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', "
            "'--cpu-sample-scale', '9']\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\nexcept SystemExit:\n    pass\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libnucleus34' not in maps and 'liboracle' not in maps, 'a project library is mapped'\n"
            "assert 'nucleus34' not in sys.modules\nprint('clean')\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().endswith("clean")
