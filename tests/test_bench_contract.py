"""The benchmark's reference arm (the oracle port on the host cores) keeps
the line format the harness parses: one JSON line from rank 0, nothing from
the other ranks; it loads no part of the engine; and its config object is
the one the engine arm prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                          capture_output=True, text=True, cwd=ROOT, env=env, timeout=900)


def test_reference_arm_line():
    r = _run({})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert "workload" in d["config"]
    # the host stripes count every embedding of the configuration's queries
    assert set(d["counts"]) == {"triangle", "4-clique+pendant"} and min(d["counts"].values()) > 0
    sys.path.insert(0, ROOT)
    import bench
    assert d["config"] == json.loads(json.dumps(bench.shared_config(d["config"]["n"], d["config"]["arcs"],
                                                                    d["config"]["max_degree"])))


def test_reference_arm_loads_no_engine_code():
    """Run the arm's setup in-process and list the shared objects it mapped."""
    code = (
        "import sys, os; sys.path.insert(0, os.getcwd()); import bench; "
        "rg = bench.oracle_ranked_graph(); "
        "import sys as s2; print('MODULES', sorted(m for m in s2.modules if m.startswith('cuts_b200'))); "
        "print('MAPS', [l.split()[-1] for l in open('/proc/self/maps') if l.rstrip().endswith('.so') "
        "and 'libcuts_b200' in l])")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "MODULES []" in r.stdout and "MAPS []" in r.stdout, r.stdout


def test_reference_arm_other_ranks_are_silent():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0
    assert not [x for x in r.stdout.splitlines() if x.strip().startswith("{")]
