"""The bench's reference arm (the reference's own CPU H.x on the host cores)
keeps its JSON contract: one line from rank 0 with the headline metric, the
unit, "impl": "reference", a cpu_baseline describing the run and an e2e
block with zero host-device bytes; other ranks print nothing and exit 0.
Runs on the CPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run(env_extra):
    env = dict(os.environ, OMP_NUM_THREADS="4", **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3",
                           "--ref-n", "22"],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)


def test_reference_arm_line():
    p = run({})
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"].startswith("Hx effective HBM GB/s") and line["unit"] == "GB/s"
    assert line["value"] > 0 and line["higher_is_better"] is True and line["steps"] == 1 and line["warmup"] == 3
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] == 4 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "heisenberg_chain_N28_Sz0_Hx"
    assert line["config"]["sample_N"] == 22 and line["config"]["same_config"] is False


def test_reference_arm_other_ranks_are_silent():
    p = run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def test_reference_sizes_follow_host_memory(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setattr(bench, "mem_available_gb", lambda: 2000.0)
    assert bench.reference_sizes() == ([28], None)
    monkeypatch.setattr(bench, "mem_available_gb", lambda: 100.0)
    sizes, why = bench.reference_sizes()
    assert sizes == [26, 24] and why["N"] == 28 and why["mem_available_gb"] == 100.0
    monkeypatch.setattr(bench, "mem_available_gb", lambda: 10.0)
    assert bench.reference_sizes()[0] == [24]
    assert bench.reference_sizes(force_n=20) == ([20], None)
