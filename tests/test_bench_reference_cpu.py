"""The reference arm of bench.py (`--impl reference`) on the CPU: the C
restatement of aca2 + hmat_matvec! timed on a bounded band of rows, printed as
the same JSON line as the GPU arm with impl = "reference"; ranks other than 0
exit without work."""
import json
import os
import subprocess
import sys

from conftest import ROOT

ARGS = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "65536",
        "--cpu-rows", "512", "--steps", "1", "--warmup", "0"]


def test_reference_line_contract():
    out = subprocess.run(ARGS, cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["n"] == 65536 and d["config"]["workload"]


def test_reference_other_ranks_silent():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    out = subprocess.run(ARGS, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0
    assert not [l for l in out.stdout.splitlines() if l.startswith("{")]


def test_oracle_lu_sample_contract():
    # the CPU H-LU sample set beside the GPU's in the bench's LU leg
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "hmatrix.jl_b200"))
    import bench
    d = bench.oracle_lu_sample(2048)
    assert d["n"] == 2048 and d["kind"] == "port" and d["cores"] >= 1
    assert d["lu_s"] > 0 and d["total_s"] >= d["lu_s"] and d["relres"] < 1e-8


def test_oracle_batch_sample_contract():
    # the CPU sample of the batched configuration set beside the GPU's
    sys.path.insert(0, ROOT)
    import bench
    rows, cores = bench.oracle_batch_sample(256, budget_s=0.2, nmax=2048)
    assert cores >= 1 and len(rows) >= 1
    probs = bench.batched_problems(256)
    for r in rows:
        assert r["n"] == len(probs[r["problem"]][0]) <= 2048
        assert r["s"] > 0 and r["relres"] < 1e-8
    # problem order, and the budget ends the sample after the problem that crosses it
    assert [r["problem"] for r in rows] == sorted(r["problem"] for r in rows)
    assert sum(r["s"] for r in rows[:-1]) < 0.2
