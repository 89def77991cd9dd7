"""The bench's reference arm runs on the host cores and prints the contract's JSON line (CPU)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*argv, env=None, timeout=600):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *argv], cwd=ROOT, env=e,
                          capture_output=True, text=True, timeout=timeout)


def test_reference_arm_prints_one_contract_line():
    r = _bench("--impl", "reference", "--steps", "2", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2 and d["n_gpus"] == 1
    assert d["metric"].startswith("sim steps/s")
    assert d["config"]["workload"].startswith("256 independent tet soft bodies")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    # a size-stratified sample of 16 bodies, scaled to the batch by its work share
    assert "16 of 256" in cb["sample"] and "work share" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work():
    r = _bench("--impl", "reference", "--steps", "2", "--warmup", "3", env={"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_fewer_than_three_warmup_steps_are_refused():
    r = _bench("--impl", "reference", "--steps", "2", "--warmup", "2", timeout=120)
    assert r.returncode == 2
    assert "--warmup must be >= 3" in r.stderr


def test_reference_arm_with_the_cpu_backend_semantics():
    """--semantics cpu: the reference arm times the oracle's restatement of the CPU backend
    (damped system, exact FP64 Cholesky, serial Gauss-Seidel contact) and says so."""
    r = _bench("--impl", "reference", "--config", "cloth", "--semantics", "cpu", "--tol", "0", "--steps", "3",
               "--warmup", "3", timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads([l for l in r.stdout.splitlines() if l.strip()][0])
    assert d["impl"] == "reference" and d["value"] > 0
    assert "CPU backend's solver" in d["metric"] and "fixed 20 ADMM iterations" in d["metric"]
    assert "Cholesky" in d["cpu_baseline"]["sample"]
