"""CPU tests of bench.py's reference arm: it times the CPU restatement of the
reference's LBGK on the porous channel, built without the CUDA library."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_loads_only_the_oracle():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--size", "48,24,24",
                        "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    line = json.loads([s for s in r.stdout.splitlines() if s.startswith("{")][-1])
    assert line["impl"] == "reference" and line["unit"] == "MLUPS" and line["value"] > 0
    assert line["steps"] == 2 and line["warmup"] == 1
    assert line["repo_libraries_loaded"] == ["oracle/liboracle.so"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    env = {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}
    import os
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--size", "48,24,24",
                        "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=600,
                       env={**os.environ, **env})
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_rank0_names_the_slab_job():
    """Under a launcher with N ranks, rank 0 samples one slab of the N-slab
    job our arm runs and names that job in its config."""
    import os
    env = {"RANK": "0", "WORLD_SIZE": "2", "LOCAL_RANK": "0"}
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--size",
                        "48,24,24", "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=600,
                       env={**os.environ, **env})
    assert r.returncode == 0, r.stderr
    line = json.loads([s for s in r.stdout.splitlines() if s.startswith("{")][-1])
    assert line["config"]["workload"] == "porous_channel_d3q19_96x24x24"
    assert line["config"]["cells"] == 2 * 48 * 24 * 24
    assert "slab" in line["cpu_baseline"]["sample"] and line["n_gpus"] == 2
