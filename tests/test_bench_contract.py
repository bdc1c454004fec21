"""The reference arm of bench.py keeps its line's contract whether the
reference build runs (a GPU box) or not (here: the FP64 C oracle on the host
cores stands in, with the reason in `note`): the product arm's metric, unit
and config, a positive value, and an e2e object with no host copies."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, timeout=900, cwd=REPO)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    sys.path.insert(0, REPO)
    import bench

    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == "MLUPS"
    assert line["config"] == bench.bench_config(1)
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    if line["cpu_baseline"]["kind"] == "port":
        assert line["note"]
