"""The bench's reference arm on the CPU (the multithreaded host port of the
reference's table semantics): one JSON line with the contract's keys, the
requested warm-up and timed steps, and its own cpu_baseline and e2e objects."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 1
    assert d["steps"] == 2 and d["warmup"] == 3 and d["higher_is_better"] is True
    assert d["metric"] == "Mops/s insert+query at 0.9 load" and d["unit"] == "Mops/s" and d["value"] > 0
    assert d["ms_per_step"] > 0 and d["scaling"] == "weak" and d["vs_baseline"] is None
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert d["config"]["slots"] == 1 << 26 and d["config"]["inserts"] == int(0.9 * (1 << 26))
