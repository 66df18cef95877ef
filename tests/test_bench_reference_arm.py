"""bench.py's reference arm on CPU: the oracle's restatement of the
reference FMM timed on the host, its JSON line in the contract's shape, and
no engine code loaded (the arm imports the oracle only)."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line_and_oracle_only():
    code = (
        "import runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--ref-sample', '8192', '--steps', '2', '--warmup', '1',"
        " '--ref-budget-s', '1']\n"
        "runpy.run_path('bench.py', run_name='__main__')\n"
        "print('ENGINE_LOADED', 'fmms_b200' in sys.modules)\n"
    )
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "bodies/s" and d["value"] > 0
    assert 1 <= d["steps"] <= 2 and d["steps_requested"] == 2
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert "ENGINE_LOADED False" in out.stdout
