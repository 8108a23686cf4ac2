"""bench.py's reference arm on the CPU: one JSON line with the GPU arm's
metric, unit and config keys, the CPU baseline it measured (labelled as an
extrapolation of a bounded sample), a zero-byte e2e, and no use of the CUDA
library (the arm reads the configuration and the phantom generator by path).
"""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

_RUN = r"""
import contextlib, io, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"]
out = io.StringIO()
with contextlib.redirect_stdout(out):
    try:
        runpy.run_path("bench.py", run_name="__main__")
    except SystemExit as e:
        assert not e.code, e.code
maps = open("/proc/self/maps").read()
print(out.getvalue().strip().splitlines()[-1])
print(int("libesb" in maps), int(any(m == "artiatomi_b200" or m.startswith("artiatomi_b200.") for m in sys.modules)))
"""


def test_reference_arm_line_and_isolation():
    r = subprocess.run([sys.executable, "-c", _RUN], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line, flags = r.stdout.strip().splitlines()[-2:]
    d = json.loads(line)
    assert flags.split() == ["0", "0"], "the reference arm loaded the CUDA library or the package"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["unit"] == "voxel-updates/s" and d["steps"] == 1
    assert d["extrapolated"] is True and d["cpu_baseline"]["kind"] == "port"
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["sample_s"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the GPU arm's config keys for the same workload
    sys.path.insert(0, str(ROOT))
    import bench

    params = bench._load_by_path("esb_configs", "artiatomi_b200/configs.py").CONFIGS["c2_sart_ctf"]
    assert d["config"] == bench.workload_config("c2_sart_ctf", params, 1)
