"""bench.py's reference arm on CPU: `--impl reference` times the reference's own CPU backend
(oracle/_ref, render_frame_tiled with its Release flags) and prints one JSON line with the keys
the benchmark contract asks for. Under torchrun, only rank 0 runs and prints it; the other ranks
exit 0 without work. The GPU arm needs a B200 and is run there."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SMALL = ["--level", "3", "--width", "128", "--height", "72", "--steps", "2", "--warmup", "3"]
KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e")


def _run(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference"] + args, cwd=ROOT, env=e,
                          capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_one_contract_line(ref):
    if not ref.available("fast"):
        pytest.skip("oracle/_ref fast flavour not built")
    p = _run(SMALL)
    assert p.returncode == 0, p.stderr
    lines = [l for l in p.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, p.stdout                      # the reference's printf stays off stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    for k in KEYS:
        assert k in line, k
    assert line["value"] > 0 and line["unit"] == "Mrays/s" and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 3 and line["n_gpus"] == 1
    assert line["config"]["workload"].startswith("config2: displaced icosphere L3 (")
    assert "128x72" in line["config"]["workload"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"] and cb["cores"] >= 1 and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    p = _run(SMALL, {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0 and p.stdout.strip() == ""


def test_reference_arm_loads_no_library_of_this_package(ref):
    """The reference arm times the reference alone: no library built from this package's sources
    (xenon_b200/lib) is loaded into its process, and its `config` is the GPU arm's."""
    if not ref.available("fast"):
        pytest.skip("oracle/_ref fast flavour not built")
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference'] + " + repr(SMALL) + "\n"
            "import bench\n"
            "from xenon_b200 import scenes\n"
            "a = bench.parse()\n"
            "with bench.quiet_stdout():\n"
            "    line = bench.reference_line(a)\n"
            "desc = scenes.icosphere_scene(level=a.level, width=a.width, height=a.height)\n"
            "maps = open('/proc/self/maps').read()\n"
            "print(json.dumps({'loaded': 'libxenon_b200' in maps, 'ref': 'libxnref_fast' in maps,\n"
            "                  'same_config': line['config'] == bench.shared_config(desc, a.level)}))\n")
    p = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    res = json.loads(p.stdout.strip().splitlines()[-1])
    assert res == {"loaded": False, "ref": True, "same_config": True}, res
