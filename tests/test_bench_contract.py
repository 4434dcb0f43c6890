"""The reference arm of bench.py on the CPU: one JSON line with the keys the
benchmark contract fixes, the oracle timed on the host cores over the whole
grid of the workload our arm runs, no host/device transfers, and none of the
product's native code mapped into the process.  The CPU suite runs it on the
small 64x64x128 workload; the driver runs it on the headline grid."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


SMALL = "c1_64x64x128_fp64"


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3", "--workload", SMALL], capture_output=True, text=True, timeout=300,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["steps"] == 1 and d["warmup"] == 3
    assert d["value"] > 0 and d["unit"] == "GCell-updates/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == SMALL and d["config"]["grid"] == [64, 64, 128]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_two_ranks_prints_once():
    # under torchrun rank 0 alone runs the reference arm; the other rank exits 0
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", "29541", os.path.join(ROOT, "bench.py"),
                        "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--workload", SMALL],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2


def test_reference_arm_maps_no_product_library():
    # the arm imports the package's deck and initial-state modules; the
    # product library must stay unmapped (only the oracle's library loads)
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3', "
            "'--workload', '%s']\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\nexcept SystemExit as e:\n"
            "    assert not e.code, e.code\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libpf3d.so' not in maps, 'libpf3d.so mapped'\n"
            "assert 'libpf_oracle.so' in maps\n"
            "print('maps checked')\n" % SMALL)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "maps checked" in r.stdout
