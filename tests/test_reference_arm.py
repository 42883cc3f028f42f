"""bench.py --impl reference: the oracle timed on the host cores, the one
baseline the bench reports against the GPU arm. It must run without the
product library (libvgi not mapped, the vgi package not imported), print the
bench contract's line with "impl": "reference", zero copy bytes, a
cpu_baseline block describing its own run, and the GPU arm's config word for
word (bench_config), so the two arms time the same workload."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = """
import runpy, sys
sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3']
runpy.run_path('bench.py', run_name='__main__')
maps = open('/proc/self/maps').read()
print(json.dumps({'libvgi_mapped': 'libvgi' in maps, 'vgi_imported': 'vgi' in sys.modules}))
"""


def test_reference_arm_runs_without_the_library_and_matches_the_gpu_config():
    out = subprocess.run([sys.executable, "-c", "import json\n" + PROBE], cwd=ROOT, capture_output=True, text=True, timeout=900,
                         env={**os.environ, "CUDA_VISIBLE_DEVICES": ""})
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(line) for line in out.stdout.splitlines() if line.startswith("{")]
    line, probe = lines[-2], lines[-1]
    assert probe == {"libvgi_mapped": False, "vgi_imported": False}
    assert line["impl"] == "reference" and line["unit"] == "rays/s" and line["value"] > 0
    assert line["e2e"] == {"value": line["value"], "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    base = line["cpu_baseline"]
    assert base["value"] == line["value"] and base["kind"] == "port" and base["cores"] >= 1 and base["sample"]
    sys.path.insert(0, ROOT)
    import bench

    assert line["config"] == bench.bench_config(line["config"]["faces"], 3)
