"""bench.py's reference arm runs the reference's CPU receive path only: building its workload
(the simulator, the descriptors) and timing it must not load this project's CUDA library, and its
line carries the same config as the GPU arm's."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))

PROBE = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"]
sys.path.insert(0, {root!r})
import bench
bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({{"mapped_product": "libpusch_b200" in maps, "mapped_reference": "libocudu_ref" in maps}}))
"""


def test_reference_arm_maps_no_product_library():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libocudu_ref.so")):
        pytest.skip("oracle/_ref not built")
    out = subprocess.run([sys.executable, "-c", PROBE.format(root=ROOT)], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    bench_line, maps = lines[0], lines[-1]
    assert not maps["mapped_product"]
    assert maps["mapped_reference"]
    assert bench_line["impl"] == "reference"
    sys.path.insert(0, ROOT)
    import bench
    from pusch_b200 import sim
    assert bench_line["config"] == bench.pusch_config(sim.uneven_cells(seed=0, nof_cells=bench.N_CELLS), 1, 0)
