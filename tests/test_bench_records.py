"""bench.py reads two figures from the committed ncu summaries: the DRAM
bytes per traversal launch (the roofline's traffic) and the stage kernels'
DRAM bytes per frame on the small terrain (stage_traffic). Both parsers
must find their lines, so a summary edit that drops them shows here and
not as a silent null in the bench line."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import bench  # noqa: E402


def test_traversal_traffic_line_is_found():
    traffic = bench.profiled_traffic()
    assert traffic is not None and 1e8 < traffic < 1e11


def test_stage_traffic_lines_are_found():
    stages = bench.profiled_stage_traffic()
    assert stages is not None
    assert stages["_faces"] > 0
    names = {k for k in stages if k != "_faces"}
    assert {"begin", "finalize"} <= names and any(k.startswith("shade") for k in names)
    assert all(v > 0 for k, v in stages.items())
