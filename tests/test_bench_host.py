"""bench.py's host-side pieces (no GPU): the CLI output parser both CLIs' lines
go through, the error metrics and their medians, and the reference arm's
unavailable lines for the workloads the reference has no path for."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench as B  # noqa: E402

OURS_PINNED = """\
graph: n=268435456 m=8472312086 chunks=133 (cap 64000000, max 64000000 edges, 16724959 vertices)  open 0.91s
fetch rule: tau = 0.785 (stream 0.128s; gather 0.008s / 0.024s / 0.065s at demand 0.050 / 0.150 / 0.400)  calibrate 0.27s
host cache: pinned, 26.72 GB (105 chunks past the GPU cache), lists read in place over the host link (GPU cache load 3.57s, read 12.49s, pinning 0.10s past the read)
staging: pinned host buffers copied to the GPU
GPU edge cache: 28/133 chunks resident (21.1% of edges)  setup 19.51s
pass   0: pending 268435456 v, demand ratio 1.0000 | resident 133 stream 0 gather 0 | cached high-degree pending 0 | faults major 0 minor 0 | gather pages 0 runs 0
passes 44  measure pr (n=268435456):  pr sum 1.391851e+08
edges pushed: 20.90 x |E|
bytes shipped: stream 0.00 GB, gather 524.93 GB (graph edges 33.89 GB)
page faults in passes: major 0, minor 0 | gather dedup on: 0 pages in 0 runs
time: open 0.91s setup 19.51s passes 12.39s [cpu io 0.00s, gpu wait 12.39s, snapshot 0.00s] result 0.89s | internal total 33.70s
"""

REFERENCE = """\
graph: n=268435456 m=8472312086 chunks=133 (cap 64000000, max 64000000 edges, 16724959 vertices)  open 0.06s
fetch rule: tau = 0.785 (measured earlier on this machine in 0.27s, /tmp/x.tau)
GPU degree cache: 112701 vertices with degree >= 12095 (28.3% of edges, 9.59 GB)  setup 2.93s
passes 50  measure pr (n=268435456):  pr sum 1.389280e+08
edges pushed: 21.59 x |E|
bytes shipped: stream 123.69 GB, gather 346.26 GB (graph edges 33.89 GB)
page faults in passes: major 0, minor 457908 | gather dedup on: 107904114 pages in 8131993 runs
time: open 0.06s setup 2.93s passes 33.23s [cpu io 29.87s, gpu wait 3.03s, snapshot 0.18s] result 0.52s | internal total 36.74s
pass   0: pending 268435456 v, demand ratio 1.0000 | resident 0 stream 133 gather 0 | cached high-degree pending 0 | faults major 0 minor 9 | gather pages 0 runs 0
pass   1: pending 33031227 v, demand ratio 0.6583 | resident 0 stream 36 gather 97 | cached high-degree pending 112701 | faults major 0 minor 301930 | gather pages 3979715 runs 77907
"""


def test_parse_cli_reads_both_clis_lines():
    f = B.parse_cli(OURS_PINNED)
    assert (f["passes"], f["pushed_x_m"], f["passes_s"]) == (44, 20.90, 12.39)
    assert (f["stream_gb"], f["gather_gb"], f["gather_passes"]) == (0.0, 524.93, 0)
    assert f["setup_s"] == 19.51 and f["tau"] == 0.785 and f["gpu_wait_s"] == 12.39
    assert f["host_cache_s"] == {"gpu_cache_load": 3.57, "read": 12.49, "pinning_past_the_read": 0.10}
    g = B.parse_cli(REFERENCE)
    assert (g["passes"], g["pushed_x_m"], g["passes_s"]) == (50, 21.59, 33.23)
    assert (g["stream_gb"], g["gather_gb"], g["major_faults"]) == (123.69, 346.26, 0)
    assert g["gather_passes"] == 1 and g["cpu_io_s"] == 29.87 and "host_cache_s" not in g


def test_error_metrics():
    rng = np.random.default_rng(5)
    ref = rng.random(5000) + 0.01
    x = (ref * (1 + 1e-3 * rng.standard_normal(5000))).astype(np.float32)
    e = B.error_vs_fp64("pr", ref, x)
    d = np.abs(x.astype(np.float64) - ref)
    assert e["l1_rel"] == pytest.approx(d.sum() / ref.sum()) and e["max_abs"] == pytest.approx(d.max())
    assert 990 <= e["top1000"] <= 1000
    # the eigenvector is compared as a unit vector with its sign fixed by its sum
    e2 = B.error_vs_fp64("ev", ref, (-3.0 * ref).astype(np.float32))
    assert e2["l1_rel"] < 1e-6 and e2["top1000"] == 1000


def test_median_errors_and_ranges():
    runs = [{"pr": {"l1_rel": a, "max_abs": b, "top1000": c}} for a, b, c in
            [(0.03, 5.0, 990), (0.01, 9.0, 999), (0.02, 1.0, 995)]]
    m = B.median_errors(runs)["pr"]
    assert (m["l1_rel"], m["max_abs"], m["top1000"]) == (0.02, 5.0, 995)
    assert m["l1_range"] == [0.01, 0.03] and m["max_abs_range"] == [1.0, 9.0]


@pytest.mark.parametrize("config,why", [("ppr256", "no batched personalized PageRank"),
                                        ("adjoint22", "no adjoint or gradient path"),
                                        ("ooc28", "does not run out of core")])
def test_reference_arm_unavailable_lines(config, why):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", config],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and why in line["unavailable"]
