"""bench.py helpers that need no GPU: the `config` both arms print is one
function of the workload (so the two JSON lines describe the same problem),
and the roofline's figures parse from the committed ncu summary."""
import os
import sys

from conftest import ROOT

sys.path.insert(0, ROOT)


def test_both_arms_share_one_config():
    import bench
    from piro_b200 import workloads as W
    cfg = W.heat_be_128()
    a = bench.bench_config(cfg, 1)
    assert a == bench.bench_config(cfg, 1)
    nx, ny, nz = cfg["n"]
    N = nx * ny * nz
    assert a["nnz_A"] == 7 * N - 2 * (nx * ny + ny * nz + nx * nz) == 14581760
    assert a["grid"] == [128, 128, 128] and a["steps_in_trajectory"] == 20
    assert bench.bench_config(cfg, 4)["parallelism"] == "replicas x4"
    # the reference arm builds its line from the same function
    src = open(os.path.join(ROOT, "bench.py")).read()
    assert src.count("bench_config(cfg,") >= 2


def test_roofline_figures_parse_from_the_committed_capture():
    import bench
    m = bench.profiled_metrics("k_be_persistent")
    assert m["traffic_bytes_per_launch"] > 0
    for k in ("lts__throughput.avg.pct_of_peak_sustained_elapsed",
              "smsp__issue_active.avg.pct_of_peak_sustained_active", "gpu__time_duration.sum"):
        assert 0 < m[k], k
    assert bench.profiled_metrics("no_such_kernel") == {}
