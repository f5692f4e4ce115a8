"""CPU checks of the measurement records `bench.py` reads: every DRAM-traffic
figure in profiles/dram_traffic.json names a committed capture summary, the
summary's read + write bytes give that figure (to its printed precision),
and the summary carries the command that made it with --clock-control none;
ncu_traffic returns the figure for the default workload's dominant kernel."""
import json
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _mb(text, metric):
    m = re.search(r"`" + re.escape(metric) + r"` \| ([0-9.]+) MB", text)
    assert m, metric
    return float(m.group(1)) * 1e6


def test_traffic_records_match_their_captures():
    rec = json.load(open(os.path.join(ROOT, "profiles", "dram_traffic.json")))
    n = 0
    for config, kernels in rec.items():
        if config.startswith("_"):
            continue
        for kernel, r in kernels.items():
            path = os.path.join(ROOT, r["capture"])
            assert os.path.exists(path), path
            text = open(path).read()
            assert "--clock-control none" in text and "ncu " in text, path
            total = _mb(text, "dram__bytes_read.sum") + _mb(text, "dram__bytes_write.sum")
            assert abs(total - r["bytes_per_launch"]) <= 0.2e6, (kernel, total, r["bytes_per_launch"])
            n += 1
    assert n >= 4


def test_bench_reads_the_dominant_kernels_traffic():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    t = bench.ncu_traffic("shear3d", "k_xmarch")
    assert t is not None and t > 1e8
    assert bench.ncu_traffic("shear3d", "no_such_kernel") is None


def test_profile_summaries_name_no_round_and_run_committed_files():
    for name in os.listdir(os.path.join(ROOT, "profiles")):
        assert not re.search(r"round|_r\d", name), name
        if name.endswith(".md"):
            text = open(os.path.join(ROOT, "profiles", name)).read()
            for cmd in re.findall(r"```\n(.*?)```", text, flags=re.S):
                # committed files only: no scratch folder, no absolute path
                assert "_work" not in cmd and not re.search(r"(^|\s)/", cmd), (name, cmd)
