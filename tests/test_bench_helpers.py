"""CPU tests of bench.py's helpers that turn committed ncu summaries into the
bench line: the DRAM traffic ratio of the panel kernel is read from the
summary of its own regime (trailing matrix larger than L2: streamed from
DRAM; smaller: resident in L2), and both summaries carry the line the bench
parses."""
import os
import sys

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..")
sys.path.insert(0, ROOT)


def test_traffic_ratio_follows_the_regime():
    import bench
    streamed, resident = bench.traffic_ratio(False), bench.traffic_ratio(True)
    assert streamed is not None and resident is not None
    # streamed: about one DRAM byte per streamed byte; resident: a few percent
    assert 0.9 <= streamed <= 1.2
    assert 0.0 < resident <= 0.1


def test_profile_summaries_name_committed_commands_only():
    # every summary's command runs committed files (no working-folder scripts)
    prof = os.path.join(ROOT, "profiles")
    for name in os.listdir(prof):
        text = open(os.path.join(prof, name)).read()
        assert "_work/" not in text, name
