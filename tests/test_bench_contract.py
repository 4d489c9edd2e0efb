"""Host-side pieces of bench.py's JSON line that need no GPU: the roofline's
DRAM traffic comes from the committed ncu summaries, and every summary
states the command that produced it (with the clock-control flag)."""
import re
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def _figure(name):
    text = (ROOT / "profiles" / name).read_text()
    return float(re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", text).group(1))


def test_span_traffic_sums_both_kernels():
    """The 3D roofline span covers the early-out pass and the clipper; its
    traffic is the sum of both kernels' per-launch DRAM bytes."""
    want = _figure("k_prefilter_tets_tet3d_27x32.md") + _figure("k_clip_tets_ix_tet3d_27x32.md")
    assert bench.profile_traffic("k_prefilter_tets+k_clip_tets_ix", "tet3d_27x32") == want
    assert want > 0


def test_traffic_for_each_workload_with_a_summary():
    assert bench.profile_traffic("k_clip_tris", "tri2d_777x1024_rot7") == _figure(
        "k_clip_tris_tri2d_777x1024_rot7.md")
    assert bench.profile_traffic("k_clip_tris", "no_such_workload") is None
    assert bench.profile_traffic("k_prefilter_tets+no_such_kernel", "tet3d_27x32") is None


def test_profiles_state_their_commands():
    files = sorted((ROOT / "profiles").glob("*.md"))
    assert files
    for f in files:
        text = f.read_text()
        assert "ncu " in text and "--clock-control none" in text, f.name
        assert len(text) < 16384, f.name  # short summaries, not raw reports


def test_whole_job_rate_counts_all_ranks():
    assert bench.whole_job_rate(10_046_724, 20, 1, 50.0) == 10_046_724 * 20 / 0.05
    assert bench.whole_job_rate(100, 10, 4, 10.0) == 4 * bench.whole_job_rate(100, 10, 1, 10.0)
