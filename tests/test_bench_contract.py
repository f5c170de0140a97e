"""Host-side parts of bench.py's contract that need no GPU."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun only rank 0 times the reference; the other ranks exit 0 and print nothing."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_roofline_inputs_from_committed_profile():
    """The SGD roofline's DRAM traffic and L2 figures come from the committed ncu summary."""
    sys.path.insert(0, ROOT)
    import bench
    tr = bench.traffic_per_epoch()
    assert tr is not None and tr > 1e8
    l2 = bench.l2_counters()
    assert l2 is not None
    for k in ("l2_throughput_pct", "l2_hit_rate_pct", "issue_active_pct"):
        assert 0.0 < l2[k] <= 100.0, (k, l2[k])
