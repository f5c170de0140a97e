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
    # the 100M-point roll's traffic scales the 40M capture by kept edges
    t40 = bench.ncu_figure("sgd_epoch_swiss_roll_40m_renamed", "traffic_bytes_per_launch")
    e40 = bench.ncu_figure("sgd_epoch_swiss_roll_40m_renamed", "kept_edges")
    assert t40 and e40 and abs(bench.swiss_traffic(2 * e40) - 2 * t40) <= 1e-6 * t40


def test_both_arms_share_one_config():
    """The default workload's `config` is built by one function for both arms from the
    workload and the cached inputs' digest, and carries no per-arm timing or work counts."""
    sys.path.insert(0, ROOT)
    import bench
    info = {"knn": "exact", "knn_rows_recomputed": 0, "inputs_sha1_16": "0123456789abcdef"}
    c1 = bench.fit_config(2_000_000, 500, 1, info)
    c2 = bench.fit_config(2_000_000, 500, 1, dict(info))
    assert c1 == c2 and c1["workload"] == "gaussians_2000000_d64_k15_500ep"
    assert not {"knn_seconds", "kept_edges", "edge_updates_per_fit"} & set(c1)
