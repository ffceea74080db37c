"""The bench's roofline arithmetic on CPU: the algorithmic bytes of a full
reorder (the figure `roofline.achieved` divides by the launch time) and the
DRAM traffic read back from the committed ncu summaries."""
import bench_workloads as bw


def test_reorder_bytes_formula():
    # passes x (8n + 4nnz + 4) + (12n + 4nnz + 4) + (12n + 8nnz + 4)
    for n, nnz, passes in ((1, 1, 1), (4096, 20224, 3), (10, 37, 0)):
        want = passes * (8 * n + 4 * nnz + 4) + (12 * n + 4 * nnz + 4) + (12 * n + 8 * nnz + 4)
        assert bw.reorder_bytes(n, nnz, passes) == want


def test_reorder_bytes_grid3d_128():
    # the 128^3 7-point grid with its 3 start-search passes: 450.6 MB a reorder
    n, nnz = 128 ** 3, 14_581_760
    assert round(bw.reorder_bytes(n, nnz, 3) / 1e6, 1) == 450.6


def test_profile_traffic_lines():
    batch = bw.profile_value("k_solo_batch_mixed_batch_4096.md", "traffic_bytes_per_launch")
    team = bw.profile_value("k_reorder_team_grid3d_128.md", "traffic_bytes_per_launch")
    assert batch == 135_000_000_000 and team == 837_455_360
    assert bw.profile_value("no_such_profile.md", "traffic_bytes_per_launch") is None
