"""The N>1 path on CPU: two gloo ranks shard cameras and pixel ranges, trace
their shares with the CPU oracle standing in for the GPU tracer, and rank 0
reassembles results identical to one process.  Also a rank that fails is seen
by the other rank on the host, through a short process-group timeout."""
from __future__ import annotations

import datetime
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir, mode):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import hadros_b200 as hb
    from hadros_b200 import shard
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    E, _, s = W.synthetic_sigma_arrays()
    try:
        if mode == "scan":
            cams = [hb.params(**W.mixed_512(nx=n, ny=m, h=0.06, precision="fp64", profile=k % 8))
                    for k, (n, m) in enumerate([(3, 2), (1, 4), (2, 2), (4, 1), (2, 3)])]
            res = shard.run_scan(cams, lambda cs: [O.oracle_image(c, E, s, threads=1) for c in cs],
                                 dist, rank, world)
            if rank == 0:
                np.save(Path(outdir) / "scan.npy", np.array(res, dtype=object), allow_pickle=True)
        elif mode == "image":
            p = hb.params(**W.mixed_512(nx=5, ny=3, h=0.06, precision="fp64"))
            img = shard.run_image_sharded(
                p, lambda q, ids: O.oracle_image(q, E, s, pixel_ids=ids, threads=1), dist, rank, world)
            t = shard.max_over_ranks(float(rank + 1), dist)
            if rank == 0:
                np.save(Path(outdir) / "image.npy", np.array([img, t], dtype=object), allow_pickle=True)
        elif mode == "robustness":
            from hadros_b200 import robustness as R
            rows, _ = R.run(None, None, pixels=2, dist=dist, rank=rank, world=world,
                            trace=lambda cs: [O.oracle_image(c, E, s, threads=1, mev=True) for c in cs])
            if rank == 0:
                np.save(Path(outdir) / "robustness.npy", np.array(rows, dtype=object), allow_pickle=True)
            else:
                assert rows is None
        elif mode == "points":
            from hadros_b200 import scan
            cams = [hb.params(**W.production_point(nx=3, ny=2, h=0.08, n_bins=2, precision="fp64",
                                                   rho0_gcm3=10.0 ** (9 + k))) for k in range(3)]

            def evaluate(k):   # the oracle stands in for the surrogate scan point
                img = O.oracle_image(cams[k], E, s, threads=1)
                return {"point": k, "rank": rank, "I_obs": img["I_obs"]}
            rows = scan.run_points(len(cams), evaluate, dist, rank, world)
            if rank == 0:
                np.save(Path(outdir) / "points.npy", np.array(rows, dtype=object), allow_pickle=True)
        elif mode == "fail":
            if rank == 1:
                raise RuntimeError("rank 1 fails before its first collective")
            try:
                shard.max_over_ranks(1.0, dist)
                (Path(outdir) / "fail.txt").write_text("no error")
            except Exception as e:   # the peer never joined: the collective errors out
                (Path(outdir) / "fail.txt").write_text("error: " + type(e).__name__)
    finally:
        if mode != "fail":
            dist.destroy_process_group()


def _spawn(mode, tmp_path, world=2):
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path), mode)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    return procs


def test_partition_balances_and_covers():
    from hadros_b200 import shard
    costs = [64 * 64, 1024 * 1024, 512 * 512, 100, 700 * 700, 64 * 64, 300 * 300]
    parts = shard.partition_cameras(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) == costs[1]          # the biggest camera alone bounds the makespan
    assert shard.pixel_range(10, 0, 3) == (0, 4) and shard.pixel_range(10, 2, 3) == (7, 10)
    assert sum(b - a for a, b in (shard.pixel_range(1001, r, 7) for r in range(7))) == 1001


def test_two_rank_camera_scan_equals_single_process(tmp_path, hb):
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    procs = _spawn("scan", tmp_path)
    assert all(p.exitcode == 0 for p in procs)
    res = np.load(tmp_path / "scan.npy", allow_pickle=True)
    E, _, s = W.synthetic_sigma_arrays()
    for k, (n, m) in enumerate([(3, 2), (1, 4), (2, 2), (4, 1), (2, 3)]):
        one = O.oracle_image(hb.params(**W.mixed_512(nx=n, ny=m, h=0.06, precision="fp64",
                                                    profile=k % 8)), E, s, threads=1)
        for key in one:
            np.testing.assert_array_equal(res[k][key], one[key], err_msg=f"camera {k} {key}")


def test_two_rank_pixel_shards_equal_single_process(tmp_path, hb):
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    procs = _spawn("image", tmp_path)
    assert all(p.exitcode == 0 for p in procs)
    img, tmax = np.load(tmp_path / "image.npy", allow_pickle=True)
    assert tmax == 2.0
    E, _, s = W.synthetic_sigma_arrays()
    one = O.oracle_image(hb.params(**W.mixed_512(nx=5, ny=3, h=0.06, precision="fp64")), E, s)
    for key in one:
        np.testing.assert_array_equal(img[key], one[key], err_msg=key)


def test_failed_rank_is_reported_not_hung(tmp_path):
    procs = _spawn("fail", tmp_path)
    assert procs[1].exitcode != 0
    assert (tmp_path / "fail.txt").read_text().startswith("error")


def test_two_rank_robustness_scan_equals_single_process(tmp_path, hb):
    """hadros_b200.robustness.run with its 47 cases split over two gloo ranks
    (the oracle tracing on CPU) gives the single-process rows."""
    from hadros_b200 import robustness as R
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    procs = _spawn("robustness", tmp_path)
    assert all(p.exitcode == 0 for p in procs)
    rows = list(np.load(tmp_path / "robustness.npy", allow_pickle=True))
    E, _, s = W.synthetic_sigma_arrays()
    one, _ = R.run(None, None, pixels=2, trace=lambda cs: [O.oracle_image(c, E, s, threads=1, mev=True)
                                                            for c in cs])
    assert len(rows) == len(one) == len(R.cases())
    assert rows == one


def test_two_rank_scan_points_meet_in_point_order(tmp_path, hb):
    """hadros_b200.scan.run_points (the production scan's driver) splits the
    points over two ranks; rank 0 gets every point's row in order."""
    from hadros_b200 import workloads as W
    from oracle import pyoracle as O
    procs = _spawn("points", tmp_path)
    assert all(p.exitcode == 0 for p in procs)
    rows = list(np.load(tmp_path / "points.npy", allow_pickle=True))
    assert [r["point"] for r in rows] == [0, 1, 2] and {r["rank"] for r in rows} == {0, 1}
    E, _, s = W.synthetic_sigma_arrays()
    for k, r in enumerate(rows):
        p = hb.params(**W.production_point(nx=3, ny=2, h=0.08, n_bins=2, precision="fp64",
                                           rho0_gcm3=10.0 ** (9 + k)))
        np.testing.assert_array_equal(r["I_obs"], O.oracle_image(p, E, s, threads=1)["I_obs"])
