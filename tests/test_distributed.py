"""Multi-rank plumbing on CPU (gloo, world size 2): query sharding, gathering,
point broadcast and the LPT forest split.  The per-rank search is the CPU oracle
here (test stand-in for the GPU search); the product path calls the GPU."""
import os
import socket

import numpy as np
import pytest


def test_shard_bounds_cover_everything():
    from cosmokdtree_b200.distributed import shard_bounds
    for n in (0, 1, 7, 100, 1001):
        for w in (1, 2, 3, 8):
            parts = [shard_bounds(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(w - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


def test_lpt_partition_balance():
    from cosmokdtree_b200.distributed import lpt_partition
    rng = np.random.default_rng(0)
    sizes = np.floor(10 ** rng.uniform(3, 6, 2000)).astype(int)
    for w in (2, 4, 8):
        parts = lpt_partition(sizes, w)
        assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
        loads = [sizes[p].sum() for p in parts]
        # LPT bound: max load <= (4/3 - 1/(3w)) OPT, and OPT >= mean
        assert max(loads) <= (4 / 3) * np.mean(loads) + sizes.max()
        assert max(loads) / np.mean(loads) < 1.01


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    import sys
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import oracle
    from cosmokdtree_b200 import distributed as D
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        rng = np.random.default_rng(5)
        P = torch.from_numpy(rng.random((5000, 3)) - 0.5) if rank == 0 else None
        P = D.broadcast_points(P)  # rank 0's points reach every rank
        Q = np.random.default_rng(6).random((1001, 3)) - 0.5
        tree = oracle.OracleTree(P.numpy(), 16, [1.0, 1.0, 1.0])

        def search(t, q, k, s):
            d, i = t.knn(q, k, sorted=s)
            return torch.from_numpy(d), torch.from_numpy(i)

        d_loc, i_loc, (lo, hi) = D.knn_sharded(tree, Q, 9, search=search)
        d_all, i_all = D.knn_sharded(tree, Q, 9, search=search, gather=True)
        ref_d, ref_i = tree.knn(Q, 9)
        ok = (np.array_equal(i_all.numpy(), ref_i) and np.array_equal(d_all.numpy(), ref_d)
              and np.array_equal(i_loc.numpy(), ref_i[lo:hi]))
        sizes = [50 + 10 * t for t in range(9)]
        trees = [np.random.default_rng(t).random((m, 3)) - 0.5 for t, m in enumerate(sizes)]
        built, owned = D.build_forest_sharded(
            trees, build=lambda pts, leaf, boxsize: [len(p) for p in pts])
        owned_all = [None] * world
        dist.all_gather_object(owned_all, owned)
        ok = ok and sorted(sum(owned_all, [])) == list(range(9)) and built == [sizes[i] for i in owned]
        with open(os.path.join(out_dir, f"r{rank}"), "w") as f:
            f.write("ok" if ok else "bad")
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    assert (tmp_path / "r0").read_text() == "ok"
    assert (tmp_path / "r1").read_text() == "ok"


def test_bench_rejects_world_size_mismatch():
    """bench.py --gpus N under a launcher that started another number of ranks stops
    with an error instead of timing the wrong number of GPUs."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 2
    assert "WORLD_SIZE=1" in json.loads(r.stdout.strip().splitlines()[-1])["error"]
