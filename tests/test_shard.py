"""Frequency sharding of one ATLAS12 model (atlas12_b200.shard) on CPU ranks.

The decomposition is checked with the oracle's iteration: two gloo ranks each
run LINOP1 and the RT pass over their frequency shard, the accumulators are
all-reduced, and both ranks finish the iteration on the total.  After two
iterations both ranks must hold the structure the unsharded iteration
produces (relative 1e-9: only the grouping of the frequency sums differs).
"""
import os
import socket
import tempfile

import numpy as np
import pytest

from atlas12_b200.shard import iterate_sharded, shard_range


@pytest.mark.parametrize("numnu,world", [(30000, 1), (30000, 2), (30000, 8), (7, 7), (1001, 4)])
def test_shard_range_covers_every_frequency_once(numnu, world):
    ranges = [shard_range(numnu, r, world) for r in range(world)]
    assert ranges[0][0] == 1 and ranges[-1][1] == numnu
    for (a0, a1), (b0, b1) in zip(ranges, ranges[1:]):
        assert b0 == a1 + 1
    sizes = [b - a + 1 for a, b in ranges]
    assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1


def test_shard_range_rejects_bad_ranks():
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)
    with pytest.raises(ValueError):
        shard_range(3, 0, 4)


def _case():
    from atlas12_b200 import surrogate, synthetic
    ws, rc = synthetic.geometric_waveset(9.0, 160000.0, 600)
    lines = synthetic.atlas_lines(3000, ws[2], ws[-3], seed=5)
    start = surrogate.grey_model(5777.0, 4.44)
    return ws, rc, lines, start


def _iteration(ws, rc, lines, start, nu0=1, nu1=None):
    import pyoracle as po
    from iteration import OracleIteration
    from atlas12_b200 import atlas
    t = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_tables.npz"))
    tables = {k: t[k] for k in t.files}
    return OracleIteration(po, atlas, tables, ws, rc, lines, start, 5777.0, 1.5, nu0=nu0, nu1=nu1)


def _rank_main(rank, world, port, out_dir):
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    from iteration import pack, unpack
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    ws, rc, lines, start = _case()
    nu0, nu1 = shard_range(ws.size, rank, world)
    it = _iteration(ws, rc, lines, start, nu0, nu1)
    nr = start["t"].size
    sums = torch.zeros(8 * nr + 1, dtype=torch.float64)

    def begin():
        sums.copy_(torch.from_numpy(pack(it.begin(), nr)))

    def allreduce():
        dist.all_reduce(sums, op=dist.ReduceOp.SUM)

    def end():
        return it.end(unpack(sums.numpy(), nr))

    n, hist = iterate_sharded(begin, allreduce, end, max_iter=2, tol_percent=0.0)
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), n=n, hist=hist, t=it.st["t"], p=it.st["p"],
             rhox=it.st["rhox"], shard=np.array([nu0, nu1]))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_sharded_iteration_matches_unsharded(po):
    import torch.multiprocessing as mp
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_rank_main, args=(world, _free_port(), d), nprocs=world, join=True)
        got = [dict(np.load(os.path.join(d, f"rank{r}.npz"))) for r in range(world)]
    ws, rc, lines, start = _case()
    full = _iteration(ws, rc, lines, start)
    hist = [full.step() for _ in range(2)]
    assert got[0]["shard"].tolist() == [1, 300] and got[1]["shard"].tolist() == [301, 600]
    for r in range(world):
        assert int(got[r]["n"]) == 2
        np.testing.assert_allclose(got[r]["hist"], hist, rtol=1e-9)
        for k in ("t", "p", "rhox"):
            np.testing.assert_allclose(got[r][k], full.st[k], rtol=1e-9, err_msg=f"rank {r} {k}")
    # both ranks finish on the same total: identical structures
    np.testing.assert_array_equal(got[0]["t"], got[1]["t"])
