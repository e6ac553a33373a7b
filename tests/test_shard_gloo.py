"""CPU, world size 2 over gloo: the G'-column sharding of one Sigma
(bgwsigma.shard) -- each rank evaluates its column block, the partials are
all-gathered and summed in rank order -- reproduces the whole-problem sum.
The per-rank compute here is the CPU oracle (this test exercises the
partition and the gather, not the kernels)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from bgwsigma import inputs as I
from bgwsigma import shard as S


def test_column_range_partitions_every_column_once():
    for P in (0, 1, 7, 102, 1638):
        for world in (1, 2, 3, 8):
            cols = []
            for r in range(world):
                p0, p1 = S.column_range(P, world, r)
                assert 0 <= p0 <= p1 <= P
                cols.extend(range(p0, p1))
            assert cols == list(range(P))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, result_path):
    import sys
    from pathlib import Path
    repo = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(repo / "berkeleygw-kernels-cpp_b200"))
    sys.path.insert(0, str(repo))
    import datetime

    import torch.distributed as dist

    from bgwsigma import inputs as I
    from bgwsigma import shard as S
    from oracle.oracle import Oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    orc = Oracle()
    g = I.gpp_seeded(16, 2, 1000, 10, seed=31)           # ngpown 100
    got_g = S.gpp_sharded(g, world, rank, compute=orc.gpp)
    f = I.ff_seeded(20, 4, 600, 45, 6, 3, seed=32)       # ngpown 45 (odd split)
    got_f = S.ff_sharded(f, world, rank, compute=lambda s: (orc.achs(s), orc.asx(s), orc.cor(s)))
    got_s = S.gpp_sigma_sharded(g, world, rank, compute=lambda s: (orc.gpp(s), orc.gpp_sx(s)))
    np.save(f"{result_path}.{rank}.npy",
            np.concatenate([got_g, [got_f[0]], got_f[1], got_f[2], got_s[0], got_s[1]]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gather_matches_whole_problem(tmp_path, oracle):
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    base = str(tmp_path / "res")
    mp.start_processes(_worker, args=(world, port, base), nprocs=world, start_method="spawn", join=True)
    r0, r1 = np.load(f"{base}.0.npy"), np.load(f"{base}.1.npy")
    assert np.array_equal(r0, r1)                           # every rank holds the same total
    g = I.gpp_seeded(16, 2, 1000, 10, seed=31)
    f = I.ff_seeded(20, 4, 600, 45, 6, 3, seed=32)
    want = np.concatenate([oracle.gpp(g), [oracle.achs(f)], oracle.asx(f), oracle.cor(f), oracle.gpp(g),
                           oracle.gpp_sx(g)])
    err = np.max(np.abs(r0 - want) / np.maximum(np.abs(want), 1e-300))
    assert err < 1e-13, err


@pytest.mark.parametrize("world", [2, 3])
def test_shards_sum_to_whole_single_process(oracle, world):
    g = I.gpp_seeded(8, 2, 700, 7, seed=5)
    parts = [oracle.gpp(S.gpp_shard(g, world, r)) for r in range(world)]
    total = np.sum(parts, axis=0)
    assert np.max(np.abs(total - oracle.gpp(g)) / np.abs(oracle.gpp(g))) < 1e-13
