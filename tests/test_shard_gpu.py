"""GPU, world size 2 over gloo: the G'-column sharding of one Sigma
(bgwsigma.shard) with its default compute -- each rank evaluates its column
block with the CUDA library on cuda:0 -- reproduces the whole-problem sum of
the long-double oracle.  The two ranks' kernels are independent (no kernel
waits on another rank); the partials are gathered on the host by gloo."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from bgwsigma import inputs as I
from conftest import FP64_RTOL

pytestmark = pytest.mark.gpu


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
    os.environ["BGW_SIGMA_NO_BUILD"] = "1"
    import datetime

    import torch
    import torch.distributed as dist

    import bgwsigma
    from bgwsigma import inputs as I
    from bgwsigma import shard as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    bgwsigma.load(build_if_needed=False)
    g = I.gpp_seeded(24, 2, 1536, 12, seed=41)             # ngpown 128
    got_host = S.gpp_sharded(g, world, rank)                # host inputs: the library stages them
    got_dev = S.gpp_sharded(g, world, rank, device=dev)      # device-resident shards
    got_s = S.gpp_sigma_sharded(g, world, rank, device=dev)
    f = I.ff_seeded(20, 4, 640, 45, 6, 3, seed=42)          # ngpown 45 (odd split)
    got_f = S.ff_sharded(f, world, rank, device=dev)
    np.save(f"{result_path}.{rank}.npy",
            np.concatenate([got_host, got_dev, got_s[0], got_s[1], [got_f[0]], got_f[1], got_f[2]]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gpu_shards_match_whole_problem(tmp_path, oracle):
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    base = str(tmp_path / "res")
    mp.start_processes(_worker, args=(world, port, base), nprocs=world, start_method="spawn", join=True)
    r0, r1 = np.load(f"{base}.0.npy"), np.load(f"{base}.1.npy")
    assert np.array_equal(r0, r1)                           # every rank holds the same total
    g = I.gpp_seeded(24, 2, 1536, 12, seed=41)
    f = I.ff_seeded(20, 4, 640, 45, 6, 3, seed=42)
    ach = oracle.gpp(g)
    want = np.concatenate([ach, ach, ach, oracle.gpp_sx(g), [oracle.achs(f)], oracle.asx(f), oracle.cor(f)])
    # Per output block (each scaled by its own magnitude).
    blocks = [(0, 3), (3, 6), (6, 9), (9, 12), (12, 13), (13, 16), (16, 19)]
    for a, b in blocks:
        err = np.max(np.abs(r0[a:b] - want[a:b])) / np.max(np.abs(want[a:b]))
        assert err < FP64_RTOL, (a, b, err)
