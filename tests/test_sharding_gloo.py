"""Multi-process sharding of the life cycle, on CPU with the gloo backend (world size 2).

Histories are independent and every tally is additive, so ranks split a segment into contiguous
history ranges (skgpu.sharding.history_range, as `bench.py` does under torchrun) and the segment's
tallies are the sum over ranks. The ranks here trace their ranges with the CPU oracle (the same
Philox streams and walkers as the CUDA library) and sum every tally (frame and SED totals, their
per-history statistics and components, the radiation field) with skgpu.sharding.allreduce_results
over gloo; the result must equal one process tracing the whole segment. The max-over-ranks timing
reduction is checked on the same group."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

N = 3000
SEED = 5


def _scene():
    from skgpu import workloads
    sc = workloads.shell_cartesian(12, 16, stats=True)
    sc.instruments[1]["comps"] = 1
    sc.store_rf = True
    sc.rf = dict(num_bins=1, borders=np.array([0.5e-6, 0.6e-6]), ellv=np.array([-1, 0, -1], np.int32))
    return sc


def _flat(res):
    from skgpu.sharding import _result_arrays
    return np.concatenate([np.asarray(a, float).ravel() for a in _result_arrays(res)])


def _worker(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "skirt9-gpu_b200"), os.path.join(root, "oracle")]
    import oracle
    from skgpu.sharding import allreduce_results, history_range
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = _scene()
        be = oracle.backend()
        sc.upload(be)
        first, count = history_range(rank, world, N)
        res = sc.run(be, N, seed=SEED, first=first, count=count)
        assert res.rf is not None and res.instruments[0]["stats"] is not None
        t = torch.from_numpy(_flat(allreduce_results(res)))
        ms = torch.tensor([10.0 + rank])
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        hist = torch.tensor([float(res.counters["histories"])])
        dist.all_reduce(hist)
        if rank == 0:
            np.save(out, np.concatenate([t.numpy(), ms.numpy(), hist.numpy()]))
        be.close()
    finally:
        dist.barrier()
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_history_ranges_partition_the_segment():
    from skgpu.sharding import history_range
    for world in (1, 2, 3, 8):
        spans = [history_range(r, world, 1001) for r in range(world)]
        assert spans[0][0] == 0 and sum(c for _, c in spans) == 1001
        assert all(spans[i][0] + spans[i][1] == spans[i + 1][0] for i in range(world - 1))


def test_two_gloo_ranks_sum_to_the_full_segment(tmp_path):
    import oracle
    out = str(tmp_path / "sum.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    sc = _scene()
    be = oracle.backend()
    sc.upload(be)
    full = _flat(sc.run(be, N, seed=SEED))
    be.close()
    assert got[-1] == N  # histories over both ranks
    assert got[-2] == 11.0  # max over ranks
    tot = got[:-2]
    assert tot.shape == full.shape
    assert np.allclose(tot, full, rtol=1e-12, atol=1e-300 + 1e-14 * np.abs(full).max())
