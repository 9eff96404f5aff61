"""Packet-range sharding over ranks, on the CPU: two gloo ranks each transport
half of the packet ids with the oracle (the device semantics, FP64) and reduce;
the sum equals one run over all packets (counters exactly, fluence to rounding).
This is the host logic that bench.py and multi-GPU users run over NCCL."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from signedmcrt_b200 import presets as P
from signedmcrt_b200.shard import run_sharded, shard_range

N = 6001
COUNTS = ("packets", "sdf_evals", "voxel_segments", "trace_steps", "scatters", "fresnel_events", "rng_draws")


def test_shard_ranges_partition_the_packets():
    for n in (0, 1, 7, 100, 10**12 + 3):
        for world in (1, 2, 3, 8):
            got = [shard_range(n, world, r) for r in range(world)]
            assert got[0][0] == 0 and sum(c for _, c in got) == n
            assert all(got[i][0] + got[i][1] == got[i + 1][0] for i in range(world - 1))
            assert max(c for _, c in got) - min(c for _, c in got) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    from oracle import binding as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    st = P.benchmark_settings("layered_vessels")
    arr = P.setup_simulation(st)
    pol = O.device_policy("fp64", st.grid_c())
    g = st.grid
    jm = torch.zeros(g.nxg * g.nyg * g.nzg, dtype=torch.float64)
    bins = torch.zeros(len(st.detectors) * 11, dtype=torch.float64)
    cnt = torch.zeros(len(COUNTS), dtype=torch.int64)

    def run_range(first, count):
        r = O.run(arr, st, nphotons=count, seed=5, first=first, policy=pol)
        jm.add_(torch.from_numpy(np.ascontiguousarray(r.jmean.reshape(-1, order="F"))))
        bins.add_(torch.from_numpy(r.bins))
        cnt.add_(torch.tensor([r.stats[k] for k in COUNTS], dtype=torch.int64))

    run_sharded(run_range, N, [jm, bins], counters=cnt)
    if rank == 0:
        out.put((jm.numpy().copy(), bins.numpy().copy(), cnt.numpy().copy()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_equal_one_run():
    from oracle import binding as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    jm, bins, cnt = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    st = P.benchmark_settings("layered_vessels")
    arr = P.setup_simulation(st)
    whole = O.run(arr, st, nphotons=N, seed=5, policy=O.device_policy("fp64", st.grid_c()))
    assert list(cnt) == [whole.stats[k] for k in COUNTS]
    np.testing.assert_array_equal(bins, whole.bins)
    ref = whole.jmean.reshape(-1, order="F")
    np.testing.assert_allclose(jm, ref, rtol=1e-11, atol=1e-13 * ref.max())
