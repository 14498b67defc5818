"""The N>1 path on CPU with gloo ranks (world size 2): packet ranges are disjoint and cover the
simulation, and the all-reduce of per-rank tallies reproduces the single-process result.  Tallies
come from the oracle run on each rank's share of the packets, so the reduction is exercised on
real frames; a deterministic additive stand-in checks exactness."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from skirt7_b200.distributed import packet_range, reduce_tallies


@pytest.mark.parametrize("npp,world", [(10, 3), (1_000_000, 2), (7, 8), (1, 4), (0, 2)])
def test_packet_ranges_partition(npp, world):
    covered = []
    for r in range(world):
        f, c = packet_range(npp, r, world)
        assert c >= 0 and f + c <= npp
        covered += list(range(f, f + c)) if npp < 10_000 else [f, f + c - 1]
    if npp < 10_000:
        assert sorted(covered) == list(range(npp))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, npp, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # additive stand-in for a phase: each packet id deposits a deterministic amount in a pixel
    f, c = packet_range(npp, rank, world)
    ids = np.arange(f, f + c)
    frame = np.zeros((16, 16))
    np.add.at(frame, (ids % 16, (ids * 7) % 16), 1.0 / (1 + ids))
    t = torch.from_numpy(frame)
    reduce_tallies([t])
    # the oracle on this rank's share, reduced
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import oracle
    from skirt7_b200 import models
    m = models.oligo_disk(N=(20, 20, 10), npix=20, with_sed=True)
    r = oracle.simulate(m, 4000, nthreads=2, seed=11 + 1000 * rank, max_packets=c and 2000)
    sed = torch.from_numpy(np.ascontiguousarray(r["seds"][1]))
    reduce_tallies([sed])
    if rank == 0:
        out.put((t.numpy().copy(), sed.numpy().copy()))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_reduction_matches_single_process():
    npp, world = 5000, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, npp, q)) for r in range(world)]
    for p in ps:
        p.start()
    frame, sed = q.get(timeout=300)
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    ids = np.arange(npp)
    ref = np.zeros((16, 16))
    np.add.at(ref, (ids % 16, (ids * 7) % 16), 1.0 / (1 + ids))
    assert np.allclose(frame, ref, rtol=1e-14, atol=0)
    # two half-runs of 2000 packets each, every packet carrying L/4000: the summed SED estimates the
    # same flux as one run (within Monte Carlo noise)
    assert sed[0, 0] > 0
