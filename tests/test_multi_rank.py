"""The N>1 path on CPU with gloo ranks: the packet ranges of skirt7_b200.distributed partition a
simulation, and the all-reduce of the ranks' tallies (reduce_tallies) reproduces the single-process
run.  Each rank runs the oracle's stellar phase on exactly its packet range (every packet on its
own counter-based stream, oracle.simulate_packets), so the reduced frames, SEDs and absorbed
luminosities must equal those of one process running all packets, up to the order of the FP64
additions."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from skirt7_b200.distributed import packet_range, reduce_tallies

NPP = 3000


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


def _model():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from helpers import cell_center_density
    from skirt7_b200 import models
    m = models.oligo_disk(N=(20, 20, 10), npix=24, with_sed=True)
    m.rho = cell_center_density(m)
    return m


def _oracle():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import oracle
    return oracle


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    f, c = packet_range(NPP, rank, world)
    r = _oracle().simulate_packets(_model(), NPP, f, c, nthreads=2, seed=99)
    t = [torch.from_numpy(np.ascontiguousarray(r["cubes"][0])), torch.from_numpy(np.ascontiguousarray(r["seds"][1])),
         torch.from_numpy(np.ascontiguousarray(r["labs_stel"]))]
    reduce_tallies(t)
    if rank == 0:
        out.put(([x.numpy().copy() for x in t], int(r["stats"]["packets"])))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_reduction_matches_single_process(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    (frame, sed, labs), _ = q.get(timeout=300)
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    whole = _oracle().simulate_packets(_model(), NPP, 0, NPP, nthreads=4, seed=99)
    assert whole["stats"]["packets"] == NPP
    for got, ref in ((frame, whole["cubes"][0]), (sed, whole["seds"][1]), (labs, whole["labs_stel"])):
        assert ref.sum() > 0
        assert np.allclose(got, ref, rtol=1e-11, atol=1e-14 * np.abs(ref).max())
    # a different split of the same packets changes nothing either; a different seed does
    half = [_oracle().simulate_packets(_model(), NPP, f, c, nthreads=2, seed=99) for f, c in ((0, 1000), (1000, 2000))]
    assert np.allclose(half[0]["cubes"][0] + half[1]["cubes"][0], whole["cubes"][0], rtol=1e-11,
                       atol=1e-14 * whole["cubes"][0].max())
    other = _oracle().simulate_packets(_model(), NPP, 0, NPP, nthreads=4, seed=98)
    assert not np.allclose(other["cubes"][0], whole["cubes"][0], rtol=1e-6)
