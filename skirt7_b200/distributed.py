"""Multi-GPU plumbing: one process per GPU, disjoint packet ranges of one simulation, one
all-reduce of the tallies per phase.

This is the reference's MPI task mode (every process runs its share of the chunks for all
wavelengths, MonteCarloSimulation.cpp:98-104, then Instrument::sumResults reduces the frames,
Instrument.cpp:57-65) on NCCL: packets are independent, so the only exchange is the sum of the
per-rank tallies at the end of a phase.  Each packet keeps the luminosity L/Npp of the whole
simulation, so the reduced tallies equal those of one device running all packets.
"""
import numpy as np


def packet_range(npp, rank, world):
    """[first, first+count) of the npp packets per wavelength that rank runs."""
    per = -(-int(npp) // int(world))
    first = min(int(npp), rank * per)
    count = max(0, min(int(npp), first + per) - first)
    return first, count


def reduce_tallies(tensors, group=None):
    """Sums per-rank tally tensors in place across the process group (NCCL on GPUs, gloo on CPU)."""
    import torch.distributed as dist
    for t in tensors:
        dist.all_reduce(t, group=group)
    return tensors


def run_phase_sharded(ctx, phase, ells, npp, seed, rank, world, precision=0, stream=None):
    """Runs this rank's share of a phase on its device context."""
    first, count = packet_range(npp, rank, world)
    ctx.run_phase(phase, np.asarray(ells, dtype=np.int32), npp, first, count, seed=seed, precision=precision,
                  stream=stream)
    return first, count
