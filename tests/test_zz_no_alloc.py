"""skg_trace_paths_noalloc (device buffers in and out, scratch in a static device array) gives
the same offsets, cells and segment lengths as skg_trace_paths, call after call (up to the
largest call the scratch array holds), allocates no device memory, and leaves the error flags of
a finished phase for skg_sync.  Named so that it is collected after every other test file."""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import models, runtime
from skirt7_b200.scene import KPC

from helpers import cell_center_density, seeded_rays

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

EXT = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)


def _ctx(N=(100, 100, 50)):
    m = models.oligo_disk(N=N)
    m.rho = cell_center_density(m)
    return runtime.Context(m)


def _noalloc(ctx, r, k, capacity, precision, stream):
    n = len(r)
    dr = torch.from_numpy(np.ascontiguousarray(r)).cuda()
    dk = torch.from_numpy(np.ascontiguousarray(k)).cuda()
    cells = torch.full((max(capacity, 1),), -7, dtype=torch.int32, device="cuda")
    ds = torch.full((max(capacity, 1),), -7.0, dtype=torch.float64, device="cuda")
    off = torch.full((n + 1,), -7, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    ctx.trace_paths_noalloc(dr.data_ptr(), dk.data_ptr(), n, cells.data_ptr(), ds.data_ptr(), off.data_ptr(),
                            capacity, precision, stream.cuda_stream)
    stream.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return off.cpu().numpy(), cells.cpu().numpy(), ds.cpu().numpy(), free1 - free0


def test_noalloc_matches_trace_paths_on_consecutive_calls():
    ctx = _ctx()
    stream = torch.cuda.Stream()
    # the larger call first, so that a read of stale scratch would show in the second one
    for call, (n, seed, prec) in enumerate([(400000, 31, A.PREC_FP64), (150000, 32, A.PREC_FP64),
                                            (150000, 33, A.PREC_FP32)]):
        r, k = seeded_rays(n, EXT, seed=seed, disk=(4 * KPC, 0.35 * KPC))
        o_ref, c_ref, d_ref = ctx.trace_paths(r, k, prec)
        tot = int(o_ref[-1])
        o, c, d, dfree = _noalloc(ctx, r, k, tot + 1000, prec, stream)
        ctx.sync()
        assert np.array_equal(o, o_ref), call
        assert np.array_equal(c[:tot], c_ref), call
        assert np.array_equal(d[:tot], d_ref), call
        assert np.all(c[tot:] == -7) and np.all(d[tot:] == -7.0)
        if call > 0:   # kernels are loaded by now: the call itself takes no device memory
            assert dfree == 0, dfree
    ctx.close()


def test_noalloc_limits():
    ctx = _ctx()
    stream = torch.cuda.Stream()
    r, k = seeded_rays(5000, EXT, seed=41, disk=(4 * KPC, 0.35 * KPC))
    o_ref, _, _ = ctx.trace_paths(r, k, A.PREC_FP64)
    tot = int(o_ref[-1])
    # too small an output: the writes stop at the capacity, the needed total is reported
    o, c, d, _ = _noalloc(ctx, r, k, tot // 2, A.PREC_FP64, stream)
    with pytest.raises(A.SkirtError) as e:
        ctx.sync()
    assert e.value.code == A.SKG_ERR_CAPACITY
    assert np.array_equal(o, o_ref)
    # more rays than the static scratch holds: rejected before any work is enqueued
    with pytest.raises(A.SkirtError) as e:
        ctx.trace_paths_noalloc(0, 0, runtime.Context.NOALLOC_MAX_RAYS + 1, 0, 0, 1, 0, A.PREC_FP64, None)
    assert e.value.code == A.SKG_ERR_CAPACITY and "maximum" in str(e.value)
    # no rays: offsets[0] = 0
    o, _, _, _ = _noalloc(ctx, r[:0], k[:0], 0, A.PREC_FP64, stream)
    assert o.tolist() == [0]
    ctx.sync()
    ctx.close()


def test_noalloc_at_the_maximum_ray_count():
    """n = SKG_NOALLOC_MAX_RAYS: the scan of the block totals runs at its full width (1024
    blocks of 1024 rays); the offsets, cells and lengths equal skg_trace_paths' on a small grid."""
    ctx = _ctx(N=(16, 16, 8))
    stream = torch.cuda.Stream()
    n = runtime.Context.NOALLOC_MAX_RAYS
    r, k = seeded_rays(n, EXT, seed=51, disk=(4 * KPC, 0.35 * KPC))
    o_ref, c_ref, d_ref = ctx.trace_paths(r, k, A.PREC_FP64)
    tot = int(o_ref[-1])
    o, c, d, _ = _noalloc(ctx, r, k, tot, A.PREC_FP64, stream)
    ctx.sync()
    assert np.array_equal(o, o_ref)
    assert np.array_equal(c[:tot], c_ref) and np.array_equal(d[:tot], d_ref)
    ctx.close()


def test_noalloc_keeps_the_phase_flags():
    """A phase whose packets ran out of their step budget (max_steps = 1) flags the context; a
    no-alloc path call made afterwards finishes that phase first and keeps its flag, so skg_sync
    still reports the phase's failure; the path call itself succeeds and its results are right."""
    ctx = _ctx(N=(20, 20, 10))
    stream = torch.cuda.Stream()
    ctx.run_phase(A.PHASE_STELLAR, [0], 20000, 0, 20000, seed=5, max_steps=1)
    r, k = seeded_rays(3000, EXT, seed=61)
    o_ref, c_ref, d_ref = ctx.trace_paths(r, k, A.PREC_FP64)
    tot = int(o_ref[-1])
    o, c, d, _ = _noalloc(ctx, r, k, tot, A.PREC_FP64, stream)
    with pytest.raises(A.SkirtError) as e:
        ctx.sync()
    assert e.value.code == A.SKG_ERR_STEP_BUDGET
    assert np.array_equal(o, o_ref) and np.array_equal(c[:tot], c_ref) and np.array_equal(d[:tot], d_ref)
    # an unknown precision is rejected before any work is enqueued (real buffers, so that only
    # the precision is wrong)
    dr = torch.from_numpy(np.ascontiguousarray(r[:10])).cuda()
    dk = torch.from_numpy(np.ascontiguousarray(k[:10])).cuda()
    cells = torch.zeros(4096, dtype=torch.int32, device="cuda")
    ds = torch.zeros(4096, dtype=torch.float64, device="cuda")
    off = torch.zeros(11, dtype=torch.int64, device="cuda")
    with pytest.raises(A.SkirtError) as e:
        ctx.trace_paths_noalloc(dr.data_ptr(), dk.data_ptr(), 10, cells.data_ptr(), ds.data_ptr(), off.data_ptr(),
                                4096, 7, None)
    assert e.value.code == A.SKG_ERR_INVALID and "precision" in str(e.value)
    ctx.close()
