"""Failure detection through the C ABI, every failure injected on the host and every wait bounded
(the reference throws FatalError at these points; here a status code comes back and the context
stays usable):

  * a NaN cell density is rejected when the scene is set up (SKG_ERR_INVALID); a finite density
    whose optical depth overflows makes the optical depth along a path not a positive number
    (DustSystem.cpp:953-955) -> SKG_ERR_NAN_TAU from skg_sync, no hang;
  * a traversal step budget of one cell (skg_run_opts.max_steps = 1) -> SKG_ERR_STEP_BUDGET, and
    the next phase with the default budget succeeds on the same context;
  * skg_sync with a zero timeout while a phase runs -> SKG_ERR_TIMEOUT; a later skg_sync
    completes the phase;
  * a packet pool larger than the device -> SKG_ERR_OOM, the context still runs phases; more work
    items than a batch holds -> SKG_ERR_CAPACITY."""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import models, runtime

from helpers import cell_center_density

pytestmark = pytest.mark.gpu


def _model(N=(20, 20, 10)):
    m = models.oligo_disk(N=N, npix=32)
    m.rho = cell_center_density(m)
    return m


def test_nan_density_is_rejected_at_setup():
    m = _model()
    m.rho[0, ::7] = np.nan
    with pytest.raises(A.SkirtError) as e:
        runtime.Context(m)
    assert e.value.code == A.SKG_ERR_INVALID and "finite" in str(e.value)


@pytest.mark.parametrize("precision", [A.PREC_FP32, A.PREC_FP64])
def test_overflowing_optical_depth_is_reported(precision):
    """Finite densities whose optical depth overflows (kappa rho ds = inf): the path's optical
    depth is not a positive number (DustSystem.cpp:953-955) -> SKG_ERR_NAN_TAU, no hang; the device
    is unaffected."""
    m = _model()
    m.rho[0, ::7] = 1e300
    ctx = runtime.Context(m)
    ctx.run_phase(A.PHASE_STELLAR, [0], 20000, 0, 20000, seed=3, precision=precision)
    with pytest.raises(A.SkirtError) as e:
        ctx.sync(60000)
    assert e.value.code == A.SKG_ERR_NAN_TAU
    assert ctx.counters()["errors"] > 0
    ctx.close()
    ok = runtime.Context(_model())
    ok.run_phase(A.PHASE_STELLAR, [0], 20000, 0, 20000, seed=3, precision=precision)
    ok.sync(60000)
    assert ok.counters()["errors"] == 0
    ok.close()


def test_step_budget_is_reported_and_cleared_by_the_next_phase():
    ctx = runtime.Context(_model())
    ctx.run_phase(A.PHASE_STELLAR, [0], 20000, 0, 20000, seed=4, max_steps=1)
    with pytest.raises(A.SkirtError) as e:
        ctx.sync(60000)
    assert e.value.code == A.SKG_ERR_STEP_BUDGET
    assert ctx.counters()["errors"] > 0
    ctx.reset_tallies()
    ctx.run_phase(A.PHASE_STELLAR, [0], 20000, 0, 20000, seed=4)
    ctx.sync(60000)
    c = ctx.counters()
    assert c["errors"] == 0 and c["packets"] == 20000
    ctx.close()


def test_zero_timeout_sync_then_completion():
    m = models.oligo_disk(npix=64)                 # configuration 1's grid: a phase of 10^7 packets
    m.rho = cell_center_density(m)                 # takes about 0.1 s
    ctx = runtime.Context(m)
    npp = 10_000_000
    ctx.run_phase(A.PHASE_STELLAR, [0], npp, 0, npp, seed=5)
    with pytest.raises(A.SkirtError) as e:
        ctx.sync(0)
    assert e.value.code == A.SKG_ERR_TIMEOUT
    ctx.sync(120000)
    c = ctx.counters()
    assert c["packets"] == npp and c["errors"] == 0
    ctx.close()


def test_oversized_requests():
    ctx = runtime.Context(_model())
    # 2^31 - 1 packets in flight would need 256 GiB of packet records
    n = 2 ** 31
    with pytest.raises(A.SkirtError) as e:
        ctx.run_phase(A.PHASE_STELLAR, [0], n, 0, n, seed=6, pool=2 ** 31 - 1)
    assert e.value.code == A.SKG_ERR_OOM
    ctx.run_phase(A.PHASE_STELLAR, [0], 20000, 0, 20000, seed=6)
    ctx.sync(60000)
    assert ctx.counters()["packets"] == 20000
    b = runtime.Batch(max_slots=2, max_items=2, max_ells=8)
    with pytest.raises(A.SkirtError) as e:
        b.run(A.PHASE_STELLAR, [(ctx, [0], 1000, 0, 1000, s) for s in range(3)])
    assert e.value.code == A.SKG_ERR_CAPACITY
    b.run(A.PHASE_STELLAR, [(ctx, [0], 1000, 0, 1000, s) for s in range(2)])
    b.sync(60000)
    b.close()
    ctx.close()
