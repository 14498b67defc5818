"""The C ABI server (skg_server_create / skg_submit / skg_poll, skirt7_b200/csrc/skg_serve.cpp):
fit variants submitted together are admitted, batched into ticks and retired by the native
loop; every request's frame equals the same simulation run alone on the plain single-simulation
path (skg_run_phase over all its packets) up to the order of the FP64 tally additions -- alone and
in the mix give the same result; a tight device-memory budget still serves every request."""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import serving

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("budget", [0, 64 << 20])
def test_native_server_equals_alone(budget):
    reqs = serving.fitskirt_requests(n=10, rate=0.0, seed=77, packets=(1e5, 6e5), grid=(32, 64))
    srv = serving.NativeServer(hbm_budget=budget, max_slots=8, tick_packets=1 << 17, tick_budget=3 << 18)
    ids = [srv.submit(serving.build_model(r, 64), [0, 1, 2], r.packets, r.seed) for r in reqs]
    got = [srv.poll(i, 300000) for i in ids]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs) and st["ticks"] >= 2
    assert st["packets"] == 3 * sum(r.packets for r in reqs)
    for r, (cube, sed, lat) in zip(reqs, got):
        alone, _ = serving.run_alone(r, npix=64)
        assert alone.sum() > 0 and lat > 0
        assert np.allclose(cube[0], alone, rtol=1e-9, atol=1e-12 * alone.max()), r.rid
    # an id is reported once
    with pytest.raises(A.SkirtError):
        srv2 = serving.NativeServer()
        try:
            srv2.poll(12345, 0)
        finally:
            srv2.close()
