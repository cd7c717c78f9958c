"""The continuous-batching request loop (vah_serve_run) on a small stream:
every request is admitted, advanced while others arrive and run, retired at
freeze-out, and timed."""
import numpy as np
import pytest

import vahlib as V

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ic_on_device", [1, 0], ids=["device_ic", "host_ic"])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_serve_small_stream_completes_every_request(precision, ic_on_device):
    res, lat = V.product.serve(rate=40.0, duration_s=1.0, seed=5, frac_3d=0.3, side2_min=21, side2_max=41,
                               side3_min=15, side3_max=21, nz3_min=5, nz3_max=9, dx=0.5, deta=0.3, b_max=10.0,
                               dt=0.05, T0_GeV=0.30, Tf_GeV=0.15, t_max=30.0, precision=precision,
                               capacity_bytes=4 << 30, chunk_steps=5, ic_threads=4, ic_on_device=ic_on_device)
    assert res["offered"] > 10
    assert res["completed"] == res["offered"] and res["timeouts"] == 0 and res["rejected"] == 0
    assert res["failed"] == 0 and 0 < res["tau_freeze_max"] < 30.0
    assert np.all(lat > 0) and res["p99_s"] >= res["p50_s"] > 0
    assert res["max_resident"] > 1  # requests overlapped on the device
    assert res["events_per_s"] > 0 and res["cell_updates"] > 0
