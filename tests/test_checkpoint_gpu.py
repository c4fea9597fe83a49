"""GPU: a device-resident step driver restarts from its own schema-3 checkpoint
exactly: the state after (save at step 2, restart, one step) equals the state of
the run that went on without stopping, bit for bit."""
import numpy as np
import pytest

from spuma_multiphysics_b200 import checkpoint as ck
from spuma_multiphysics_b200.flow import Flow
from test_flow_gpu import small_case

pytestmark = pytest.mark.gpu


def test_flow_restarts_from_checkpoint_bitwise(tmp_path):
    n, dt = 12, 1e-8
    faces, volume, init = small_case(n)
    kw = dict(viscosity=1.821e-5, conductivity=0.02587, wale_cw=0.325)
    args = (faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"])
    a = Flow(*args, **kw)
    b = Flow(*args, **kw)
    try:
        for _ in range(2):
            a.step(dt)
        a.check(dt)
        path = a.save_checkpoint(tmp_path, time=2 * dt, last_dt=dt)
        assert path.name == "2e-08"
        ck.verify(path)
        a.step(dt)
        hist = b.load_checkpoint(path)
        assert hist.steps == 2 and hist.last_dt == dt
        b.step(dt)
        b.check(dt)
        assert np.array_equal(a.conserved(), b.conserved())
        assert a.states().tobytes() == b.states().tobytes()
    finally:
        a.close()
        b.close()
