"""GPU: the z-slab decomposition of the impingement box against the undivided
box. Every slab of a 24^3 box (viscous + conduction + WALE) runs on one device
with the halo exchange as device copies; after three SSPRK2 + HEM steps every own
cell's conserved state, thermo state and transport state equal the undivided
run's bit for bit, the CFL minimum over slabs equals the undivided one, and the
slabs' ledgers sum to the undivided ledger (a different summation order)."""
import numpy as np
import pytest
import torch

from spuma_multiphysics_b200 import cases
from spuma_multiphysics_b200.flow import Flow
from spuma_multiphysics_b200.slab import LocalSlabs

pytestmark = pytest.mark.gpu

N = 24
EDGE = N * 1e-3
PORTS = dict(port_diameter=0.005, port_z=N * 0.5e-3, port_offset=0.004)
VISCOUS = dict(viscosity=1.821e-5, conductivity=0.02587, wale_cw=0.325)


@pytest.mark.parametrize("world,extra", [
    (2, dict(precision="fp64")),
    (3, dict(precision="mixed")),
    (4, dict(precision="fp64", flux="hllc")),
    (2, dict(precision="mixed", turbulent_prandtl=0.9, turbulent_schmidt=0.7)),
])
def test_slabs_match_the_undivided_box_bitwise(world, extra):
    init = cases.impingement(N, seed=7)
    faces, volume = cases.cartesian_faces(N, edge=EDGE, **PORTS)
    kw = dict(VISCOUS, **extra)
    whole = Flow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"], **kw)
    slabs = LocalSlabs(N, world, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"], edge=EDGE,
                       ports=PORTS, **kw)
    try:
        dt = 1e-8
        for step in range(3):
            whole.step(dt)
            slabs.step(dt, graph=step % 2 == 0)  # captured halves and plain launches
        whole.check(dt)
        cfl = slabs.check(dt)["cfl_dt"]
        q, s, tr = slabs.gather()
        assert torch.equal(q, whole.qn[:, :whole.cells])
        assert torch.equal(s, whole.sn)
        assert torch.equal(tr, whole.tr[:whole.cells])
        assert cfl == whole.dt_cfl.min().item()
        ledger, ref = slabs.ledger(dt), whole.ledger(dt)
        assert np.allclose(ledger, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    finally:
        whole.close()
        slabs.close()
