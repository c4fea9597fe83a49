"""GPU: the work-queue flash's two-phase admissibility bound. Skipping the
two-phase seeds of cells outside every (widened) saturation tie line must not
change a single bit of any result: states, success flags and the transport
states equal those of the exhaustive search on the synthetic batch, on states
placed just inside and just outside the saturation dome, and on the impingement
flow's cells; the bound skips the ambient gas's seeds."""
import ctypes as C

import numpy as np
import pytest
import torch

from spuma_multiphysics_b200 import _abi as A, _lib, cases
from spuma_multiphysics_b200.eos import PureFluid
from spuma_multiphysics_b200.hem import GpuHem
from spuma_multiphysics_b200.thermo_data import N2O

pytestmark = pytest.mark.gpu


def bound(hem, request):
    active = C.c_int(-1)
    err = C.create_string_buffer(256)
    assert _lib.load().reactive_gpu_hem_two_phase_bound_v3(hem.handle, request, C.byref(active), err,
                                                            len(err)) == 0, err.value
    return active.value


def flash(hem, rho, e, guess):
    n = len(rho)
    cons = torch.zeros((5, n), dtype=torch.float64, device="cuda")
    cons[0] = torch.from_numpy(np.ascontiguousarray(rho)).cuda()
    cons[4] = torch.from_numpy(np.ascontiguousarray(e)).cuda()
    seed = torch.from_numpy(guess.view(np.uint8).copy()).cuda()
    state = torch.zeros_like(seed)
    tr = torch.zeros((n, 7), dtype=torch.float64, device="cuda")
    ok = torch.zeros(n, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    hem.counters(s)
    hem.run_device(cons, n, n, 5, seed, state, tr, ok, s)
    prof = hem.counters(s)
    return state.cpu().numpy().tobytes(), tr.cpu().numpy().tobytes(), ok.cpu().numpy(), prof


def both(rho, e, guess):
    hem = GpuHem(capacity=len(rho))
    try:
        assert bound(hem, -1) == 1  # on by default for the pure fluid
        on = flash(hem, rho, e, guess)
        assert bound(hem, 0) == 0
        off = flash(hem, rho, e, guess)
        assert bound(hem, 1) == 1
    finally:
        hem.close()
    return on, off


def assert_same(on, off):
    assert on[0] == off[0] and on[1] == off[1]
    assert np.array_equal(on[2], off[2])
    assert on[3].flashCandidates == off[3].flashCandidates
    assert on[3].stableCandidates == off[3].stableCandidates


def test_bound_keeps_the_synthetic_batch_bitwise():
    rho, e, guess = cases.flash_batch(60000, seed=4242)[:3]
    on, off = both(rho, e, guess)
    assert_same(on, off)
    assert on[3].phaseEvaluations < off[3].phaseEvaluations


def test_bound_keeps_states_at_the_dome_edge_bitwise():
    """Saturated vapour and liquid states moved in specific volume and energy by
    relative steps from 1e-9 to 3e-2 both ways, seeded by the saturation state:
    inside, on and outside the dome."""
    fluid = PureFluid(N2O)
    T = np.linspace(200.0, 308.0, 61)
    ps, gas, liq = fluid.saturation(T)
    steps = np.concatenate([-np.logspace(-9, -1.5, 12), [0.0], np.logspace(-9, -1.5, 12)])
    rho, e, seeds = [], [], []
    for side in (gas, liq):
        for dv in steps:
            for du in steps:
                v = (1 / side["rho"]) * (1 + dv)
                u = side["e"] * (1 + du)
                rho.append(1 / v)
                e.append(u / v)
                g = np.zeros(len(T), dtype=A.THERMO_DTYPE)
                g["p"], g["T"], g["rho"] = ps, T, 1 / v
                seeds.append(g)
    rho, e, guess = np.concatenate(rho), np.concatenate(e), np.concatenate(seeds)
    on, off = both(rho, e, guess)
    assert_same(on, off)


def test_bound_keeps_states_near_the_critical_point_and_the_table_ends_bitwise():
    """Single-phase states on both branches at pressures from 1e-9 to 1e-2 of
    the saturation pressure on either side, at temperatures up to 0.1 K below
    the critical point (305-309.4 K, where the tie lines collapse) and at the
    saturation table's cold end (the liquid range's lower end, 148 K, and just
    above it), seeded at their own (p, T): with the bound on (and with it the
    saturation-table stability shortcut) every bit equals the exhaustive
    search's."""
    fluid = PureFluid(N2O)
    T = np.concatenate([[148.0, 148.0 + 1e-6, 148.01, 148.5, 150.0], np.linspace(305.0, 309.4, 12)])
    ps, _, _ = fluid.saturation(T)
    ps = np.where(T > 308.0, 7.2446e6, ps)  # above 308 K: about the critical pressure
    offsets = np.concatenate([-np.logspace(-9, -2, 8), [0.0], np.logspace(-9, -2, 8)])
    rho, e, seeds = [], [], []
    for root in ("gas", "liquid"):
        for d in offsets:
            p = ps * (1 + d)
            props = fluid.tp(T, p, root=root)
            ok = np.isfinite(props["rho"]) & np.isfinite(props["e"]) & (props["rho"] > 0)
            rho.append(props["rho"][ok])
            e.append(props["rho"][ok] * props["e"][ok])
            g = np.zeros(int(ok.sum()), dtype=A.THERMO_DTYPE)
            g["p"], g["T"], g["rho"] = p[ok], T[ok], props["rho"][ok]
            seeds.append(g)
    rho, e, guess = np.concatenate(rho), np.concatenate(e), np.concatenate(seeds)
    assert len(rho) > 400
    on, off = both(rho, e, guess)
    assert_same(on, off)


def test_bound_keeps_the_impingement_flash_bitwise():
    from spuma_multiphysics_b200.flow import Flow
    n = 24
    faces, volume = cases.cartesian_faces(n, edge=n * 1e-3, port_diameter=0.005, port_z=n * 0.5e-3,
                                          port_offset=0.004)
    init = cases.impingement(n, seed=7)
    flow = Flow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"])
    try:
        for _ in range(3):
            flow.step(1e-8)
        flow.check(1e-8)
        q = flow.qn[:, :flow.cells].cpu().numpy()
        rho = q[0]
        e = q[4] - .5 * (q[1:4] ** 2).sum(0) / q[0]
        guess = flow.states()
    finally:
        flow.close()
    on, off = both(rho, e, guess)
    assert_same(on, off)
    # the ambient gas's two-phase seeds are skipped: most of the evaluations go
    assert on[3].phaseEvaluations < .5 * off[3].phaseEvaluations
