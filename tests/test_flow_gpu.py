"""GPU: the device-resident SSPRK2 + HEM step driver (plain launches and the
captured CUDA graph) against the CPU restatement of the reference RK driver over
the reference's own transport and flash, on a small N2O impingement cube with
a liquid inlet, viscosity, conduction and WALE. Per-field relative error of
rho, momentum, total energy, p and T after several steps, plus conservation
against the boundary ledger."""
import numpy as np
import pytest

from spuma_multiphysics_b200 import cases, thermo_data as td
from spuma_multiphysics_b200.flow import Flow, FlowError, field_errors
import rk_oracle

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-9


def small_case(n=12):
    faces, volume = cases.cartesian_faces(n, edge=n * 1e-3, port_diameter=0.005, port_z=n * 0.5e-3,
                                          port_offset=0.004)
    init = cases.impingement(n, seed=11)
    return faces, volume, init


@pytest.mark.parametrize("graph", [False, True])
def test_flow_matches_reference_rk_driver(graph):
    n, steps, dt = 12, 3, 1e-8
    faces, volume, init = small_case(n)
    assert (faces["kind"] == 3).sum() > 0
    kw = dict(viscosity=1.821e-5, conductivity=0.02587, wale_cw=0.325)
    flow = Flow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"], **kw)
    ref = rk_oracle.ReferenceFlow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"],
                                  image=td.model_bytes(td.pure_model()), **kw)
    mass0 = (init["q"] * volume[:, None]).sum(axis=0)
    ledger = np.zeros(5)
    for _ in range(steps):
        flow.step(dt, graph=graph)
        ref.step(dt)
        ledger += ref.boundary
    flow.check(dt)
    q, s = flow.conserved(), flow.states()
    rel = lambda a, b, scale: float(np.max(np.abs(a - b)) / scale)
    assert rel(q[:, 0], ref.q[:, 0], ref.q[:, 0].max()) < FIELD_TOL
    assert rel(q[:, 1:4], ref.q[:, 1:4], max(1.0, np.abs(ref.q[:, 1:4]).max())) < 1e-7
    assert rel(q[:, 4], ref.q[:, 4], np.abs(ref.q[:, 4]).max()) < FIELD_TOL
    assert rel(s["p"], ref.states["p"], ref.states["p"].max()) < FIELD_TOL
    assert rel(s["T"], ref.states["T"], ref.states["T"].max()) < FIELD_TOL
    # conservation: change of the integrals equals minus the boundary ledger
    mass = (q * volume[:, None]).sum(axis=0)
    assert abs((mass[0] - mass0[0]) + ledger[0]) <= 1e-10 * mass0[0]
    assert abs((mass[4] - mass0[4]) + ledger[4]) <= 1e-10 * abs(mass0[4])
    ref.close()
    flow.close()


def test_mixed_precision_flow_against_fp64():
    """FP32 gradients/WALE/fluxes with compensated sums against the FP64 path
    (itself matched to the reference RK driver above): per-field error after 10
    steps, and the mixed run conserves against its own ledger."""
    n, steps, dt = 16, 10, 1e-8
    faces, volume, init = small_case(n)
    kw = dict(viscosity=1.821e-5, conductivity=0.02587, wale_cw=0.325)
    fp64 = Flow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"], **kw)
    mixed = Flow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"], precision="mixed",
                 **kw)
    mass0 = (init["q"] * volume[:, None]).sum(axis=0)
    ledger = np.zeros(5)
    for _ in range(steps):
        fp64.step(dt)
        mixed.step(dt)
        ledger += mixed.ledger(dt)
    fp64.check(dt)
    mixed.check(dt)
    q, s = mixed.conserved(), mixed.states()
    errors = field_errors(q, s, fp64.conserved(), fp64.states())
    # p and T within 1e-6 (and the other positive fields)
    assert max(errors[k] for k in ("rho", "rhoE", "p", "T")) < 1e-6, errors
    # momentum scaled by its own (small, the flow starts at rest) maximum: the
    # FP32 pressure-flux differences of the 40 bar background set its error
    assert max(errors[k] for k in ("rhoU", "rhoV", "rhoW")) < 1e-5, errors
    assert errors["rho"] > 0  # the mixed form does differ from FP64
    mass = (q * volume[:, None]).sum(axis=0)
    assert abs((mass[0] - mass0[0]) + ledger[0]) <= 1e-10 * mass0[0]
    assert abs((mass[4] - mass0[4]) + ledger[4]) <= 1e-10 * abs(mass0[4])
    fp64.close()
    mixed.close()


def test_autotune_keeps_results():
    """The autotuner changes launch shapes only: a tuned flow reproduces the
    untuned one's states bit for bit."""
    n, steps, dt = 12, 2, 1e-8
    faces, volume, init = small_case(n)
    kw = dict(viscosity=1.821e-5, conductivity=0.02587, wale_cw=0.325)
    runs = []
    for tune in (False, True):
        flow = Flow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"], **kw)
        if tune:
            chosen = flow.autotune()
            assert chosen["stage_block"] in (0, 1, 64, 96, 128) and chosen["flash_blocks_per_sm"] >= 1
        for _ in range(steps):
            flow.step(dt)
        flow.check(dt)
        runs.append((flow.conserved(), flow.states()))
        flow.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1].view(np.uint8), runs[1][1].view(np.uint8))


def _case_flow(n=12, **extra):
    faces, volume, init = small_case(n)
    kw = dict(viscosity=1.821e-5, conductivity=0.02587, wale_cw=0.325)
    kw.update(extra)
    return Flow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"], **kw)


def test_advance_halves_dt_until_the_step_is_admitted():
    """A step 3.2 times the CFL step fails (CFL, and recoveries of the wrecked
    stage states), is rolled back to the step-start state and retried with dt/2
    and dt/4 (the reference driver's retry loop, ReactiveFoam.C:1434-1494); the
    accepted step equals a direct step of dt/4 bit for bit."""
    import torch
    probe = _case_flow()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert probe.lib.reactive_transport_stable_step_device_v3(probe.transport, probe.qn.data_ptr(),
                                                              probe.tr.data_ptr(), probe.cfl, 1.0, out.data_ptr(),
                                                              probe.stream.cuda_stream) == 0
    probe.stream.synchronize()
    cfl = out.item()
    probe.close()
    assert 0 < cfl < 1e-6
    big = 3.2 * cfl
    flow, ref = _case_flow(), _case_flow()
    try:
        taken = flow.advance(big)
        assert taken == big / 4
        assert flow.retries == 2 and flow.steps == 1
        assert "CFL" in flow.last_failure or "recovery" in flow.last_failure
        ref.step(big / 4, graph=False)
        ref.check(big / 4)
        assert np.array_equal(flow.conserved(), ref.conserved())
        assert flow.states().tobytes() == ref.states().tobytes()
        # an admitted step is taken once, with no retry
        assert flow.advance(big / 4) == big / 4 and flow.retries == 2 and flow.steps == 2
    finally:
        flow.close()
        ref.close()


def test_advance_gives_up_after_the_retries_and_restores_the_step_start():
    """One cell whose conserved energy no state can recover (set on the host
    before the step) fails every attempt: after 12 halvings FlowError is raised
    and the conserved and thermodynamic states are the step-start ones again."""
    import torch
    flow = _case_flow()
    try:
        c = 5
        flow.qn[4, c] = -1e12  # internal energy far below any PR state: the recovery fails
        torch.cuda.synchronize()
        q0, s0 = flow.conserved(), flow.states().copy()
        with pytest.raises(FlowError, match="retries"):
            flow.advance(1e-9, max_retries=12)
        assert flow.retries == 12
        assert "recovery failed" in flow.last_failure
        assert np.array_equal(flow.conserved(), q0)
        assert flow.states().tobytes() == s0.tobytes()
        assert flow.steps == 0
    finally:
        flow.close()
