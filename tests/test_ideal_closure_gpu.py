"""GPU: the ideal-gas closure (reactive_ideal_gas_run_device_v3) against the
reference's own CUDA scalar closure (src/reactiveTransport/reactiveClosureScalar.cuh,
built for sm_100a from the reference sources into oracle/_ref/libref_closure.so)
on the states of the 64^3 two-species blast box.

The reference closure takes per-cell inputs its host pool prepares
(src/reactiveThermo/reactiveClosurePool.inc:57-83): the mass fractions' mixture
of the NASA coefficients of the region holding the seed temperature, premixed
into one polynomial (src/reactiveThermo/reactiveCaloricFast.h:69-103), the
temperature interval of that region, and the specific internal energy. That
preparation is restated here on the host; this library's closure mixes the
species' own tables per cell on the device. Both recover T by the same
bracket-and-Newton steps to the same tolerance, so T, p and cv agree to
round-off wherever the reference's fixed-region interval admits the result.
"""
import numpy as np
import pytest
import torch

from oracle import oracle
from spuma_multiphysics_b200 import cases
from spuma_multiphysics_b200.adjoint import IdealGasBox
from spuma_multiphysics_b200.thermo_data import GAS_CONSTANT

pytestmark = pytest.mark.gpu

TOL = 1e-12


def reference_inputs(q, species, T_seed, Tmin, Tmax, tolerance):
    """ReactiveClosureScalarInputV1 records of conserved states q (nv, cells),
    as the reference pool prepares them for pr = 0; cells whose seed sits on a
    region boundary (the reference sends those to its CPU path) are disabled."""
    ns = len(species)
    n = q.shape[1]
    rho = q[:ns].sum(axis=0)
    Y = q[:ns] / rho
    m2 = q[ns] * q[ns] + q[ns + 1] * q[ns + 1] + q[ns + 2] * q[ns + 2]
    energy = (q[ns + 3] - .5 * m2 / rho) / rho
    inv_w = sum(Y[k] / sp["W"] for k, sp in enumerate(species))
    W = 1 / inv_w
    T = np.clip(np.full(n, float(T_seed)), Tmin, Tmax)
    rec = np.zeros(n, dtype=oracle.CLOSURE_IN_DTYPE)
    coeff = np.zeros((n, 8))
    lower, upper = np.full(n, float(Tmin)), np.full(n, float(Tmax))
    enabled = np.ones(n, dtype=bool)
    for k, sp in enumerate(species):
        active = Y[k] != 0
        bounds = sp["ranges"][1:-1]        # the minimum temperatures of regions 1..
        region = np.zeros(n, dtype=int)
        for j, b in enumerate(bounds, start=1):
            region = np.where(T >= b, j, region)    # NASA9: a region starts at its bound inclusive
        a = np.array(sp["nasa9"])[region]           # (n, 9)
        w = Y[k] * (GAS_CONSTANT / sp["W"])
        coeff += np.where(active[:, None], w[:, None] * a[:, :8], 0.0)
        for b in bounds:
            on = active & (T == b)
            enabled &= ~on
            below = active & (b < T)
            above = active & (b > T)
            lower = np.where(below, np.maximum(lower, np.nextafter(b, T)), lower)
            upper = np.where(above, np.minimum(upper, np.nextafter(b, T)), upper)
    rec["coeff"] = coeff
    rec["W"] = W
    rec["r"] = GAS_CONSTANT / W
    rec["rho"] = rho
    rec["energy"] = energy
    rec["T"] = T
    rec["lower"], rec["upper"] = lower, upper
    rec["tolerance"] = tolerance
    rec["pmin"], rec["pmax"] = 1e3, 5e7
    rec["pr"] = 0
    rec["enabled"] = enabled.astype(np.int32)
    return rec


def test_ideal_closure_matches_reference_closure_on_blast_box_states():
    n = 64
    spec = cases.blast_box(n, edge=n * 1e-3, radius=n * 0.25e-3)
    box = IdealGasBox(spec["faces"], spec["volume"], spec["species"])
    try:
        rho0 = torch.from_numpy(spec["rho0"]).cuda()
        p_drive = torch.tensor(spec["p_drive"], dtype=torch.float64, device="cuda")
        q = cases.blast_initial(spec, rho0, p_drive, xp=torch).contiguous()
        dt = .3 * box.stable_dt(q)
        compared = 0
        for step in range(51):
            if step in (0, 10, 25, 50):
                T, tr = box.closure(q)
                torch.cuda.synchronize()
                ok = box.success.cpu().numpy() != 0
                T, tr = T.cpu().numpy(), tr.cpu().numpy()
                qh = q.cpu().numpy()
                rec = reference_inputs(qh, spec["species"], float(box.T_guess[0]), 150.0, 3000.0, 1e-13)
                ref = oracle.ref_closure_run(rec)
                done = ref["success"] != 0
                # the reference converges in its seed's NASA region on (nearly) every cell,
                # and this closure converges wherever the reference does
                assert done.mean() > 0.999, (step, done.mean())
                assert ok[done].all(), step
                rel = lambda a, b: float(np.max(np.abs(a - b) / np.abs(b)))
                errors = {"T": rel(T[done], ref["T"][done]), "p": rel(tr[done, 0], ref["p"][done]),
                          "cv": rel(tr[done, 3], ref["cv"][done])}
                assert max(errors.values()) <= TOL, (step, errors)
                compared += int(done.sum())
            if step < 50:
                q, _ = box.forward_step(q, dt)
        box.check()
        assert compared > 4 * 0.999 * n ** 3
    finally:
        box.close()
