"""GPU: the hand-written adjoint of the SSPRK2 step (ideal-gas box, inviscid
HLL, structured path) against the plain PyTorch reference step differentiated by
autograd, checkpointed rollouts against uncheckpointed ones, and gradients of a
small blast-box loss against FP64 central finite differences."""
import numpy as np
import pytest
import torch

from spuma_multiphysics_b200 import cases, thermo_data as td
from spuma_multiphysics_b200.adjoint import IdealGasBox, SSPRK2Step, rollout
import torch_step as TS
from test_torch_step import DIMS, H, KINDS, SPECIES, random_state

pytestmark = pytest.mark.gpu


def scaled(a, b):
    scale = np.maximum(np.abs(b).max(axis=1, keepdims=True), 1e-300)
    return float(np.max(np.abs(a - b) / scale))


@pytest.fixture(scope="module")
def box():
    faces, volume = cases.box_faces(DIMS, H, KINDS)
    b = IdealGasBox(faces, volume, SPECIES)
    yield b
    b.close()


def test_step_matches_torch_reference(box):
    q, _ = random_state(DIMS, seed=5)
    qd = torch.from_numpy(q).cuda()
    dt = .3 * box.stable_dt(qd)
    got, _ = box.forward_step(qd, dt)
    box.check()
    exp = TS.step(torch.from_numpy(q), dt, DIMS, H, KINDS, SPECIES).numpy()
    assert scaled(got.cpu().numpy(), exp) < 1e-12


def test_step_vjp_matches_autograd(box):
    q, _ = random_state(DIMS, seed=6)
    qd = torch.from_numpy(q).cuda()
    dt = .3 * box.stable_dt(qd)
    lam = np.random.default_rng(7).normal(size=q.shape) * np.abs(q).max(axis=1, keepdims=True) ** -1
    _, saved = box.forward_step(qd, dt)
    got = box.step_vjp(torch.from_numpy(lam).cuda(), saved, dt).cpu().numpy()
    box.check()
    qt = torch.from_numpy(q).requires_grad_(True)
    out = TS.step(qt, dt, DIMS, H, KINDS, SPECIES)
    (exp,) = torch.autograd.grad(out, qt, torch.from_numpy(lam))
    assert scaled(got, exp.numpy()) < 1e-9


def test_autograd_function_and_checkpointing(box):
    q, _ = random_state(DIMS, seed=8)
    dt = .2 * box.stable_dt(torch.from_numpy(q).cuda())
    w = torch.from_numpy(np.random.default_rng(9).normal(size=q.shape)).cuda()
    grads = []
    for every in (5, 100):
        qd = torch.from_numpy(q).cuda().requires_grad_(True)
        out = rollout(box, qd, 12, dt, checkpoint_every=every)
        (g,) = torch.autograd.grad((out * w).sum(), qd)
        grads.append(g.cpu().numpy())
    box.check()
    assert scaled(grads[0], grads[1]) < 1e-12
    # one step through the autograd.Function equals the direct VJP
    qd = torch.from_numpy(q).cuda().requires_grad_(True)
    (g1,) = torch.autograd.grad((SSPRK2Step.apply(qd, box, dt) * w).sum(), qd)
    _, saved = box.forward_step(torch.from_numpy(q).cuda(), dt)
    assert torch.equal(g1, box.step_vjp(w, saved, dt))


def test_blast_gradient_against_finite_differences():
    n, steps, every = 16, 12, 4
    spec = cases.blast_box(n, edge=n * 1e-3, radius=4e-3)
    b = IdealGasBox(spec["faces"], spec["volume"], spec["species"])
    try:
        rho0 = torch.from_numpy(spec["rho0"]).cuda()
        p_drive = torch.tensor(spec["p_drive"], dtype=torch.float64, device="cuda")
        q0 = cases.blast_initial(spec, rho0, p_drive, xp=torch)
        dt = .3 * b.stable_dt(q0)
        k, j, i = np.indices((n, n, n))
        sub = ((i >= 9) & (i < 13) & (j >= 6) & (j < 10) & (k >= 6) & (k < 10)).ravel()
        mask = torch.from_numpy(sub.astype(np.float64)).cuda() * b.volume

        def loss(r, p):
            return (rollout(b, cases.blast_initial(spec, r, p, xp=torch), steps, dt, every)[0] * mask).sum()

        r = rho0.clone().requires_grad_(True)
        p = p_drive.clone().requires_grad_(True)
        g_rho, g_p = torch.autograd.grad(loss(r, p), (r, p))
        b.check()
        rng = np.random.default_rng(11)
        # probes within the loss sub-box's domain of dependence (12 steps)
        near = np.flatnonzero((i >= 6) & (i < 16) & (j >= 3) & (j < 13) & (k >= 3) & (k < 13))
        probes = rng.choice(near, 8, replace=False)

        def central(c, rel):
            h = rel * float(rho0[c])
            rp, rm = rho0.clone(), rho0.clone()
            rp[c] += h
            rm[c] -= h
            return (loss(rp, p_drive) - loss(rm, p_drive)).item() / (2 * h)

        with torch.no_grad():
            g = g_rho[probes].cpu().numpy()
            fd6 = np.array([central(c, 1e-6) for c in probes])
            fd4 = np.array([central(c, 1e-4) for c in probes])
            hp = 1e-6 * spec["p_drive"]
            fd_p = (loss(rho0, p_drive + hp) - loss(rho0, p_drive - hp)).item() / (2 * hp)
        b.check()
        # h = 1e-6 (relative): the loss moves by ~1e-14 of itself, so round-off
        # bounds each difference; compare on the scale of the largest gradient
        assert np.max(np.abs(g - fd6)) <= 1e-4 * np.max(np.abs(fd6)), (g, fd6)
        # h = 1e-4: truncation O(h^2), relative agreement on every probe that
        # carries signal
        big = np.abs(fd4) > 1e-3 * np.max(np.abs(fd4))
        assert np.max(np.abs(g - fd4)[big] / np.abs(fd4[big])) < 1e-4, (g, fd4)
        # the driver pressure aggregates all sphere cells: relative 1e-6
        assert abs(g_p.item() - fd_p) <= 1e-6 * abs(fd_p)
    finally:
        b.close()
