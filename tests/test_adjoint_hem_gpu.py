"""GPU: the adjoint pieces of the HEM step (config-5 physics) against finite
differences of the forward entries they differentiate:

* the viscous/conduction/WALE rate VJP (reactive_transport_rate_vjp_v3) by the
  dot-product test <w, dL v> = <L^T w, v> with dL v from central differences of
  the host-array RHS of the same operator (reactive_transport_rhs, which the
  structured path equals bitwise);
* the flash VJP by the implicit function theorem
  (reactive_gpu_hem_vjp_device_v3), cell by cell, against central differences
  of the flash's transport-state outputs;
* the whole SSPRK2 + HEM step adjoint (adjoint.HemStep) on a small impingement
  cube against central differences of the loss."""
import ctypes as C

import numpy as np
import pytest
import torch

from spuma_multiphysics_b200 import _abi as A, _lib, cases, thermo_data as td
from spuma_multiphysics_b200.adjoint import HemStep, hem_rollout
from spuma_multiphysics_b200.flow import Flow
from spuma_multiphysics_b200.hem import GpuHem
import transport_cases as T
from test_structured_gpu import box_case, mixed_kinds

pytestmark = pytest.mark.gpu

STATE_FIELDS = ("p", "T", "rho", "sound")


@pytest.mark.parametrize("ns,wale,kinds,viscous", [(1, .325, "mixed", True), (2, .5, (1, 2, 3, 2, 1, 2), True),
                                                   (1, None, (2,) * 6, True), (2, None, "mixed", False)])
def test_rate_vjp_dot_product(ns, wale, kinds, viscous):
    """viscous=False: the inviscid operator (the hand-derived reverse-mode HLL
    kernel); True: viscosity and conduction (the dual-number kernels)."""
    import torch
    L = _lib.load()
    lib = T.bind(L)
    dims = (6, 5, 4)
    kinds = mixed_kinds(dims, 23) if kinds == "mixed" else kinds
    case = box_case(dims, ns, kinds, viscous=viscous, conduction=viscous, seed=4)
    h = T.create(lib, 1, case, wale_cw=wale)
    nc, nv = case["nc"], case["nv"]
    rng = np.random.default_rng(31 + ns)
    try:
        q, st = case["q"], case["states"]

        def rhs(qq, ss):
            out, br = np.empty_like(qq), np.empty(nv)
            assert lib.reactive_transport_rhs(h, T.dp(np.ascontiguousarray(qq)), T.states_ptr(ss), None, None,
                                              T.dp(out), T.dp(br)) == 0, lib.reactive_transport_error(h)
            return out

        vq = rng.normal(size=q.shape) * np.abs(q).max(axis=0)
        vs = {f: rng.normal(size=nc) * np.abs(st[f]).max() * .1 for f in STATE_FIELDS}
        w = rng.normal(size=q.shape)
        eps = 1e-6
        sp, sm = st.copy(), st.copy()
        for f in STATE_FIELDS:
            sp[f] += eps * vs[f]
            sm[f] -= eps * vs[f]
        fd = float(np.sum(w * (rhs(q + eps * vq, sp) - rhs(q - eps * vq, sm)) / (2 * eps)))
        # the adjoint through the device entry
        cells, fixed, nvar, nsp = (C.c_size_t() for _ in range(4))
        assert L.reactive_transport_layout_v3(h, C.byref(cells), C.byref(fixed), C.byref(nvar), C.byref(nsp)) == 0
        all_ = nc + fixed.value
        stream = torch.cuda.current_stream().cuda_stream
        qd = torch.zeros((nv, all_), dtype=torch.float64, device="cuda")
        qd[:, :nc] = torch.from_numpy(q.T.copy()).cuda()
        sd = torch.zeros((all_, 7), dtype=torch.float64, device="cuda")
        sd[:nc] = torch.from_numpy(st.view(np.float64).reshape(nc, 7)).cuda()
        assert L.reactive_transport_fill_fixed_v3(h, qd.data_ptr(), sd.data_ptr(), stream) == 0
        wd = torch.from_numpy(w.T.copy()).cuda()
        q_bar = torch.empty((nv, nc), dtype=torch.float64, device="cuda")
        s_bar = torch.empty((nc, 7), dtype=torch.float64, device="cuda")
        assert L.reactive_transport_rate_vjp_v3(h, qd.data_ptr(), sd.data_ptr(), wd.data_ptr(), q_bar.data_ptr(),
                                                s_bar.data_ptr(), stream) == 0, lib.reactive_transport_error(h)
        torch.cuda.synchronize()
        qb = q_bar.cpu().numpy().T
        sb = s_bar.cpu().numpy().view(A.STATE_DTYPE).reshape(nc)
        adj = float(np.sum(qb * vq)) + sum(float(np.sum(sb[f] * vs[f])) for f in STATE_FIELDS)
        assert abs(adj - fd) <= 1e-6 * max(abs(fd), 1e-300), (adj, fd)
    finally:
        lib.reactive_transport_destroy(h)


def test_hem_vjp_against_cellwise_differences():
    n = 3000
    rho, e, guess = cases.flash_batch(n, seed=515)[:3]
    rng = np.random.default_rng(5)
    u = rng.normal(0, 20, (3, n))
    q = np.zeros((5, n))
    q[0], q[1:4], q[4] = rho, rho * u, e + .5 * rho * (u ** 2).sum(0)
    hem = GpuHem(capacity=n)
    seed = torch.from_numpy(guess.view(np.uint8).copy()).cuda()

    def flash(qq):
        cons = torch.from_numpy(np.ascontiguousarray(qq)).cuda()
        state = torch.zeros_like(seed)
        tr = torch.zeros((n, 7), dtype=torch.float64, device="cuda")
        ok = torch.zeros(n, dtype=torch.int32, device="cuda")
        hem.run_device(cons, n, n, 5, seed, state, tr, ok, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        return cons, state, tr.cpu().numpy(), ok.cpu().numpy()

    cons, state, tr0, ok0 = flash(q)
    scale = np.abs(tr0).max(axis=0)
    scale[scale == 0] = 1.0
    ybar = rng.normal(size=(n, 7)) / scale
    ybar[:, 6] = 0
    q_bar = torch.zeros((5, n), dtype=torch.float64, device="cuda")
    failed = torch.zeros(1, dtype=torch.int32, device="cuda")
    err = C.create_string_buffer(512)
    lib = _lib.load()
    assert lib.reactive_gpu_hem_vjp_device_v3(hem.handle, cons.data_ptr(), n, n, 5, state.data_ptr(),
                                              torch.from_numpy(ybar).cuda().data_ptr(), q_bar.data_ptr(), n,
                                              failed.data_ptr(), torch.cuda.current_stream().cuda_stream, err,
                                              len(err)) == 0, err.value
    torch.cuda.synchronize()
    assert failed.item() == 0
    # per-element directions: a relative perturbation of 1e-4 of each variable
    v = rng.normal(size=q.shape) * np.maximum(np.abs(q), 1e-3 * np.abs(q).max(axis=1, keepdims=True))
    eps = 1e-4
    _, sp, trp, okp = flash(q + eps * v)
    _, sm, trm, okm = flash(q - eps * v)
    labels = [cases.phase_label(x.cpu().numpy().view(A.THERMO_DTYPE)) for x in (state, sp, sm)]
    same = (ok0 != 0) & (okp != 0) & (okm != 0) & (labels[0] == labels[1]) & (labels[0] == labels[2])
    fd = np.sum(ybar * (trp - trm) / (2 * eps), axis=1)
    adj = np.sum(q_bar.cpu().numpy() * v, axis=0)
    scale = np.maximum(np.abs(fd), 1e-12 * np.abs(fd).max())
    rel = np.abs(adj - fd)[same] / scale[same]
    assert same.sum() > .97 * n
    assert np.median(rel) < 1e-5, np.median(rel)
    assert np.percentile(rel, 99) < 1e-3, np.percentile(rel, 99)
    hem.close()


def test_hem_step_gradient_against_finite_differences():
    n, steps, dt = 12, 2, 1e-8
    faces, volume = cases.cartesian_faces(n, edge=n * 1e-3, port_diameter=0.005, port_z=n * 0.5e-3,
                                          port_offset=0.004)
    init = cases.impingement(n, seed=11)
    flow = Flow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"], viscosity=1.821e-5,
                conductivity=0.02587, wale_cw=0.325)
    stepper = HemStep(flow)
    cells = flow.cells
    try:
        q0 = flow.qn.clone()
        s0 = flow.sn.clone()
        k, j, i = np.indices((n, n, n))
        sub = ((i >= 2) & (i < 6) & (j >= 2) & (j < 6) & (k >= 4) & (k < 8)).ravel()
        weight = torch.zeros_like(q0)
        weight[0, :cells] = torch.from_numpy(sub * volume).cuda()
        weight[4, :cells] = torch.from_numpy(sub * volume).cuda() * 1e-6

        def loss(q):
            # the rollout starts from the recovery of q itself
            s = stepper.recover(q.detach(), s0)
            out, _ = hem_rollout(stepper, q, s, steps, dt, checkpoint_every=1)
            return (out * weight).sum()

        qg = q0.clone().requires_grad_(True)
        (g,) = torch.autograd.grad(loss(qg), qg)
        stepper.check()
        rng = np.random.default_rng(3)
        probes = rng.choice(np.flatnonzero(sub), 6, replace=False)
        with torch.no_grad():
            for c in probes:
                for var in (0, 4):
                    h = 1e-6 * abs(float(q0[var, c]))
                    qp, qm = q0.clone(), q0.clone()
                    qp[var, c] += h
                    qm[var, c] -= h
                    fd = (loss(qp) - loss(qm)).item() / (2 * h)
                    got = g[var, c].item()
                    assert abs(got - fd) <= 2e-4 * abs(fd) + 1e-12 * abs(g[var]).max().item(), (c, var, got, fd)
        stepper.check()
    finally:
        flow.close()


@pytest.mark.parametrize("ns,wale,kinds,viscous", [(1, .325, "mixed", True), (2, None, (1, 2, 3, 2, 1, 2), False),
                                                   (3, .5, (3, 1, 1, 2, 2, 3), True)])
def test_hllc_rate_vjp_dot_product(ns, wale, kinds, viscous):
    """The HLLC operator's VJP (dual numbers through the templated face flux,
    star-side switches taken on the forward's branch) by the dot-product test
    against central differences of the oracle's HLLC right-hand side (the
    oracle's HLLC core equals the reference's bit for bit)."""
    from oracle import oracle
    L = _lib.load()
    lib = T.bind(L)
    dims = (6, 5, 4)
    kinds = mixed_kinds(dims, 23) if kinds == "mixed" else kinds
    case = box_case(dims, ns, kinds, viscous=viscous, conduction=viscous, seed=4)
    h = T.create(lib, 1, case, wale_cw=wale)
    nc, nv = case["nc"], case["nv"]
    rng = np.random.default_rng(37 + ns)
    cw = -1.0 if wale is None else wale
    oracle.set_flux_scheme(1)
    try:
        assert L.reactive_transport_flux_v3(h, 1, None) == 0
        q, st = case["q"], case["states"]

        def rhs(qq, ss):
            out, _, _, _, status = oracle.transport_rhs(case, np.ascontiguousarray(qq), ss.ctypes.data_as(C.c_void_p),
                                                        wale_cw=cw)
            assert status == 0
            return out

        vq = rng.normal(size=q.shape) * np.abs(q).max(axis=0)
        vs = {f: rng.normal(size=nc) * np.abs(st[f]).max() * .1 for f in STATE_FIELDS}
        w = rng.normal(size=q.shape)
        eps = 1e-6
        sp, sm = st.copy(), st.copy()
        for f in STATE_FIELDS:
            sp[f] += eps * vs[f]
            sm[f] -= eps * vs[f]
        fd = float(np.sum(w * (rhs(q + eps * vq, sp) - rhs(q - eps * vq, sm)) / (2 * eps)))
        cells, fixed, nvar, nsp = (C.c_size_t() for _ in range(4))
        assert L.reactive_transport_layout_v3(h, C.byref(cells), C.byref(fixed), C.byref(nvar), C.byref(nsp)) == 0
        all_ = nc + fixed.value
        stream = torch.cuda.current_stream().cuda_stream
        qd = torch.zeros((nv, all_), dtype=torch.float64, device="cuda")
        qd[:, :nc] = torch.from_numpy(q.T.copy()).cuda()
        sd = torch.zeros((all_, 7), dtype=torch.float64, device="cuda")
        sd[:nc] = torch.from_numpy(st.view(np.float64).reshape(nc, 7)).cuda()
        assert L.reactive_transport_fill_fixed_v3(h, qd.data_ptr(), sd.data_ptr(), stream) == 0
        wd = torch.from_numpy(w.T.copy()).cuda()
        q_bar = torch.empty((nv, nc), dtype=torch.float64, device="cuda")
        s_bar = torch.empty((nc, 7), dtype=torch.float64, device="cuda")
        assert L.reactive_transport_rate_vjp_v3(h, qd.data_ptr(), sd.data_ptr(), wd.data_ptr(), q_bar.data_ptr(),
                                                s_bar.data_ptr(), stream) == 0, lib.reactive_transport_error(h)
        torch.cuda.synchronize()
        qb = q_bar.cpu().numpy().T
        sb = s_bar.cpu().numpy().view(A.STATE_DTYPE).reshape(nc)
        adj = float(np.sum(qb * vq)) + sum(float(np.sum(sb[f] * vs[f])) for f in STATE_FIELDS)
        assert abs(adj - fd) <= 1e-6 * max(abs(fd), 1e-300), (adj, fd)
        # the HLLC operator's derivative is not the HLL one's
        assert L.reactive_transport_flux_v3(h, 0, None) == 0
        assert L.reactive_transport_rate_vjp_v3(h, qd.data_ptr(), sd.data_ptr(), wd.data_ptr(), q_bar.data_ptr(),
                                                s_bar.data_ptr(), stream) == 0
        torch.cuda.synchronize()
        hll = float(np.sum(q_bar.cpu().numpy().T * vq))
        assert abs(hll - float(np.sum(qb * vq))) > 1e-6 * abs(hll)
    finally:
        oracle.set_flux_scheme(0)
        lib.reactive_transport_destroy(h)


def test_hllc_hem_step_gradient_against_finite_differences():
    """The SSPRK2 + HEM step adjoint with the HLLC flux (config-5 physics)."""
    n, steps, dt = 12, 2, 1e-8
    faces, volume = cases.cartesian_faces(n, edge=n * 1e-3, port_diameter=0.005, port_z=n * 0.5e-3,
                                          port_offset=0.004)
    init = cases.impingement(n, seed=11)
    flow = Flow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"], viscosity=1.821e-5,
                conductivity=0.02587, wale_cw=0.325, flux="hllc")
    stepper = HemStep(flow)
    cells = flow.cells
    try:
        q0 = flow.qn.clone()
        s0 = flow.sn.clone()
        k, j, i = np.indices((n, n, n))
        sub = ((i >= 2) & (i < 6) & (j >= 2) & (j < 6) & (k >= 4) & (k < 8)).ravel()
        weight = torch.zeros_like(q0)
        weight[0, :cells] = torch.from_numpy(sub * volume).cuda()
        weight[4, :cells] = torch.from_numpy(sub * volume).cuda() * 1e-6

        def loss(q):
            s = stepper.recover(q.detach(), s0)
            out, _ = hem_rollout(stepper, q, s, steps, dt, checkpoint_every=1)
            return (out * weight).sum()

        qg = q0.clone().requires_grad_(True)
        (g,) = torch.autograd.grad(loss(qg), qg)
        stepper.check()
        rng = np.random.default_rng(5)
        probes = rng.choice(np.flatnonzero(sub), 6, replace=False)
        with torch.no_grad():
            for c in probes:
                for var in (0, 4):
                    h = 1e-6 * abs(float(q0[var, c]))
                    qp, qm = q0.clone(), q0.clone()
                    qp[var, c] += h
                    qm[var, c] -= h
                    fd = (loss(qp) - loss(qm)).item() / (2 * h)
                    got = g[var, c].item()
                    assert abs(got - fd) <= 2e-4 * abs(fd) + 1e-12 * abs(g[var]).max().item(), (c, var, got, fd)
        stepper.check()
    finally:
        flow.close()
