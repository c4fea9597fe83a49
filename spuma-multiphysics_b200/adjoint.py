"""Differentiable SSPRK2 steps on a structured box with a hand-written adjoint.

One step of the reference's RK driver (src/reactiveFoam/ReactiveFoam.C:961-1019,
fixed dt, chemistry off) on an ideal-gas mixture box:

    s_n   = closure(q_n)
    q_1   = q_n + dt L(q_n, s_n)                 (transport stage 0)
    s_1   = closure(q_1)
    q_n+1 = q_n / 2 + (q_1 + dt L(q_1, s_1)) / 2 (transport stage 1)

is a torch.autograd.Function (`SSPRK2Step`) whose forward runs the CUDA stage
and closure entries and whose backward is the hand-written adjoint of the same
step, lambda_n = (d q_n+1 / d q_n)^T lambda_n+1:

    w_1     = dt/2 lambda
    qbar_1  = lambda/2 + L_q(q_1)^T w_1 + closure_q(q_1)^T L_s(q_1)^T w_1
    w_0     = dt qbar_1
    lambda_n = lambda/2 + qbar_1 + L_q(q_n)^T w_0 + closure_q(q_n)^T L_s(q_n)^T w_0

with L_q^T w and L_s^T w from reactive_transport_rate_vjp_v3 (the HLL flux
differentiated piecewise through its wave-speed switches) and closure_q^T from
reactive_ideal_gas_vjp_device_v3 (temperature by the implicit function theorem
at the converged state, no Newton unrolling). `rollout` chains steps in
segments of `checkpoint_every` under torch.utils.checkpoint: only the segment
inputs are kept in the forward pass; the reverse pass recomputes a segment's
steps and then runs their adjoints.
"""
import ctypes as C

import numpy as np
import torch
import torch.utils.checkpoint

from . import _abi as A, _lib
from .thermo_data import N2, N2O, gas_table


class AdjointError(RuntimeError):
    pass


class IdealGasBox:
    """A structured Cartesian box of an ideal-gas mixture (inviscid HLL
    transport, ideal-gas closure), device resident, with the vector-Jacobian
    products its adjoint needs. Conserved tensors are SoA (nv, cells), FP64."""

    def __init__(self, faces, volume, species=(N2O, N2), T_guess=300.0, Tmin=150.0, Tmax=3000.0,
                 tolerance=1e-13, device="cuda"):
        self.lib = _lib.load()
        self.device = torch.device(device)
        self.cells = len(volume)
        self.ns = len(species)
        self.nv = self.ns + 4
        faces = np.ascontiguousarray(faces)
        if np.any(faces["kind"] == 3):
            raise AdjointError("fixed-state boundary faces are not supported by the ideal-gas box")
        cfg = A.Config(self.cells, self.ns, self.nv, len(faces), 0, 0.0, 0.0, 0.0, 1.1, 1.6e11, 0)
        err = C.create_string_buffer(2048)
        self._faces = faces
        self._volume = np.ascontiguousarray(volume, dtype=np.float64)
        h = self.lib.reactive_transport_create(1, C.byref(cfg), A.dptr(self._volume),
                                               faces.ctypes.data_as(C.POINTER(A.Face)), None, None, None, None,
                                               err, len(err))
        if not h:
            raise AdjointError(err.value.decode())
        self.transport = C.c_void_p(h)
        active = C.c_int()
        self._check(self.lib.reactive_transport_structured_v3(self.transport, -1, C.byref(active)))
        if not active.value:
            raise AdjointError("the face list is not a structured Cartesian box in canonical order")
        table = gas_table(species)
        g = self.lib.reactive_ideal_gas_create_v3(table, len(table), Tmin, Tmax, tolerance, err, len(err))
        if not g:
            raise AdjointError(err.value.decode())
        self.gas = C.c_void_p(g)
        f64 = dict(dtype=torch.float64, device=self.device)
        self.T_guess = torch.full((self.cells,), float(T_guess), **f64)
        self.volume = torch.from_numpy(self._volume).to(self.device)
        self.success = torch.zeros(self.cells, dtype=torch.int32, device=self.device)
        self.failures = torch.zeros((), dtype=torch.int64, device=self.device)  # closure failures since check()
        self.err = C.create_string_buffer(1024)

    # ------------------------------------------------------------- plumbing
    def _check(self, rc):
        if rc:
            raise AdjointError(self.lib.reactive_transport_error(self.transport).decode())

    def _gas_check(self, rc):
        if rc:
            raise AdjointError(self.err.value.decode())

    def close(self):
        if getattr(self, "transport", None):
            torch.cuda.synchronize(self.device)
            self.lib.reactive_transport_destroy(self.transport)
            self.transport = None
        if getattr(self, "gas", None):
            self.lib.reactive_ideal_gas_destroy_v3(self.gas)
            self.gas = None

    def closure(self, q):
        """States of q (nv, cells): (T, transport states (cells, 7)); every cell
        is seeded from the fixed guess temperature, so a recomputation gives
        the same bits."""
        s = torch.cuda.current_stream().cuda_stream
        T = torch.empty(self.cells, dtype=torch.float64, device=self.device)
        tr = torch.empty((self.cells, 7), dtype=torch.float64, device=self.device)
        self._gas_check(self.lib.reactive_ideal_gas_run_device_v3(
            self.gas, q.data_ptr(), q.shape[1], self.cells, self.nv, self.T_guess.data_ptr(), T.data_ptr(),
            tr.data_ptr(), self.success.data_ptr(), s, self.err, len(self.err)))
        self.failures += (self.success == 0).sum()
        return T, tr

    def stage(self, q_in, q_out, tr, dt, stage):
        self._check(self.lib.reactive_transport_stage_device_v3(self.transport, q_in.data_ptr(), q_out.data_ptr(),
                                                               tr.data_ptr(), dt, stage, None,
                                                               torch.cuda.current_stream().cuda_stream))

    def rate_vjp(self, q, tr, w):
        """(dL/dq)^T w (nv, cells) and (dL/dstate)^T w (cells, 7)."""
        q_bar = torch.empty((self.nv, self.cells), dtype=torch.float64, device=self.device)
        tr_bar = torch.empty((self.cells, 7), dtype=torch.float64, device=self.device)
        self._check(self.lib.reactive_transport_rate_vjp_v3(self.transport, q.data_ptr(), tr.data_ptr(),
                                                            w.contiguous().data_ptr(), q_bar.data_ptr(),
                                                            tr_bar.data_ptr(), torch.cuda.current_stream().cuda_stream))
        return q_bar, tr_bar

    def closure_vjp(self, q, T, tr_bar, q_bar):
        """q_bar += (d state / d q)^T tr_bar (in place)."""
        self._gas_check(self.lib.reactive_ideal_gas_vjp_device_v3(
            self.gas, q.data_ptr(), q.shape[1], self.cells, self.nv, T.data_ptr(), tr_bar.data_ptr(),
            q_bar.data_ptr(), q_bar.shape[1], torch.cuda.current_stream().cuda_stream, self.err, len(self.err)))
        return q_bar

    # ---------------------------------------------------------- the step
    def forward_step(self, q_n, dt):
        """One SSPRK2 step; returns q_n+1 and what its adjoint needs."""
        q_n = q_n.contiguous()
        T_n, tr_n = self.closure(q_n)
        q_1 = torch.empty_like(q_n)
        self.stage(q_n, q_1, tr_n, dt, 0)
        T_1, tr_1 = self.closure(q_1)
        q_next = q_n.clone()
        self.stage(q_1, q_next, tr_1, dt, 1)
        return q_next, (q_n, q_1, T_n, T_1, tr_n, tr_1)

    def step_vjp(self, lam, saved, dt):
        q_n, q_1, T_n, T_1, tr_n, tr_1 = saved
        lam = lam.contiguous()
        q_bar1, tr_bar1 = self.rate_vjp(q_1, tr_1, (.5 * dt) * lam)
        q_bar1 += .5 * lam
        self.closure_vjp(q_1, T_1, tr_bar1, q_bar1)
        q_barn, tr_barn = self.rate_vjp(q_n, tr_n, dt * q_bar1)
        q_barn += .5 * lam + q_bar1
        self.closure_vjp(q_n, T_n, tr_barn, q_barn)
        return q_barn

    def check(self):
        """Every closure since the last check converged (synchronises)."""
        failed = int(self.failures.item())
        self.failures.zero_()
        if failed:
            raise AdjointError(f"ideal-gas closure failed in {failed} cells")

    def stable_dt(self, q, cfl=0.5):
        """The CFL step of state q (host float; synchronises)."""
        q = q.contiguous()
        _, tr = self.closure(q)
        dt = torch.zeros(1, dtype=torch.float64, device=self.device)
        self._check(self.lib.reactive_transport_stable_step_device_v3(self.transport, q.data_ptr(), tr.data_ptr(),
                                                                     cfl, 1.0, dt.data_ptr(),
                                                                     torch.cuda.current_stream().cuda_stream))
        return dt.item()


class SSPRK2Step(torch.autograd.Function):
    """q_n+1 = step(q_n) with the hand-written adjoint as its backward."""

    @staticmethod
    def forward(ctx, q, box, dt):
        q_next, saved = box.forward_step(q.detach(), dt)
        ctx.box, ctx.dt = box, dt
        ctx.save_for_backward(*saved)
        return q_next

    @staticmethod
    def backward(ctx, lam):
        return ctx.box.step_vjp(lam, ctx.saved_tensors, ctx.dt), None, None


def _segment(q, box, dt, steps):
    for _ in range(steps):
        q = SSPRK2Step.apply(q, box, dt)
    return q


def rollout(box, q0, steps, dt, checkpoint_every=10):
    """`steps` SSPRK2 steps from q0 (nv, cells). With autograd recording, the
    steps run in segments of `checkpoint_every` under torch.utils.checkpoint:
    the forward keeps only segment inputs, the backward recomputes each segment
    (its steps re-save their stage states) and then runs their adjoints."""
    q = q0
    done = 0
    while done < steps:
        n = min(checkpoint_every, steps - done)
        if torch.is_grad_enabled() and q.requires_grad:
            q = torch.utils.checkpoint.checkpoint(_segment, q, box, dt, n, use_reentrant=False)
        else:
            q = _segment(q, box, dt, n)
        done += n
    return q


# --------------------------------------------------------------------------
# The HEM step (pure-fluid PR flash, structured viscous/WALE transport)


def _compact(states_u8, cells):
    """Transport states (cells, 7) of thermo states (uint8 view of cells x 176 B):
    p, T, rho, cv, frozen sound, gas mass, 0 (the reference's compact,
    ReactiveFoam.C:419-420)."""
    s = states_u8.view(torch.float64).view(cells, 22)
    tr = torch.zeros((cells, 7), dtype=torch.float64, device=states_u8.device)
    tr[:, 0:3] = s[:, 0:3]
    tr[:, 3] = s[:, 20]
    tr[:, 4] = s[:, 5]
    tr[:, 5] = s[:, 18]
    return tr


class HemStep:
    """Functional SSPRK2 + HEM steps over a `flow.Flow`'s transport and HEM
    handles (FP64, structured path), and their adjoint:

        s_n = flash(q_n) (the previous step's recovery), tr = compact(s)
        q_1 = q_n + dt L(q_n, tr_n);  s_1 = flash(q_1; seed s_n)
        q_n+1 = q_n/2 + (q_1 + dt L(q_1, tr_1))/2;  s_n+1 = flash(q_n+1; seed s_n)

    Conserved tensors are SoA (nv, cells + fixed) with the flow's fixed tail."""

    def __init__(self, flow):
        self.flow = flow
        self.lib = flow.lib
        self.cells, self.fixed, self.nv = flow.cells, flow.fixed, flow.nv
        self.fixed_tr = flow.tr[self.cells:].clone()
        self.failed = torch.zeros(1, dtype=torch.int32, device=flow.device)
        self.err = C.create_string_buffer(1024)
        if flow.precision != "fp64":
            raise AdjointError("the adjoint differentiates the FP64 operator: use a precision='fp64' flow")

    def _check(self, rc):
        if rc:
            raise AdjointError(self.lib.reactive_transport_error(self.flow.transport).decode())

    def _tr_all(self, tr_cells):
        return torch.cat([tr_cells, self.fixed_tr], 0).contiguous()

    def _flash(self, q, seed):
        f = self.flow
        s = torch.cuda.current_stream().cuda_stream
        out = torch.empty_like(seed)
        tr = torch.empty((self.cells + self.fixed, 7), dtype=torch.float64, device=f.device)
        tr[self.cells:] = self.fixed_tr
        f.hem.run_device(q, q.shape[1], self.cells, self.nv, seed, out, tr, f.success, s)
        self.failed += (f.success == 0).sum().to(torch.int32)
        return out, tr

    def _stage(self, q_in, q_out, tr, dt, stage):
        f = self.flow
        self._check(self.lib.reactive_transport_stage_device_v3(f.transport, q_in.data_ptr(), q_out.data_ptr(),
                                                               tr.data_ptr(), dt, stage, None,
                                                               torch.cuda.current_stream().cuda_stream))

    def recover(self, q, seed):
        """The recovered states of q (the flash seeded by `seed`): the s_n a
        rollout from q must start with."""
        states, _ = self._flash(q.contiguous(), seed)
        return states

    def forward_step(self, q_n, s_n, dt):
        q_n = q_n.contiguous()
        tr_n = self._tr_all(_compact(s_n, self.cells))
        q_1 = q_n.clone()
        self._stage(q_n, q_1, tr_n, dt, 0)
        s_1, tr_1 = self._flash(q_1, s_n)
        q_next = q_n.clone()
        self._stage(q_1, q_next, tr_1, dt, 1)
        s_next, _ = self._flash(q_next, s_n)
        return q_next, s_next, (q_n, s_n, tr_n, q_1, s_1, tr_1)

    def rate_vjp(self, q, tr, w):
        f = self.flow
        q_bar = torch.empty((self.nv, self.cells), dtype=torch.float64, device=f.device)
        tr_bar = torch.empty((self.cells, 7), dtype=torch.float64, device=f.device)
        self._check(self.lib.reactive_transport_rate_vjp_v3(f.transport, q.data_ptr(), tr.data_ptr(),
                                                            w.contiguous().data_ptr(), q_bar.data_ptr(),
                                                            tr_bar.data_ptr(), torch.cuda.current_stream().cuda_stream))
        return q_bar, tr_bar

    def hem_vjp(self, q, states, tr_bar, q_bar):
        f = self.flow
        rc = self.lib.reactive_gpu_hem_vjp_device_v3(f.hem.handle, q.data_ptr(), q.shape[1], self.cells, self.nv,
                                                     states.data_ptr(), tr_bar.data_ptr(), q_bar.data_ptr(),
                                                     q_bar.shape[1], self.failed.data_ptr(),
                                                     torch.cuda.current_stream().cuda_stream, self.err, len(self.err))
        if rc:
            raise AdjointError(self.err.value.decode())
        return q_bar

    def step_vjp(self, lam, saved, dt):
        q_n, s_n, tr_n, q_1, s_1, tr_1 = saved
        lam = lam.contiguous()
        q_bar1, tr_bar1 = self.rate_vjp(q_1, tr_1, (.5 * dt) * lam)
        q_bar1 += .5 * lam
        self.hem_vjp(q_1, s_1, tr_bar1, q_bar1)
        q_barn, tr_barn = self.rate_vjp(q_n, tr_n, dt * q_bar1)
        q_barn += .5 * lam + q_bar1
        self.hem_vjp(q_n, s_n, tr_barn, q_barn)
        return q_barn

    def check(self):
        """Every flash and every flash derivative since the last check succeeded,
        and the transport status word is clear (synchronises)."""
        n = int(self.failed.item())
        self.failed.zero_()
        status = C.c_uint()
        self._check(self.lib.reactive_transport_status_v3(self.flow.transport, C.byref(status), 1,
                                                          torch.cuda.current_stream().cuda_stream))
        if n:
            raise AdjointError(f"{n} cell flashes or flash derivatives failed")
        if status.value:
            raise AdjointError(f"transport status {status.value:#x} (1 WALE, 2 HLLC, 4 WALE scalar field)")


class HemSSPRK2Step(torch.autograd.Function):
    """(q_n+1, s_n+1) = step(q_n, s_n) with the hand-written adjoint for q. The
    states s are the step-start recoveries (a function of q through the flash);
    they carry no gradient of their own."""

    @staticmethod
    def forward(ctx, q, s, stepper, dt):
        q_next, s_next, saved = stepper.forward_step(q.detach(), s, dt)
        ctx.stepper, ctx.dt = stepper, dt
        ctx.save_for_backward(*saved)
        ctx.mark_non_differentiable(s_next)
        return q_next, s_next

    @staticmethod
    def backward(ctx, lam, _s_bar):
        cells = ctx.stepper.cells
        q_bar = ctx.stepper.step_vjp(lam[:, :cells], ctx.saved_tensors, ctx.dt)
        # the fixed tail is constant: its adjoint is dropped
        full = torch.zeros_like(lam)
        full[:, :cells] = q_bar
        return full, None, None, None


def _hem_segment(q, s, stepper, dt, steps):
    for _ in range(steps):
        q, s = HemSSPRK2Step.apply(q, s, stepper, dt)
    return q, s


def hem_rollout(stepper, q0, s0, steps, dt, checkpoint_every=10):
    """`steps` HEM steps from (q0, s0), s0 the recovery of q0
    (`HemStep.recover`); with autograd recording, segments of `checkpoint_every`
    run under torch.utils.checkpoint (recomputed in the reverse pass)."""
    q, s = q0, s0
    done = 0
    while done < steps:
        n = min(checkpoint_every, steps - done)
        if torch.is_grad_enabled() and q.requires_grad:
            q, s = torch.utils.checkpoint.checkpoint(_hem_segment, q, s, stepper, dt, n, use_reentrant=False)
        else:
            q, s = _hem_segment(q, s, stepper, dt, n)
        done += n
    return q, s
