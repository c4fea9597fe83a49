"""SSPRK2 + HEM step driver (the RK stage driver of the hot path), device resident.

One accepted step follows the reference's Flow::step
(src/reactiveFoam/ReactiveFoam.C:961-1019) with chemistry off:
    CFL query at the step-start state                      (:1443, stableStep :798-812)
    stage 0   q1 = qn + dt L(qn; thermo_n)                 (transportStage :651-661)
    recovery  thermo_1 = flash(q1) seeded by thermo_n       (recover :732-751)
    CFL recheck at q1                                       (:993)
    stage 1   q_{n+1} = qn/2 + (q1 + dt L(q1; thermo_1))/2
    recovery  thermo_{n+1} = flash(q_{n+1}) seeded by thermo_n (step-start seed, :1011-1013)
    boundary ledger  .5 dt (B0 + B1)                        (:1014-1016)
Transport uses the frozen sound speed (compact, :419-420).

Unlike the reference, q and the thermodynamic states never leave HBM between
stages: the transport *_v3 and HEM run_device_v3 entry points work on the same
SoA conserved arrays, and with `graph=True` the whole step (2 CFL reductions,
2 transport stages, 2 flashes, the ledger) replays as one captured CUDA graph.
"""
import ctypes as C

import numpy as np
import torch

from . import _abi as A, _lib
from .hem import GpuHem
from .thermo_data import pure_model


class FlowError(RuntimeError):
    pass


def field_errors(q, s, ref_q, ref_s):
    """Per-field error of a run (cell-major q, thermo states s) against a
    reference run: relative per cell for the positive fields (each species mass,
    rho, rhoE, p, T), scaled by the field's largest magnitude for the momentum
    components (which pass through zero)."""
    ns = q.shape[1] - 4
    rel = lambda a, b: float(np.max(np.abs(a - b) / np.abs(b)))
    out = {"rho": rel(q[:, :ns].sum(axis=1), ref_q[:, :ns].sum(axis=1))}
    if ns > 1:
        out.update({f"q{k}": rel(q[:, k], ref_q[:, k]) for k in range(ns)})
    for d, name in enumerate(("rhoU", "rhoV", "rhoW")):
        m = ref_q[:, ns + d]
        out[name] = float(np.max(np.abs(q[:, ns + d] - m)) / max(np.abs(m).max(), 1e-300))
    out["rhoE"] = rel(q[:, ns + 3], ref_q[:, ns + 3])
    out["p"] = rel(s["p"], ref_s["p"])
    out["T"] = rel(s["T"], ref_s["T"])
    return out


def _check(lib, handle, rc):
    if rc:
        raise FlowError(lib.reactive_transport_error(handle).decode())


class Flow:
    def __init__(self, faces, volume, q0, guess0, fixed_q, fixed_guess, viscosity=0.0, conductivity=0.0,
                 wale_cw=None, wave_factor=1.1, model=None, cfl=0.5, device="cuda", precision="fp64",
                 turbulent_prandtl=None, turbulent_schmidt=None, flux="hll", owned=None):
        """faces: FACE_DTYPE array; q0: cell-major (cells, 5) conserved state;
        guess0/fixed_guess: THERMO_DTYPE seeds used for the initial recovery.
        precision: "fp64", or "mixed" (FP32 gradients, WALE and face fluxes with
        compensated per-cell sums into the FP64 state; needs a structured box).
        turbulent_prandtl / turbulent_schmidt: the WALE scalar closure (needs
        wale_cw; 0 disables a term), fed each stage with the mixture cp of that
        stage's equilibrium states. flux: "hll", or "hllc" (the contact-preserving
        flux; needs a structured box). owned: (begin, end), the cells this flow
        updates, recovers and counts in its CFL minimum and ledger (a z-slab's
        own cells; the others are halo cells that a halo exchange fills)."""
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"unknown precision {precision!r}")
        if flux not in ("hll", "hllc"):
            raise ValueError(f"unknown flux {flux!r}")
        self.lib = _lib.load()
        self.device = torch.device(device)
        self.cells = len(volume)
        self.volume = np.ascontiguousarray(volume, dtype=np.float64)
        self.fixed = len(fixed_q)
        self.nv = q0.shape[1]
        self.cfl = cfl
        self.hem = GpuHem(model=model if model is not None else pure_model(), capacity=max(self.cells, self.fixed))
        # Initial recoveries on the host path (once): fixed inlet states and cells.
        fixed_state = fixed_guess.copy()
        e_fixed = fixed_q[:, 4] - .5 * np.sum(fixed_q[:, 1:4] ** 2, axis=1) / fixed_q[:, 0]
        ok, _ = self.hem.run(np.ascontiguousarray(fixed_q[:, 0]), e_fixed, fixed_state)
        if not ok.all():
            raise FlowError("fixed-state recovery failed")
        state0 = guess0.copy()
        e0 = q0[:, 4] - .5 * np.sum(q0[:, 1:4] ** 2, axis=1) / q0[:, 0]
        ok, _ = self.hem.run(np.ascontiguousarray(q0[:, 0]), e0, state0)
        if not ok.all():
            raise FlowError(f"initial recovery failed in {int((ok == 0).sum())} cells")
        fixed_tr = np.zeros(self.fixed, dtype=A.STATE_DTYPE)
        for k_out, k_in in (("p", "p"), ("T", "T"), ("rho", "rho"), ("cv", "cv"), ("sound", "soundFrozen"),
                            ("gasMass", "gasMass")):
            fixed_tr[k_out] = fixed_state[k_in]
        cfg = A.Config(self.cells, 1, self.nv, len(faces), self.fixed, viscosity, conductivity, 0.0, wave_factor,
                       1.6e11, 0)
        self._faces = np.ascontiguousarray(faces)
        err = C.create_string_buffer(2048)
        h = self.lib.reactive_transport_create(
            1, C.byref(cfg), A.dptr(np.ascontiguousarray(volume, dtype=np.float64)),
            self._faces.ctypes.data_as(C.POINTER(A.Face)), A.dptr(np.ascontiguousarray(fixed_q, dtype=np.float64)),
            fixed_tr.ctypes.data_as(C.POINTER(A.State)), None, None, err, len(err))
        if not h:
            raise FlowError(err.value.decode())
        self.transport = C.c_void_p(h)
        if wale_cw is not None:
            opts = A.WaleOptions(1, C.sizeof(A.WaleOptions), wale_cw)
            _check(self.lib, self.transport, self.lib.reactive_transport_set_wale_v1(self.transport, C.byref(opts)))
        self.scalars = turbulent_prandtl is not None or turbulent_schmidt is not None
        if self.scalars:
            opts = A.WaleScalarOptions(1, C.sizeof(A.WaleScalarOptions), turbulent_prandtl or 0.0,
                                       turbulent_schmidt or 0.0)
            _check(self.lib, self.transport,
                   self.lib.reactive_transport_set_wale_scalars_v1(self.transport, C.byref(opts)))
        self.precision = precision
        if precision == "mixed":
            _check(self.lib, self.transport, self.lib.reactive_transport_precision_v3(self.transport, 1, None))
        self.flux = flux
        if flux == "hllc":
            _check(self.lib, self.transport, self.lib.reactive_transport_flux_v3(self.transport, 1, None))
        self.own = (0, self.cells) if owned is None else (int(owned[0]), int(owned[1]))
        if owned is not None:
            _check(self.lib, self.transport,
                   self.lib.reactive_transport_owned_cells_v3(self.transport, self.own[0], self.own[1]))
        all_ = self.cells + self.fixed
        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.qn = torch.zeros((self.nv, all_), **f64)
        self.qn[:, :self.cells] = torch.from_numpy(np.ascontiguousarray(q0.T)).to(dev)
        self.q1 = torch.zeros_like(self.qn)
        self.tr = torch.zeros((all_, 7), **f64)
        self.sn = torch.from_numpy(state0.view(np.uint8).copy()).to(dev)   # step-start thermo (seeds)
        self.s1 = torch.zeros_like(self.sn)                                   # stage-1 thermo
        # per-cell success flags of each stage's recovery (a failure in either fails the step)
        self.success_stages = torch.zeros((2, self.cells), dtype=torch.int32, device=dev)
        self.success = self.success_stages[1]
        self.boundary = torch.zeros((2, self.nv), **f64)
        self.dt_cfl = torch.zeros(2, **f64)
        self.stream = torch.cuda.Stream(device=dev)
        s = self.stream.cuda_stream
        tr0 = np.zeros(self.cells, dtype=A.STATE_DTYPE)
        for k_out, k_in in (("p", "p"), ("T", "T"), ("rho", "rho"), ("cv", "cv"), ("sound", "soundFrozen"),
                            ("gasMass", "gasMass")):
            tr0[k_out] = state0[k_in]
        self.tr[:self.cells] = torch.from_numpy(tr0.view(np.float64).reshape(self.cells, 7)).to(dev)
        # fixed-state thermo (constant): the WALE scalar closure's fixed cp
        self.fixed_thermo = torch.from_numpy(fixed_state.view(np.uint8).copy()).to(dev)
        torch.cuda.synchronize(dev)
        if self.scalars:
            self._scalar_fields(self.sn, fixed=True)
        _check(self.lib, self.transport,
               self.lib.reactive_transport_fill_fixed_v3(self.transport, self.qn.data_ptr(), self.tr.data_ptr(), s))
        _check(self.lib, self.transport,
               self.lib.reactive_transport_fill_fixed_v3(self.transport, self.q1.data_ptr(), self.tr.data_ptr(), s))
        self.stream.synchronize()
        self.graph = None
        self.graph_dt = None
        self.steps = 0
        self.retries = 0           # dt halvings taken by advance()
        self.last_failure = None   # why advance()'s last failed attempt failed

    # ------------------------------------------------------------------ step
    _CP_OFFSET = A.THERMO_DTYPE.fields["cp"][1]
    _THERMO_DOUBLES = A.THERMO_DTYPE.itemsize // 8

    def _scalar_fields(self, thermo, fixed=False):
        """Point the WALE scalar closure at the mixture cp of `thermo` (one
        species: no enthalpies are needed)."""
        lib, t, s = self.lib, self.transport, self.stream.cuda_stream
        fixed_cp = self.fixed_thermo.data_ptr() + self._CP_OFFSET if fixed and self.fixed else None
        _check(lib, t, lib.reactive_transport_wale_scalar_fields_device_v3(
            t, thermo.data_ptr() + self._CP_OFFSET, None, fixed_cp, None, self._THERMO_DOUBLES, 1, s))

    def _flash(self, q, out, per_cell=False, stage=0):
        """Recovery of the own cells of q (SoA, stride cells+fixed) seeded by the
        step-start states, into `out` and the transport states."""
        b, e = self.own
        size = A.THERMO_DTYPE.itemsize
        success = self.success_stages[stage]
        self.hem.run_device(q.data_ptr() + 8 * b, self.qn.shape[1], e - b, self.nv, self.sn.data_ptr() + size * b,
                            out.data_ptr() + size * b, self.tr.data_ptr() + 56 * b, success.data_ptr() + 4 * b,
                            self.stream.cuda_stream, per_cell)

    def _launch_half(self, dt, stage, per_cell=False):
        """Stage 0 (CFL query, q1 = qn + dt L(qn), recovery of q1 into s1) or
        stage 1 (CFL recheck at q1, q_{n+1} into qn, recovery in place)."""
        lib, t, s = self.lib, self.transport, self.stream.cuda_stream
        q_in, q_out, seed_out = (self.qn, self.q1, self.s1) if stage == 0 else (self.q1, self.qn, self.sn)
        if self.scalars:
            self._scalar_fields(self.sn if stage == 0 else self.s1)
        # the CFL query at q_in and the stage from q_in in one call (the results of
        # stable_step_device_v3 then stage_device_v3, bit for bit)
        _check(lib, t, lib.reactive_transport_stage_cfl_device_v3(
            t, q_in.data_ptr(), q_out.data_ptr(), self.tr.data_ptr(), dt, stage, self.boundary[stage].data_ptr(),
            self.cfl, dt, self.dt_cfl[stage:].data_ptr(), s))
        # both recoveries are seeded by the step-start states; the second one in place
        self._flash(q_out, seed_out, per_cell, stage)

    def _launch_step(self, dt, per_cell=False):
        self._launch_half(dt, 0, per_cell)
        self._launch_half(dt, 1, per_cell)

    def two_phase_bound(self, on=None):
        """Query (on=None) or set the flash's two-phase admissibility bound
        (reactive_gpu_hem_two_phase_bound_v3); drops a captured graph."""
        active = C.c_int()
        err = C.create_string_buffer(512)
        request = -1 if on is None else int(bool(on))
        if self.lib.reactive_gpu_hem_two_phase_bound_v3(self.hem.handle, request, C.byref(active), err, len(err)):
            raise FlowError(err.value.decode())
        if on is not None:
            self.graph = None
        return bool(active.value)

    def stage0(self, dt):
        """Stage 0 of a step on the resident state (CFL query and q1 = qn + dt L(qn)),
        leaving q1 and the step-start states as the step's first recovery takes
        them (asynchronous on the flow's stream)."""
        lib, t, s = self.lib, self.transport, self.stream.cuda_stream
        if self.scalars:
            self._scalar_fields(self.sn)
        _check(lib, t, lib.reactive_transport_stage_cfl_device_v3(
            t, self.qn.data_ptr(), self.q1.data_ptr(), self.tr.data_ptr(), dt, 0, self.boundary[0].data_ptr(),
            self.cfl, dt, self.dt_cfl.data_ptr(), s))

    def autotune(self):
        """Choose the launch shapes of this flow's transport and flash kernels by
        timing the candidates on its current state (synchronous; drops a
        captured graph so the next step recaptures with the new shapes)."""
        lib, t, s = self.lib, self.transport, self.stream.cuda_stream
        chosen = (C.c_uint * 3)()
        _check(lib, t, lib.reactive_transport_autotune_v3(t, self.qn.data_ptr(), self.tr.data_ptr(), s, chosen))
        blocks = C.c_int()
        err = C.create_string_buffer(1024)
        if lib.reactive_gpu_hem_autotune_v3(self.hem.handle, self.qn.data_ptr(), self.qn.shape[1], self.cells, self.nv,
                                            self.sn.data_ptr(), s, C.byref(blocks), err, len(err)):
            raise FlowError(err.value.decode())
        self.stream.synchronize()
        self.graph = None
        return {"stage_block": chosen[0], "gradient_block": chosen[1], "cfl_block": chosen[2],
                "flash_blocks_per_sm": blocks.value}

    def ledger(self, dt):
        """Boundary ledger of the last step, .5 dt (B0 + B1) per variable (host;
        synchronises the flow's stream)."""
        self.stream.synchronize()
        b = self.boundary.cpu().numpy()
        return .5 * dt * (b[0] + b[1])

    def capture(self, dt):
        """Capture one step as a CUDA graph (replayed by step(dt) for this dt)."""
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=self.stream):
            self._launch_step(dt)
        self.graph_dt = dt

    def step(self, dt, graph=True, per_cell=False):
        """One step. graph: replay the captured graph (work-queue flash); per_cell:
        launch one by one with the plain one-thread-per-cell flash."""
        if graph and not per_cell:
            if self.graph is None or self.graph_dt != dt:
                self.capture(dt)  # records the launches; nothing executes until replay
            with torch.cuda.stream(self.stream):  # replay() launches on the current stream
                self.graph.replay()
        else:
            with torch.cuda.stream(self.stream):
                self._launch_step(dt, per_cell)
        self.steps += 1

    def _failure(self, dt, totals0=None):
        """Why the last step failed, or None (synchronises): a recovery that
        failed in any own cell at either stage, a CFL step (at the step start or at
        RK1) that does not admit dt, a transport status bit (WALE / HLLC / scalar
        field), or, with totals0 (the step-start totals), the boundary-corrected
        mass and total-energy balances of the reference driver
        (src/reactiveFoam/ReactiveFoam.C:1458-1470: mass within 1e-7 of the mass,
        energy within 1e-9 of the energy scale)."""
        self.stream.synchronize()
        status = C.c_uint()
        _check(self.lib, self.transport,
               self.lib.reactive_transport_status_v3(self.transport, C.byref(status), 1, self.stream.cuda_stream))
        own = slice(self.own[0], self.own[1])
        failed = int((self.success_stages[:, own] == 0).any(dim=0).sum().item())
        if failed:
            return f"HEM recovery failed in {failed} cells"
        cfl = self.dt_cfl.min().item()
        if not (cfl > 0 and dt <= cfl * (1 + 1e-10)):
            return f"dt={dt} exceeds the wave/diffusion CFL step {cfl}"
        if status.value & 7:
            return f"transport status {status.value}"
        if totals0 is not None:
            totals = self._totals()
            ledger = torch.from_numpy(self.ledger(dt)).to(self.device)
            balance = totals - totals0 + ledger
            mass0 = float(totals0[:self.nv - 4].sum())
            energy_scale = max(float(self._energy_magnitude()), mass0 * 1e5)
            mass_error = abs(float(balance[:self.nv - 4].sum())) / mass0
            energy_error = abs(float(balance[self.nv - 1])) / energy_scale
            if not (np.isfinite(mass_error) and np.isfinite(energy_error) and mass_error < 1e-7
                    and energy_error < 1e-9):
                return f"boundary-corrected balance failed (mass {mass_error:.3e}, energy {energy_error:.3e})"
        return None

    def _totals(self):
        """Volume integrals of the own cells' conserved variables (device, FP64)."""
        b, e = self.own
        if not hasattr(self, "_volume_device"):
            self._volume_device = torch.from_numpy(self.volume).to(self.device)
        with torch.cuda.stream(self.stream):
            return (self.qn[:, b:e] * self._volume_device[b:e]).sum(dim=1)

    def _energy_magnitude(self):
        b, e = self.own
        with torch.cuda.stream(self.stream):
            return (self.qn[self.nv - 1, b:e].abs() * self._volume_device[b:e]).sum()

    def advance(self, dt, max_retries=12, graph=True, balance=True):
        """One accepted step with the reference driver's failure handling
        (src/reactiveFoam/ReactiveFoam.C:1434-1494): the step-start conserved and
        thermodynamic states are kept on the device; a step that fails (see
        _failure; balance=False skips the balance check) is rolled back to them
        and retried with half the step, at most max_retries times (and not below
        1e-15 s). Returns the dt taken. When the retries run out the state is the
        step-start state again and FlowError is raised. The retries launch the
        kernels one by one (the captured graph holds the caller's dt)."""
        if not hasattr(self, "_saved"):
            self._saved = [torch.empty_like(self.qn), torch.empty_like(self.sn), torch.empty_like(self.tr)]
        with torch.cuda.stream(self.stream):
            for dst, src in zip(self._saved, (self.qn, self.sn, self.tr)):
                dst.copy_(src)
        totals0 = self._totals() if balance else None
        steps0 = self.steps
        attempt_dt = dt
        for retry in range(max_retries + 1):
            self.step(attempt_dt, graph=graph and attempt_dt == dt)
            reason = self._failure(attempt_dt, totals0)
            if reason is None:
                return attempt_dt
            with torch.cuda.stream(self.stream):
                for dst, src in zip((self.qn, self.sn, self.tr), self._saved):
                    dst.copy_(src)
            self.steps = steps0
            self.last_failure = reason
            if retry == max_retries or attempt_dt * .5 <= 1e-15:
                break
            self.retries += 1
            attempt_dt *= .5
        self.stream.synchronize()
        raise FlowError(f"step failed after {max_retries} retries with dt halved to {attempt_dt}: {reason}")

    def check(self, dt):
        """Host check after a run of steps: every flash succeeded, dt within CFL,
        no WALE failure (synchronises)."""
        self.stream.synchronize()
        status = C.c_uint()
        _check(self.lib, self.transport,
               self.lib.reactive_transport_status_v3(self.transport, C.byref(status), 1, self.stream.cuda_stream))
        failed = int((self.success_stages[:, self.own[0]:self.own[1]] == 0).any(dim=0).sum().item())
        cfl = self.dt_cfl.min().item()
        if status.value & 1:
            raise FlowError("WALE gradient/viscosity/traction became non-finite")
        if status.value & 2:
            raise FlowError("an HLLC face flux could not be formed")
        if status.value & 4:
            raise FlowError("a WALE scalar field (mixture cp) was not finite and positive")
        if failed:
            raise FlowError(f"HEM recovery failed in {failed} cells")
        if not (cfl > 0 and dt <= cfl * (1 + 1e-10)):
            raise FlowError(f"dt={dt} exceeds the wave/diffusion CFL step {cfl}")
        return dict(cfl_dt=cfl)

    # ----------------------------------------------------------- checkpoints
    def history(self, time, initial=None, boundary=None):
        """A checkpoint history for the current state: the conservation scales
        the solver derives at start (src/reactiveFoam/ReactiveFoam.C:1402-1407),
        the current totals as the baseline unless given, zero boundary
        integral unless given."""
        from .checkpoint import History
        q, s = self.conserved(), self.states()
        totals = (q * self.volume[:, None]).sum(axis=0)
        speed = np.sqrt((q[:, 1:4] ** 2).sum(axis=1)) / q[:, 0] + s["soundFrozen"]
        mass0 = float(totals[0] if initial is None else initial[0])
        energy_scale = max(float((np.abs(q[:, 4]) * self.volume).sum()), mass0 * 1e5)
        return History(initial=totals if initial is None else np.asarray(initial, float),
                       boundary=np.zeros(self.nv) if boundary is None else np.asarray(boundary, float),
                       steps=self.steps, time=float(time), velocity_scale=max(1.0, float(speed.max())),
                       energy_scale=energy_scale)

    def save_checkpoint(self, root, time, history=None, identity=None, last_dt=0.0, run_id="b200"):
        """Commit a schema-3 checkpoint of the current state under root/<time>
        (synchronises). identity: the identity dictionary's fields; by default
        this library's own digests of the model image (a reference solver
        restart needs the reference's own hashes)."""
        import hashlib
        from . import checkpoint
        hist = history if history is not None else self.history(time)
        hist.last_dt = last_dt
        if identity is None:
            image = self.hem.image
            digest = hashlib.sha256(image).hexdigest()
            identity = dict(fingerprint=digest, physical_model_hash=digest,
                            numerical_policy_hash=hashlib.sha256(image[-2448:]).hexdigest(), species_count=1,
                            closure="HEM")
        return checkpoint.save(root, self.conserved(), self.states(), hist, identity, run_id=run_id)

    def load_checkpoint(self, directory):
        """Restart from a committed checkpoint: its conserved state and its
        thermodynamic states (the next step's seeds) replace this flow's
        (synchronises). Returns the checkpoint's History."""
        from . import checkpoint
        q, states, hist, _ = checkpoint.load(directory, self.cells, self.nv)
        self.stream.synchronize()
        self.qn[:, :self.cells] = torch.from_numpy(np.ascontiguousarray(q.T)).to(self.device)
        self.sn.copy_(torch.from_numpy(states.view(np.uint8).copy()))
        tr = np.zeros(self.cells, dtype=A.STATE_DTYPE)
        for k_out, k_in in (("p", "p"), ("T", "T"), ("rho", "rho"), ("cv", "cv"), ("sound", "soundFrozen"),
                            ("gasMass", "gasMass")):
            tr[k_out] = states[k_in]
        self.tr[:self.cells] = torch.from_numpy(tr.view(np.float64).reshape(self.cells, 7)).to(self.device)
        torch.cuda.synchronize(self.device)
        self.steps = int(hist.steps)
        return hist

    # --------------------------------------------------------------- views
    def conserved(self):
        """Cell-major host copy of the conserved state (cells, nv)."""
        self.stream.synchronize()
        return self.qn[:, :self.cells].T.contiguous().cpu().numpy()

    def states(self):
        """Host copy of the thermodynamic states (THERMO_DTYPE)."""
        self.stream.synchronize()
        return self.sn.cpu().numpy().view(A.THERMO_DTYPE)

    def close(self):
        if getattr(self, "transport", None):
            self.stream.synchronize()
            self.graph = None
            self.lib.reactive_transport_destroy(self.transport)
            self.transport = None
            self.hem.close()
