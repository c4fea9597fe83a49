#!/usr/bin/env python3
"""Benchmark: Mcell-steps/s of the SSPRK2 + HEM step on the N2O impingement cube.

Workload (default): 160^3 = 4,096,000 cells, 80 mm edge, pure N2O (Peng-Robinson,
HEM UV flash), gas at 40 bar / 293.15 K with a seeded +-1% density perturbation,
two 5 mm liquid inlets at 56.01325 bar / 293.15 K, transmissive walls, HLL,
viscosity 1.821e-5 Pa s, conduction 0.02587 W/m/K, WALE Cw 0.325, dt = 1e-8 s.
One step = CFL query, stage 0, HEM recovery of every cell, CFL recheck, stage 1,
HEM recovery of every cell (both seeded with the step-start states), boundary
ledger.

Keys of the one JSON line rank 0 prints:
  value       FP64 device-resident step, inputs resident in HBM, one captured CUDA
              graph per step (FP64 structured transport, work-queue FP64 flash)
  mixed       the same step with FP32 transport arithmetic (compensated sums into
              the FP64 state) and its per-field error against the FP64 run
  plain_fp64  FP64, kernels launched one by one, flash one thread per cell
  e2e         the same steps through the reference-facing C ABI with host arrays
              (upload_conserved / advance_resident_v2 / download_conserved /
              reactive_gpu_hem_run_v1 per stage, as the reference solver calls it)
  roofline    the dominant kernel (the flash) against the measured FP64 FMA rate
`--impl reference` times the reference's own CPU implementation (its transport
built for the CPU, serial, and its flash compiled for the host on every core)
on a bounded sample: the same case at 40^3, the same step window W+1..W+K;
`same_window_40` puts the GPU's FP64 graph on that sample beside it.
With N > 1 ranks (torchrun) the case is split into z-slabs, one per GPU, with a
halo exchange over NCCL after each recovery (strong scaling);
`--decompose replicas` runs N independent copies instead (weak scaling).
"""
import argparse
import contextlib
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mcell-steps/s at 160³, plain FP64 vs mixed/batched; adjoint/forward time"
UNIT = "Mcell-steps/s"
# Per-unit figures of the dominant kernel (the flash: its one-thread-per-cell
# single-phase pass, with the work queue for the cells the two-phase bound keeps),
# each per PR phase evaluation (the device counter the flash reports; a gas
# probe's root check decided without the root solve is not one), from ncu
# captures of one recovery of the impingement flow at 80^3, steps 21-22: FP64
# FLOPs = 2 DFMA + DADD + DMUL thread instructions, and DRAM read+write bytes
# (more cells than resident threads, as at 160^3, so the pass's stack frames do
# not stay in L2). Both include the single-phase pass's own formation of the
# flash inputs from the conserved rows and the seeds.
FLOPS_PER_PHASE_EVAL = 652.3
FLASH_BYTES_PER_CELL = 40 + 24 + 184 + 56
DRAM_BYTES_PER_PHASE_EVAL = 196.7
VISCOSITY, CONDUCTIVITY, WALE_CW, DT = 1.821e-5, 0.02587, 0.325, 1e-8
REFERENCE_SAMPLE = 40  # cube size of the reference CPU arm's bounded sample


def load_package():
    import importlib.util
    name = "spuma_multiphysics_b200"
    if name not in sys.modules:
        pkg = ROOT / "spuma-multiphysics_b200"
        spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py", submodule_search_locations=[str(pkg)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def step_kernels(stream, launch):
    """Kernels one step launches: `launch` (the step's launches, as a step graph
    records them) captured into a throwaway CUDA graph that is never replayed,
    and its kernel nodes counted through the driver API. None when that fails."""
    import torch
    try:
        cuda = C.CDLL("libcuda.so.1")
        g = torch.cuda.CUDAGraph(keep_graph=True)
        with torch.cuda.graph(g, stream=stream):
            launch()
        handle = C.c_void_p(g.raw_cuda_graph())
        count = C.c_size_t(0)
        if cuda.cuGraphGetNodes(handle, None, C.byref(count)):
            return None
        nodes = (C.c_void_p * count.value)()
        if count.value and cuda.cuGraphGetNodes(handle, nodes, C.byref(count)):
            return None
        kind, total = C.c_int(), 0
        for node in nodes[:count.value]:
            if cuda.cuGraphNodeGetType(C.c_void_p(node), C.byref(kind)):
                return None
            total += kind.value == 0  # CU_GRAPH_NODE_TYPE_KERNEL
        del g
        return total
    except (OSError, AttributeError, RuntimeError, TypeError):
        return None


def workload(n, precision="FP64 (state, transport and flash)"):
    q_mb = 5 * 8 * n ** 3 / 1e6
    return {"workload": f"N2O impingement {n}^3 ({n ** 3:,} cells), 40 bar ambient, 2 liquid inlets, "
                        f"viscous + conduction + WALE, SSPRK2 + 2 HEM UV flashes per step, dt=1e-8 s",
            "cells": n ** 3, "faces": 3 * n * n * (n - 1) + 6 * n * n, "species": 1, "variables": 5,
            "flux": "HLL", "precision": precision,
            "l2": f"no flush: the step's inputs are larger than L2 (q alone {q_mb:.0f} MB, thermo states "
                  f"{176 * n ** 3 / 1e6:.0f} MB)" if q_mb > 126 else "inputs smaller than L2 (not a timed headline)"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.proc, self.lines = str(index), None, []
        try:
            import torch
            self.index = f"GPU-{torch.cuda.get_device_properties(int(index)).uuid}"
        except Exception:
            pass

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.index, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the sampler's start-up takes longer than a short timed region: wait for its
            # first line and keep only the samples taken after it
            deadline = time.perf_counter() + 5
            while not self.lines and self.proc.poll() is None and time.perf_counter() < deadline:
                time.sleep(0.01)
            self.lines.clear()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, val in zip(names, parts[3:7]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(x, world, device=None):
    """Maximum of a per-rank float over all ranks (the job's time is the slowest
    rank's); identity for one rank. Works on NCCL (device tensor) and gloo (host)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def measured_peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        return {}


def fp64_peak(lib, torch):
    """Measured FP64 FMA rate (TFLOP/s) with the library's FMA-chain probe."""
    scratch = torch.zeros(148 * 64, dtype=torch.float64, device="cuda")
    flops = C.c_double()
    s = torch.cuda.current_stream()
    lib.rb200_probe_fp64_fma_v1.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                            C.POINTER(C.c_double)]
    for _ in range(2):
        lib.rb200_probe_fp64_fma_v1(148 * 8, 256, 2000, scratch.data_ptr(), s.cuda_stream, C.byref(flops))
    best = 0.0
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        lib.rb200_probe_fp64_fma_v1(148 * 8, 256, 2000, scratch.data_ptr(), s.cuda_stream, C.byref(flops))
        b.record(s)
        b.synchronize()
        best = max(best, flops.value / (a.elapsed_time(b) * 1e-3) / 1e12)
    return best


class HostPath:
    """The reference solver's call pattern (ReactiveFoam.C:961-1019, transportStage
    :651-661, stableStep :798-812) on this library with host arrays: q and the
    thermo states cross PCIe every stage, exactly as the reference drop-in runs.
    The caller's arrays are pinned (page-locked) host memory and its own
    bookkeeping (transport-state compaction with the primitives, the flash
    inputs, the step-start state copies) runs through the library's parallel
    host helpers (reactive_b200_host_*_v3), as the solver's own parallel loops."""

    def __init__(self, pkg, faces, volume, flow, fixed_q):
        import torch
        from spuma_multiphysics_b200 import _abi as A
        self.torch = torch
        self.A, self.lib = A, pkg._lib.load()
        self.cells = n = len(volume)
        self._pins = []
        self.q = self._pinned((n, 5), np.float64)
        self.q[:] = flow.conserved()
        self.states = self._pinned((n,), A.THERMO_DTYPE)
        self.states[:] = flow.states()
        self.start = self._pinned((n,), A.THERMO_DTYPE)
        self.seeds = self._pinned((n,), A.THERMO_DTYPE)
        self.tr = self._pinned((n,), A.STATE_DTYPE)
        self.prim = self._pinned((n, 4), np.float64)
        self.rho = self._pinned((n,), np.float64)
        self.e = self._pinned((n,), np.float64)
        self.ok = self._pinned((n,), np.int32)
        # the seed copy of a stage runs beside the transport stage it does not depend on
        import concurrent.futures
        self._pool = concurrent.futures.ThreadPoolExecutor(1)
        self.hem = flow.hem
        cfg = A.Config(n, 1, 5, len(faces), len(fixed_q), VISCOSITY, CONDUCTIVITY, 0.0, 1.1, 1.6e11, 0)
        fixed_tr = np.frombuffer(flow.tr[n:].cpu().numpy().tobytes(), dtype=A.STATE_DTYPE).copy()
        opts = A.OptionsV2(1, C.sizeof(A.OptionsV2), 256, 0, b"0" * 64)
        err = C.create_string_buffer(2048)
        self.faces = np.ascontiguousarray(faces)
        self.volume = np.ascontiguousarray(volume)
        self.fixed_q = np.ascontiguousarray(fixed_q, dtype=np.float64)
        h = self.lib.reactive_transport_create_v2(1, C.byref(cfg), C.byref(opts), A.dptr(self.volume),
                                                  self.faces.ctypes.data_as(C.POINTER(A.Face)),
                                                  A.dptr(self.fixed_q), fixed_tr.ctypes.data_as(C.POINTER(A.State)),
                                                  None, None, err, len(err))
        assert h, err.value
        self.t = C.c_void_p(h)
        wale = A.WaleOptions(1, C.sizeof(A.WaleOptions), WALE_CW)
        assert self.lib.reactive_transport_set_wale_v1(self.t, C.byref(wale)) == 0
        self.version, self.attempt = 0, 0
        self.h2d = self.d2h = 0
        self.library_s = 0.0
        self.library_calls = {}

    def _pinned(self, shape, dtype):
        dtype = np.dtype(dtype)
        t = self.torch.empty(int(np.prod(shape)) * dtype.itemsize, dtype=self.torch.uint8, pin_memory=True)
        self._pins.append(t)
        return t.numpy().view(dtype).reshape(shape)

    def _copy(self, dst, src):
        """dst[:] = src for host arrays (the library's parallel host copy)."""
        assert self.lib.reactive_b200_host_copy_v3(dst.ctypes.data, src.ctypes.data, src.nbytes) == 0
        return dst

    def _compact(self, states):
        """Transport states (p, T, rho, cv, frozen sound, gas mass) of thermo
        states and the primitives (rho, u) from them and q, in one parallel pass."""
        assert self.lib.reactive_b200_host_transport_states_v3(
            states.ctypes.data, self.cells, self.A.dptr(self.q), 5, 1, self.tr.ctypes.data,
            self.prim.ctypes.data) == 0
        return self.tr

    def _primitives(self, tr):
        return self.prim

    def _energy(self):
        assert self.lib.reactive_b200_host_recovery_inputs_v3(self.A.dptr(self.q), self.cells, 5, 1,
                                                             self.A.dptr(self.rho), self.A.dptr(self.e)) == 0

    def _check(self, rc):
        if rc:
            raise RuntimeError(self.lib.reactive_transport_error(self.t).decode())

    def _call(self, fn, *args):
        """One library call, its wall time added to library_s and to its entry's share."""
        t0 = time.perf_counter()
        try:
            return fn(*args)
        finally:
            dt = time.perf_counter() - t0
            self.library_s += dt
            name = getattr(fn, "__name__", "call").replace("reactive_transport_", "").replace("reactive_gpu_hem_", "")
            self.library_calls[name] = self.library_calls.get(name, 0.0) + dt

    def step(self, dt):
        A, lib, t, call = self.A, self.lib, self.t, self._call
        # the step-start states stay untouched for the whole step; each flash
        # works in place on its own copy of them (ReactiveFoam.C:1011)
        start = self.states
        self.states, self.start = self.start, start
        dtc = C.c_double()
        tr0 = self._compact(start)
        prim = self._primitives(tr0)
        self._check(call(lib.reactive_transport_stable_step_primitives, t,
                         prim.ctypes.data_as(C.POINTER(A.Primitive)), tr0.ctypes.data_as(C.POINTER(A.State)), .5,
                         dt, C.byref(dtc)))
        self.h2d += tr0.nbytes + prim.nbytes
        self.attempt += 1
        self._check(call(lib.reactive_transport_begin_attempt, t, b"0" * 64, self.attempt))
        self.version += 1
        self._check(call(lib.reactive_transport_upload_conserved, t, A.dptr(self.q), self.version))
        self.h2d += self.q.nbytes
        br = np.zeros(5)
        stage_states = None
        tr = tr0  # the step-start states' transport states, compacted once for the CFL query and stage 0
        for stage in (0, 1):
            out = self.seeds if stage == 0 else self.states
            copied = self._pool.submit(self._copy, out, start)
            before = A.Token(self.attempt, stage, self.version)
            self.version += 1
            after = A.Token(self.attempt, stage + 1, self.version)
            try:
                self._check(call(lib.reactive_transport_advance_resident_v2, t, before, after,
                                 tr.ctypes.data_as(C.POINTER(A.State)), None, None, None, dt, A.dptr(br)))
                self._check(call(lib.reactive_transport_download_conserved, t, after, A.dptr(self.q)))
            finally:
                copied.result()
            self.h2d += tr.nbytes
            self.d2h += self.q.nbytes
            self._energy()
            ok, _ = call(self.hem.run, self.rho, self.e, out, self.ok)
            if not ok.all():
                raise RuntimeError("HEM recovery failed")
            self.h2d += self.rho.nbytes + self.e.nbytes + out.nbytes
            self.d2h += out.nbytes + ok.nbytes
            if stage == 0:
                stage_states = out
                tr = self._compact(stage_states)  # reused by stage 1
                prim = self._primitives(tr)
                self._check(call(lib.reactive_transport_stable_step_primitives, t,
                                 prim.ctypes.data_as(C.POINTER(A.Primitive)), tr.ctypes.data_as(C.POINTER(A.State)),
                                 .5, dt, C.byref(dtc)))
                self.h2d += tr.nbytes + prim.nbytes
        self._check(call(lib.reactive_transport_end_attempt, t, self.attempt, 1))

    def close(self):
        self._pool.shutdown()
        self.lib.reactive_transport_destroy(self.t)


def run_slab(args, rank, world):
    """The 160^3 case decomposed into z-slabs over the ranks (strong scaling):
    each rank steps its own layers plus two halo layers (the headline's FP64
    form, each half step a captured graph), with the halo exchange over NCCL
    after each recovery; the CFL minimum over ranks is checked after the run.
    One rank runs the undivided box through the same code."""
    import torch
    load_package()
    from spuma_multiphysics_b200 import cases
    from spuma_multiphysics_b200.slab import SlabFlow, global_cfl
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    n = args.size
    init = cases.impingement(n, seed=2026)
    slab = SlabFlow(n, rank, world, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"],
                    viscosity=VISCOSITY, conductivity=CONDUCTIVITY, wale_cw=WALE_CW)
    f = slab.flow
    pkg = load_package()
    stats0 = pkg._abi.Stats()
    f.lib.reactive_transport_stats(f.transport, C.byref(stats0))
    slab.capture(DT)
    stats1 = pkg._abi.Stats()
    f.lib.reactive_transport_stats(f.transport, C.byref(stats1))
    # transport launches counted by the handle while capturing both half steps,
    # plus five per flash (single-phase pass, queue, selection, restart queue,
    # restart selection)
    launches_per_step = int(stats1.kernelLaunches - stats0.kernelLaunches) + 2 * 5

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        slab.step(DT)
    barrier()
    sampler = ClockSampler(torch.cuda.current_device())
    with sampler:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(f.stream)
        for _ in range(args.steps):
            slab.step(DT)
        b.record(f.stream)
        barrier()
    ms = max_over_ranks(a.elapsed_time(b) / args.steps, world, "cuda")
    cfl = global_cfl(slab, world)
    failed = int((f.success[f.own[0]:f.own[1]] == 0).sum().item())
    failed = int(max_over_ranks(float(failed), world, "cuda"))
    if failed or not DT <= cfl * (1 + 1e-10):
        raise RuntimeError(f"slab step failed: {failed} failed recoveries, CFL step {cfl}")
    L = slab.layout
    line = {"metric": METRIC, "value": n ** 3 / (ms * 1e-3) / 1e6, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {**workload(n), "parallelism": f"z-slabs x{world} (own layers + 2 halo layers, "
                                                     f"NCCL halo exchange after each recovery)",
                       "own_layers_rank0": L.z1 - L.z0},
            "e2e": None, "roofline": None, "cpu_baseline": None, "clocks": sampler.summary(),
            "gpu_launches": launches_per_step * args.steps}
    slab.close()
    return line


def run_ours(args, rank, world):
    import torch
    pkg = load_package()
    from spuma_multiphysics_b200 import cases
    from spuma_multiphysics_b200.flow import Flow, field_errors
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    n = args.size
    t0 = time.time()
    faces, volume = cases.cartesian_faces(n)
    init = cases.impingement(n, seed=2026 + rank)
    kw = dict(viscosity=VISCOSITY, conductivity=CONDUCTIVITY, wale_cw=WALE_CW)
    case = (faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"])
    # the headline form: FP64 structured transport + work-queue FP64 flash, one CUDA graph per step
    flow = Flow(*case, **kw)
    # the same step with FP32 transport arithmetic (compensated sums into the FP64 state)
    mixed = Flow(*case, precision="mixed", **kw)
    setup_s = time.time() - t0
    lib = flow.lib
    rank_dev = int(os.environ.get("LOCAL_RANK", 0))

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks_(x):
        return max_over_ranks(x, world, "cuda")

    def timed_graph_steps(f, sample_clocks, snapshot=None, steps=None):
        """W warm-up then K timed graph replays of flow f (CUDA events on its
        stream); `snapshot` (a list) receives the state the timed steps start from."""
        steps = args.steps if steps is None else steps
        f.capture(DT)
        for _ in range(args.warmup):
            f.step(DT)
        f.check(DT)
        if snapshot is not None:
            snapshot[:] = [f.qn.clone(), f.sn.clone(), f.tr.clone()]
        barrier()
        sampler = ClockSampler(rank_dev) if sample_clocks else contextlib.nullcontext()
        with sampler as clocks_:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.nvtx.range_push("timed_step")
            a.record(f.stream)
            for _ in range(steps):
                f.step(DT)
            b.record(f.stream)
            barrier()
            torch.cuda.nvtx.range_pop()
        f.check(DT)
        return max_over_ranks_(a.elapsed_time(b) / steps), clocks_

    # kernels launched per step: the kernel nodes of the step's launches captured
    # once more (else the transport's call count plus five per flash:
    # single-phase pass, queue, selection, restart queue, restart selection)
    stats0 = pkg._abi.Stats()
    lib.reactive_transport_stats(flow.transport, C.byref(stats0))
    flow.capture(DT)
    stats1 = pkg._abi.Stats()
    lib.reactive_transport_stats(flow.transport, C.byref(stats1))
    launches_per_step = (step_kernels(flow.stream, lambda: flow._launch_step(DT))
                         or int(stats1.kernelLaunches - stats0.kernelLaunches) + 2 * 5)
    tuned = {"fp64": flow.autotune(), "mixed": mixed.autotune()}
    if args.stage_shape is not None:  # a fixed stage launch shape (e.g. for a profile of one stage kernel)
        for form, f in (("fp64", flow), ("mixed", mixed)):
            shapes = (C.c_uint * 3)(args.stage_shape, tuned[form]["gradient_block"], tuned[form]["cfl_block"])
            assert f.lib.reactive_transport_launch_shapes_v3(f.transport, shapes, None) == 0
            f.graph = None
            tuned[form]["stage_block"] = args.stage_shape
    start = []
    graph_ms, clocks = timed_graph_steps(flow, True, start)
    mixed_ms, _ = timed_graph_steps(mixed, False)
    # both runs took the same W + K steps from the same state
    mixed_errors = field_errors(mixed.conserved(), mixed.states(), flow.conserved(), flow.states())
    mixed.close()
    # the flash alone (the headline's work-queue search) on exactly the states of
    # the timed steps: the headline flow goes back to the state its timed steps
    # started from and takes the same K steps again launch by launch (the same
    # kernels, so the same trajectory), with CUDA events on the flash's stream
    # around each step's first recovery and its work counters read around it
    stream = flow.stream
    for dst, src in zip((flow.qn, flow.sn, flow.tr), start):
        dst.copy_(src)
    del start
    times, flash_phase_evals = [], 0.0
    for _ in range(args.steps):
        flow.stage0(DT)
        flow.hem.counters(stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("flash_alone")
        e0.record(stream)
        flow._flash(flow.q1, flow.s1)
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        flash_phase_evals += flow.hem.counters(stream.cuda_stream).phaseEvaluations
        with torch.cuda.stream(stream):
            flow._launch_half(DT, 1)
        times.append((e0, e1))
    stream.synchronize()
    flash_ms = statistics.mean(x.elapsed_time(y) for x, y in times)
    flash_phase_evals /= len(times)
    flow.check(DT)
    # the reference's alternative search policy (closureSearch stableGasPrune,
    # ReactiveFoam.C:332-334): two-phase seeds skipped where the all-gas candidate
    # is stable; reported beside the headline, which uses the default search
    pruned_ms = None
    if not args.skip_plain:
        from spuma_multiphysics_b200.thermo_data import pure_model
        pruned = Flow(*case, model=pure_model(stable_gas_prune=1), **kw)
        pruned.autotune()
        pruned_ms, _ = timed_graph_steps(pruned, False)
        pruned.close()
    # the same headline step with the flash's two-phase admissibility bound off
    # (every candidate solved; results are the same bits)
    exhaustive_ms = None
    if not args.skip_plain:
        full = Flow(*case, **kw)
        full.two_phase_bound(False)
        full.autotune()
        exhaustive_ms, _ = timed_graph_steps(full, False)
        full.close()
    cells = n ** 3
    value = world * cells / (graph_ms * 1e-3) / 1e6

    # ---- plain launches: FP64, kernels one by one, the plain one-thread-per-cell flash
    plain_ms = None
    plain_steps = min(args.steps, 3)  # about 1.4 s a step at 160^3
    if not args.skip_plain:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        a.record(stream)
        for _ in range(plain_steps):
            flow.step(DT, graph=False, per_cell=True)
        b.record(stream)
        barrier()
        plain_ms = max_over_ranks_(a.elapsed_time(b) / plain_steps)

    # ---- e2e through the reference-facing C ABI with host arrays
    e2e = None
    if not args.skip_e2e:
        host = HostPath(pkg, faces, volume, flow, init["fixed_q"])
        host.step(DT)  # warm-up
        host.h2d = host.d2h = 0
        host.library_s = 0.0
        host.library_calls = {}
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            host.step(DT)
        barrier()
        e2e_s = max_over_ranks_((time.perf_counter() - t0) / args.e2e_steps)
        library_s = host.library_s / args.e2e_steps
        e2e = {"value": world * cells / e2e_s / 1e6, "unit": UNIT, "ms_per_step": e2e_s * 1e3,
               "h2d_bytes_per_step": host.h2d // args.e2e_steps, "d2h_bytes_per_step": host.d2h // args.e2e_steps,
               "library_ms_per_step": library_s * 1e3, "caller_ms_per_step": (e2e_s - library_s) * 1e3,
               "library_calls_ms_per_step": {k: round(v * 1e3 / args.e2e_steps, 3)
                                             for k, v in sorted(host.library_calls.items())},
               "path": "the reference solver's calls with host arrays: stable_step_primitives, upload_conserved, "
                       "2 x (advance_resident_v2, download_conserved, reactive_gpu_hem_run_v1); library = time "
                       "inside those calls (their PCIe copies included), caller = the caller's own host "
                       "bookkeeping (state compaction, primitives, flash inputs, state copies) through the "
                       "library's parallel host helpers"}
        host.close()

    # ---- the reference CPU arm's bounded sample, on the GPU: 40^3, same step window
    same_window = None
    if not args.skip_cpu:
        fs, vs = cases.cartesian_faces(REFERENCE_SAMPLE)
        i40 = cases.impingement(REFERENCE_SAMPLE, seed=2026)
        f40 = Flow(fs, vs, i40["q"], i40["guess"], i40["fixed_q"], i40["fixed_guess"], **kw)
        ms40, _ = timed_graph_steps(f40, False)
        f40.close()
        same_window = {"cells": REFERENCE_SAMPLE ** 3, "gpu_fp64_graph_ms_per_step": ms40,
                       "gpu_fp64_graph_value": REFERENCE_SAMPLE ** 3 / (ms40 * 1e-3) / 1e6,
                       "steps": f"{args.warmup + 1}-{args.warmup + args.steps}"}

    peaks = measured_peaks()
    fp64 = fp64_peak(lib, torch)
    roofline = None
    if flash_ms:
        flops_per_eval = args.flops_per_phase_eval
        achieved = flops_per_eval * flash_phase_evals / (flash_ms * 1e-3) / 1e12 if flops_per_eval else None
        roofline = {"bound": "fp64", "achieved": achieved, "peak": fp64, "unit": "TFLOP/s",
                    "frac": achieved / fp64 if achieved else None,
                    "traffic": args.dram_bytes_per_phase_eval * flash_phase_evals,
                    "peak_source": "measured in this run (FP64 FMA-chain probe)",
                    "kernel": "HEM flash, one recovery of all cells (passSinglePhase + passQueue + selection + "
                              "restarts): the first recovery of each timed step, re-run from the timed steps' "
                              "start state",
                    "traffic_note": "DRAM bytes per launch, ncu per-phase-evaluation figure x this launch's "
                                    "phase evaluations",
                    "ms_per_launch": flash_ms, "phase_evaluations_per_launch": flash_phase_evals,
                    "flops_per_phase_evaluation": flops_per_eval,
                    # a recovery's own bytes: the conserved row (40 B) and the seed's p, T and
                    # liquid mass (24 B) read, the thermo state (184 B) and transport state
                    # (56 B) written
                    "algorithmic_bytes_per_launch": FLASH_BYTES_PER_CELL * cells,
                    "traffic_over_algorithmic": args.dram_bytes_per_phase_eval * flash_phase_evals
                    / (FLASH_BYTES_PER_CELL * cells)}
    # HBM roofline of the whole step (algorithmic bytes per cell-step, FP64, nv=5, 4 transport thermo fields)
    bytes_per_cell_step = 8 * (5 * 5 + 2 * 4) + 2 * (8 * 5 + 80)
    hbm = peaks.get("hbm_gbs", 6650.0)
    step_roofline = {"bound": "hbm", "bytes_per_cell_step": bytes_per_cell_step,
                     "achieved": value * 1e6 * bytes_per_cell_step / 1e9, "peak": hbm, "unit": "GB/s",
                     "frac": value * 1e6 * bytes_per_cell_step / 1e9 / hbm,
                     "peak_source": "of measured" if "hbm_gbs" in peaks else "of fallback"}
    adjoint = None if args.skip_adjoint else {
        "hem": hem_adjoint_run(flow, n, steps=10, every=10),
        "ideal_gas_blast_64": adjoint_run(64, steps=50, every=10, probes=0)}
    cpu = None
    if rank == 0 and not args.skip_cpu:
        _, cpu = cpu_reference(args.warmup, args.cpu_steps, REFERENCE_SAMPLE)
        same_window["reference_cpu_value"] = cpu["value"]
    clock = clocks.summary()
    mixed_value = world * cells / (mixed_ms * 1e-3) / 1e6
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": graph_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded N2O impingement initial state)",
            "mixed": {"value": mixed_value, "ms_per_step": mixed_ms, "over_fp64_graph": mixed_value / value,
                      "over_plain_fp64": graph_ms and plain_ms and plain_ms / mixed_ms,
                      "field_error_vs_fp64": {"steps": args.warmup + args.steps, **mixed_errors}},
            "plain_fp64": {"value": world * cells / (plain_ms * 1e-3) / 1e6 if plain_ms else None,
                           "ms_per_step": plain_ms, "steps": plain_steps if plain_ms else None},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "same_window_40": same_window,
            "clocks": clock, "gpu_launches": launches_per_step * args.steps,
            "config": {**workload(n, "FP64 (state, transport and flash)"),
                       "parallelism": f"{world} independent replicas (one per GPU)",
                       "autotuned_launch_shapes": tuned},
            "form": "FP64 structured transport, work-queue FP64 flash with the two-phase admissibility bound, one "
                    "CUDA graph per step; mixed = the same with FP32 transport arithmetic and compensated sums; "
                    "plain_fp64 = kernels one by one, flash one thread per cell (no work queue, no bound)",
            "roofline_step_hbm": step_roofline,
            "stable_gas_prune_graph": None if pruned_ms is None else {
                "ms_per_step": pruned_ms, "value": world * cells / (pruned_ms * 1e-3) / 1e6},
            "exhaustive_search_graph": None if exhaustive_ms is None else {
                "ms_per_step": exhaustive_ms, "value": world * cells / (exhaustive_ms * 1e-3) / 1e6},
            "adjoint": adjoint, "fp64_peak_tflops": fp64, "setup_s": setup_s}
    flow.close()
    return line


def cpu_reference(warmup, steps, n=40):
    """The reference's own CPU code on the same case at n^3 (a bounded sample of
    the 160^3 workload): its transport built for the CPU (serial by construction)
    and its flash compiled for the host, threaded over all cores. The sample
    advances `warmup` steps untimed and times the next `steps` steps, the same
    step window (W+1 .. W+K) that the GPU arms time. Returns the per-step
    samples and the baseline record."""
    sys.path.insert(0, str(ROOT / "tests"))
    load_package()
    from spuma_multiphysics_b200 import cases, thermo_data as td
    from oracle import oracle
    import rk_oracle
    threads = oracle.cpu_threads()
    faces, volume = cases.cartesian_faces(n)
    init = cases.impingement(n, seed=2026)
    image = td.model_bytes(td.pure_model())
    ref = rk_oracle.ReferenceFlow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"],
                                  VISCOSITY, CONDUCTIVITY, WALE_CW, image, threads=threads)
    for _ in range(warmup):
        ref.step(DT)
    samples = []
    for _ in range(steps):
        t0 = time.perf_counter()
        ref.step(DT)
        samples.append(time.perf_counter() - t0)
    ref.close()
    s = statistics.mean(samples)
    return samples, {"value": n ** 3 / s / 1e6, "unit": UNIT, "cores": threads, "kind": "reference",
                     "sample": f"{n}^3 ({n ** 3:,} cells) sample of the same case, steps {warmup + 1}-{warmup + steps} "
                               f"timed (the GPU arms' window); transport serial (reference CPU build), flash on "
                               f"{threads} threads",
                     "seconds_per_step": s}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    n = REFERENCE_SAMPLE
    samples, cpu = cpu_reference(args.warmup, args.steps, n)
    value = cpu["value"]
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(samples),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded N2O impingement initial state)", "impl": "reference",
            "cpu_baseline": cpu, "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                         "d2h_bytes_per_step": 0},
            "config": {**workload(n, "FP64 (the reference's CPU code)"),
                       "sample_of": "the 160^3 impingement case (per-cell throughput; same physics, dt and step "
                                    "window, 2 mm cells instead of 0.5 mm)",
                       "parallelism": "reference CPU code on host cores"}}


def run_flash_batch(args):
    """Standalone batched HEM flash (the 4,096,000-state configuration when
    --flash-batch 4096000): states generated forward from a seed, 60% saturated
    two-phase, 40% single-phase; seeds are the generating states."""
    import torch
    pkg = load_package()
    from spuma_multiphysics_b200 import _abi as A, cases, thermo_data as td
    from spuma_multiphysics_b200.hem import GpuHem
    t0 = time.time()
    if args.flash_checkpoint:
        # the cells of a committed checkpoint, seeded by their committed states
        from spuma_multiphysics_b200 import checkpoint
        q, e, guess, _ = checkpoint.flash_batch(args.flash_checkpoint)
        n = len(q)
        workload = f"batched HEM UV flash of the {n:,} cells of checkpoint {Path(args.flash_checkpoint).name}"
        data = "checkpoint cells"
    else:
        n = args.flash_batch
        q, e, guess = cases.flash_batch(n, seed=20260303, saturation_levels=65536 if n > 1000000 else 0)
        workload = f"batched HEM UV flash, {n:,} pure-N2O cells, 60% two-phase"
        data = "synthetic (seeded pure-N2O states generated forward)"
    gen_s = time.time() - t0
    hem = GpuHem(model=td.pure_model(stable_gas_prune=args.flash_prune), capacity=n)
    dev = torch.device("cuda")
    cons = torch.zeros((5, n), dtype=torch.float64, device=dev)
    cons[0] = torch.from_numpy(q).to(dev)
    cons[4] = torch.from_numpy(e).to(dev)
    seed = torch.from_numpy(guess.view(np.uint8).copy()).to(dev)
    state = torch.zeros_like(seed)
    ok = torch.zeros(n, dtype=torch.int32, device=dev)
    s = torch.cuda.Stream()
    for _ in range(args.warmup):
        hem.run_device(cons, n, n, 5, seed, state, None, ok, s.cuda_stream)
    s.synchronize()
    hem.counters(s.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clocks:
        a.record(s)
        for _ in range(args.steps):
            hem.run_device(cons, n, n, 5, seed, state, None, ok, s.cuda_stream)
        b.record(s)
        s.synchronize()
    ms = a.elapsed_time(b) / args.steps
    prof = hem.counters(s.cuda_stream)
    out = state.cpu().numpy().view(A.THERMO_DTYPE)
    labels = cases.phase_label(out)
    iters = out["iterations"]
    generated_two = guess["liquidMass"][:, 0] > 0  # generated on the saturation curve with quality in [0, 1)
    return {"metric": "HEM UV flash calls/s (standalone batch)", "value": n / (ms * 1e-3), "unit": "flash/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "dtype": "f64", "data": data,
            "config": {"workload": workload, "stableGasPrune": args.flash_prune},
            "succeeded": int(ok.sum().item()), "labels": np.bincount(labels, minlength=3).tolist(),
            "iterations": {"p50": float(np.percentile(iters, 50)), "p90": float(np.percentile(iters, 90)),
                           "p99": float(np.percentile(iters, 99)), "max": int(iters.max()),
                           "histogram": np.bincount(iters.clip(0, 31), minlength=32).tolist()},
            "generated_phase_agreement": None if args.flash_checkpoint else {
                "two_phase_recovered_two_phase": float(np.mean(labels[generated_two] == 2)),
                "single_phase_recovered_single_phase": float(np.mean(labels[~generated_two] != 2))},
            "cpu_label_agreement": "bit-exact labels against the reference flash on seeded samples "
                                   "(tests/test_flash_gpu.py)",
            "phase_evaluations_per_cell": prof.phaseEvaluations / (args.steps * n),
            "residual_evaluations_per_cell": prof.residualEvaluations / (args.steps * n),
            "clocks": clocks.summary(), "generation_s": gen_s}


def hem_adjoint_run(flow, n, steps=10, every=10):
    """The adjoint of the last `steps` steps of the 160^3 HEM case (config 5):
    from the flow's current state, `steps` FP64 SSPRK2 + HEM steps recorded
    with checkpoints every `every` steps, loss = N2O mass in the off-centre
    sub-box [n/2, 3n/4) x [n/4, n/2) x [n/4, n/2), gradient with respect to the
    state `steps` steps earlier by the hand-written adjoint (transport VJP with
    viscous/WALE terms, flash by the implicit function theorem). Forward alone
    and forward + adjoint timed with CUDA events."""
    import torch
    from spuma_multiphysics_b200.adjoint import HemStep, hem_rollout
    stepper = HemStep(flow)
    q0, s0 = flow.qn.clone(), flow.sn.clone()
    k, j, i = np.indices((n, n, n))
    sub = ((i >= n // 2) & (i < 3 * n // 4) & (j >= n // 4) & (j < n // 2) & (k >= n // 4) & (k < n // 2)).ravel()
    weight = torch.zeros_like(q0)
    weight[0, :flow.cells] = torch.from_numpy(sub.astype(np.float64) * (0.08 / n) ** 3).cuda()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    # untimed warm-up of both paths (first launches, allocator growth, autograd set-up)
    qw = q0.clone().requires_grad_(True)
    torch.autograd.grad((hem_rollout(stepper, qw, s0, steps, DT, every)[0] * weight).sum(), qw)
    del qw
    with torch.no_grad():
        hem_rollout(stepper, q0, s0, steps, DT, every)
        ev[0].record()
        hem_rollout(stepper, q0, s0, steps, DT, every)
        ev[1].record()
    qg = q0.clone().requires_grad_(True)
    ev[2].record()
    out, _ = hem_rollout(stepper, qg, s0, steps, DT, every)
    (grad,) = torch.autograd.grad((out * weight).sum(), qg)
    ev[3].record()
    torch.cuda.synchronize()
    stepper.check()
    fwd, both = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3])
    return {"workload": f"adjoint of the last {steps} steps of the {n}^3 HEM case (viscous + WALE, flash by IFT), "
                        f"checkpoints every {every}",
            "forward_ms_per_step": fwd / steps, "forward_plus_adjoint_ms_per_step": both / steps,
            "adjoint_ms_per_step": (both - fwd) / steps, "adjoint_over_forward": (both - fwd) / fwd,
            "gradient_norm": float(grad.norm().item())}


def adjoint_run(n=64, steps=50, every=10, probes=0, seed=11):
    """The two-species ideal-gas blast box (N2O sphere at 10 bar in N2 at 1 bar,
    300 K, +-0.5% density noise, dx = 1 mm, transmissive sides), `steps` fixed
    SSPRK2 steps (dt = 0.3 x the initial CFL step), loss = N2O mass in the
    off-centre 16^3 sub-box [40,56) x [24,40) x [24,40) (scaled to n). The
    gradient of the loss with respect to the initial density field and the
    driver pressure by the hand-written adjoint with checkpoints every `every`
    steps; timings of the forward alone and of forward + adjoint; with probes >
    0, central differences (h = 1e-6 relative) on that many random cells within
    the sub-box's domain of dependence and on the driver pressure."""
    import torch
    load_package()
    from spuma_multiphysics_b200 import cases
    from spuma_multiphysics_b200.adjoint import IdealGasBox, rollout
    spec = cases.blast_box(n, edge=n * 1e-3, radius=n * 0.25e-3)
    box = IdealGasBox(spec["faces"], spec["volume"], spec["species"])
    rho0 = torch.from_numpy(spec["rho0"]).cuda()
    p_drive = torch.tensor(spec["p_drive"], dtype=torch.float64, device="cuda")
    dt = .3 * box.stable_dt(cases.blast_initial(spec, rho0, p_drive, xp=torch))
    lo, hi = int(n * 40 / 64), int(n * 56 / 64)
    lo2, hi2 = int(n * 24 / 64), int(n * 40 / 64)
    k, j, i = np.indices((n, n, n))
    sub = ((i >= lo) & (i < hi) & (j >= lo2) & (j < hi2) & (k >= lo2) & (k < hi2)).ravel()
    mask = torch.from_numpy(sub.astype(np.float64)).cuda() * box.volume

    def loss(r, p):
        return (rollout(box, cases.blast_initial(spec, r, p, xp=torch), steps, dt, every)[0] * mask).sum()

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    # warm-up of both paths (the recorded one sets up autograd and checkpointing)
    rw = rho0.clone().requires_grad_(True)
    torch.autograd.grad(loss(rw, p_drive), rw)
    with torch.no_grad():
        loss(rho0, p_drive)
        ev[0].record()
        J = loss(rho0, p_drive)
        ev[1].record()
    r = rho0.clone().requires_grad_(True)
    p = p_drive.clone().requires_grad_(True)
    ev[2].record()
    Jg = loss(r, p)
    ev[3].record()
    g_rho, g_p = torch.autograd.grad(Jg, (r, p))
    ev[4].record()
    torch.cuda.synchronize()
    box.check()
    fwd = ev[0].elapsed_time(ev[1])
    rec, bwd = ev[2].elapsed_time(ev[3]), ev[3].elapsed_time(ev[4])
    out = {"workload": f"ideal-gas N2O/N2 blast box {n}^3, {steps} SSPRK2 steps, checkpoints every {every}",
           "dt": dt, "loss": J.item(), "forward_ms_per_step": fwd / steps,
           "recorded_forward_ms_per_step": rec / steps, "adjoint_ms_per_step": bwd / steps,
           "adjoint_over_forward": bwd / fwd, "forward_plus_adjoint_over_forward": (rec + bwd) / fwd,
           "dJ_dp_drive": g_p.item()}
    if probes:
        rng = np.random.default_rng(seed)
        reach = int(np.ceil(steps * .3 * 1.2)) + 1  # CFL 0.3: at most ~0.4 cells per step either way
        near = np.flatnonzero((i >= lo - reach) & (i < hi + reach) & (j >= lo2 - reach) & (j < hi2 + reach)
                              & (k >= lo2 - reach) & (k < hi2 + reach))
        cells = rng.choice(near, probes, replace=False)
        fd = []
        with torch.no_grad():
            for c in cells:
                h = 1e-6 * float(rho0[c])
                rp, rm = rho0.clone(), rho0.clone()
                rp[c] += h
                rm[c] -= h
                fd.append((loss(rp, p_drive) - loss(rm, p_drive)).item() / (2 * h))
            hp = 1e-6 * spec["p_drive"]
            fd_p = (loss(rho0, p_drive + hp) - loss(rho0, p_drive - hp)).item() / (2 * hp)
        box.check()
        g = g_rho[torch.as_tensor(cells)].cpu().numpy()
        fd = np.array(fd)
        big = np.abs(fd) > 1e-3 * np.abs(fd).max()
        out["finite_differences"] = {
            "probes": int(probes), "h": "1e-6 relative", "max_abs_gradient": float(np.abs(fd).max()),
            "scaled_error": float(np.max(np.abs(g - fd)) / np.abs(fd).max()),
            "relative_error_median": float(np.median(np.abs(g - fd)[big] / np.abs(fd[big]))),
            "relative_error_max": float(np.max(np.abs(g - fd)[big] / np.abs(fd[big]))),
            "p_drive_relative_error": abs(g_p.item() - fd_p) / abs(fd_p)}
    box.close()
    return out


def run_adjoint_check(args):
    line = {"metric": "adjoint gradient check and adjoint/forward time", "unit": "relative",
            "data": "synthetic (seeded ideal-gas blast box)",
            **adjoint_run(args.adjoint_check, steps=args.adjoint_steps, every=10, probes=32)}
    return line


def run_precision_study(args):
    """The 80^3 impingement case (viscosity, conduction, WALE) run in FP64 and in
    the mixed form side by side for --study-steps steps from the same state; the
    per-field error of the mixed run against the FP64 run (the FP64 device path is
    the one matched to the reference's CPU RK driver in the tests)."""
    import torch
    load_package()
    from spuma_multiphysics_b200 import cases
    from spuma_multiphysics_b200.flow import Flow, field_errors
    n, steps = args.precision_study, args.study_steps
    faces, volume = cases.cartesian_faces(n)
    init = cases.impingement(n, seed=2026)
    kw = dict(viscosity=VISCOSITY, conductivity=CONDUCTIVITY, wale_cw=WALE_CW)
    out = {}
    flows = {}
    for name in ("fp64", "mixed"):
        f = Flow(faces, volume, init["q"], init["guess"], init["fixed_q"], init["fixed_guess"], precision=name, **kw)
        f.capture(DT)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(f.stream)
        for _ in range(steps):
            f.step(DT)
        b.record(f.stream)
        f.check(DT)
        out[name] = {"ms_per_step": a.elapsed_time(b) / steps}
        flows[name] = f
    errors = field_errors(flows["mixed"].conserved(), flows["mixed"].states(), flows["fp64"].conserved(),
                          flows["fp64"].states())
    for f in flows.values():
        f.close()
    return {"metric": "per-field error of the mixed form against FP64 after the run", "unit": "relative",
            "config": {**workload(n, "FP64 and mixed side by side"), "steps": steps},
            "errors": errors, "error_definition": "max over cells of |mixed - fp64| / |fp64| (rho, rhoE, p, T); "
                                                  "momentum: max |mixed - fp64| / max |fp64|",
            "timing": out, "data": "synthetic (seeded N2O impingement initial state)"}


def main():
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--size", type=int, default=160)
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--skip-plain", action="store_true")
    p.add_argument("--skip-e2e", action="store_true")
    p.add_argument("--skip-cpu", action="store_true")
    p.add_argument("--cpu-steps", type=int, default=2,
                   help="timed steps of the CPU baseline sample (after --warmup untimed steps)")
    p.add_argument("--flops-per-phase-eval", type=float, default=FLOPS_PER_PHASE_EVAL,
                   help="FP64 FLOPs per PR phase evaluation of the flash kernels (from an ncu capture)")
    p.add_argument("--dram-bytes-per-phase-eval", type=float, default=DRAM_BYTES_PER_PHASE_EVAL,
                   help="DRAM bytes per PR phase evaluation of the flash kernels (from an ncu capture)")
    p.add_argument("--flash-batch", type=int, default=0, help="run the standalone batched flash on this many cells")
    p.add_argument("--flash-prune", type=int, default=0, help="the model's stableGasPrune flag for --flash-batch")
    p.add_argument("--flash-checkpoint", default=None,
                   help="flash the cells of this committed checkpoint time directory (the --flash-batch mode)")
    p.add_argument("--precision-study", type=int, default=0,
                   help="run FP64 and mixed side by side on this cube size and report per-field errors")
    p.add_argument("--study-steps", type=int, default=20)
    p.add_argument("--adjoint-check", type=int, default=0,
                   help="run the ideal-gas blast box adjoint check on this cube size")
    p.add_argument("--adjoint-steps", type=int, default=50)
    p.add_argument("--skip-adjoint", action="store_true")
    p.add_argument("--stage-shape", type=int, choices=(0, 1, 64, 96, 128), default=None,
                   help="fix the structured stage's launch shape after autotuning (0 tiled, 1 split stage, "
                        "64/96/128 per-cell block sizes); results do not depend on it")
    p.add_argument("--decompose", choices=("auto", "replicas", "slab"), default="auto",
                   help="N > 1: the case split into z-slabs with a halo exchange (strong scaling; the default) "
                        "or independent replicas (weak scaling); N = 1 runs the undivided case")
    args = p.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.flash_batch or args.flash_checkpoint:
            line = run_flash_batch(args)
        elif args.precision_study:
            line = run_precision_study(args)
        elif args.adjoint_check:
            line = run_adjoint_check(args)
        else:
            if args.impl == "reference":
                line = run_reference(args, rank, world)
            elif args.decompose == "slab" or (args.decompose == "auto" and world > 1):
                line = run_slab(args, rank, world)
            else:
                line = run_ours(args, rank, world)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()
    if rank == 0 and line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
