"""GPU: the reference's device-resident HEM batch (reactive_gpu_hem_run_resident_v1)
and host capillary batch (reactive_gpu_hem_run_v2) without a pressure jump: the
same states and flags as the host batch (run_v1) on the same cells, results
scattered to the named global cells, a failed cell returning its seed, and a
pressure jump or the frozen partition refused with a message."""
import ctypes as C

import numpy as np
import pytest
import torch

from spuma_multiphysics_b200 import _abi as A, _lib, cases
from spuma_multiphysics_b200.hem import GpuHem

pytestmark = pytest.mark.gpu

# a near-critical state the reference flash cannot recover (test_flash_gpu)
FAIL_Q, FAIL_E = 432.822060758171, 729723467.9575783
FAIL_P, FAIL_T = 7822403.962295835, 312.965328917707


def batch(n, seed):
    rho, e, guess = cases.flash_batch(n, seed=seed)[:3]
    rho, e = np.append(rho, FAIL_Q), np.append(e, FAIL_E)
    g = np.zeros(1, dtype=A.THERMO_DTYPE)
    g["p"], g["T"], g["rho"] = FAIL_P, FAIL_T, FAIL_Q
    return rho, e, np.concatenate([guess, g])


def test_resident_batch_matches_host_batch():
    rho, e, guess = batch(3000, 77)
    n = len(rho)
    rng = np.random.default_rng(9)
    total = n + 541
    order = rng.permutation(total)[:n].astype(np.uint32)
    q_g = np.zeros(total)
    e_g = np.zeros(total)
    seed_g = np.zeros(total, dtype=A.THERMO_DTYPE)
    q_g[order], e_g[order], seed_g[order] = rho, e, guess
    cap = np.zeros(total, dtype=A.CAPILLARY_DTYPE)
    cap["color"] = rng.uniform(0, 1, total)
    cap["equilibrium"] = 1
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()
    dq, de, dseed, dcap, dorder = dev(q_g), dev(e_g), dev(seed_g), dev(cap), dev(order)
    out = torch.zeros(total * A.HEM_OUTPUT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    lib = _lib.load()
    hem = GpuHem(capacity=n, resident=True)
    host = GpuHem(capacity=n)
    err = C.create_string_buffer(1024)
    try:
        prof = A.HemProfile(1, C.sizeof(A.HemProfile))
        assert lib.reactive_gpu_hem_run_resident_v1(hem.handle, dq.data_ptr(), de.data_ptr(), dseed.data_ptr(),
                                                    dcap.data_ptr(), dorder.data_ptr(), n, out.data_ptr(),
                                                    C.byref(prof), err, len(err)) == 0, err.value
        got = out.cpu().numpy().view(A.HEM_OUTPUT_DTYPE)
        exp = guess.copy()
        ok, _ = host.run(rho, e, exp)
        assert np.array_equal(got["success"][order], ok)
        assert got["state"][order].tobytes() == exp.tobytes()
        assert ok[-1] == 0 and got["state"][order[-1]].tobytes() == guess[-1:].tobytes()
        rest = np.setdiff1d(np.arange(total), order)
        assert not got[rest].view(np.uint8).any()
        assert prof.submitted == n and prof.succeeded == int(ok.sum()) and prof.deviceFailures == n - int(ok.sum())
        assert prof.phaseEvaluations > 0
        # NULL capillary input is the same batch
        out.zero_()
        assert lib.reactive_gpu_hem_run_resident_v1(hem.handle, dq.data_ptr(), de.data_ptr(), dseed.data_ptr(), None,
                                                    dorder.data_ptr(), n, out.data_ptr(), C.byref(prof), err,
                                                    len(err)) == 0, err.value
        assert out.cpu().numpy().view(A.HEM_OUTPUT_DTYPE)["state"][order].tobytes() == exp.tobytes()
        # a pressure jump or the frozen partition on a named cell is refused
        for field, value in (("pressureJump", 3.5e3), ("equilibrium", 0)):
            bad = cap.copy()
            bad[field][order[17]] = value
            assert lib.reactive_gpu_hem_run_resident_v1(hem.handle, dq.data_ptr(), de.data_ptr(), dseed.data_ptr(),
                                                        dev(bad).data_ptr(), dorder.data_ptr(), n, out.data_ptr(),
                                                        C.byref(prof), err, len(err)) == 1
            assert b"pressure jump" in err.value
        # a jump on a cell the batch does not name is not read
        other = cap.copy()
        other["pressureJump"][rest[0]] = 3.5e3
        assert lib.reactive_gpu_hem_run_resident_v1(hem.handle, dq.data_ptr(), de.data_ptr(), dseed.data_ptr(),
                                                    dev(other).data_ptr(), dorder.data_ptr(), n, out.data_ptr(),
                                                    C.byref(prof), err, len(err)) == 0, err.value
    finally:
        hem.close()
        host.close()


def test_host_capillary_batch_without_jump_is_run_v1():
    rho, e, guess = batch(800, 78)
    n = len(rho)
    cap = np.zeros(n, dtype=A.CAPILLARY_DTYPE)
    cap["color"] = .3
    cap["equilibrium"] = 1
    lib = _lib.load()
    hem = GpuHem(capacity=n)
    err = C.create_string_buffer(1024)
    try:
        got = guess.copy()
        ok2 = np.zeros(n, dtype=np.int32)
        prof = A.HemProfile(1, C.sizeof(A.HemProfile))
        assert lib.reactive_gpu_hem_run_v2(hem.handle, A.dptr(rho), A.dptr(e), cap.ctypes.data_as(C.c_void_p), n,
                                           got.ctypes.data_as(C.c_void_p), ok2.ctypes.data_as(C.POINTER(C.c_int)),
                                           C.byref(prof), err, len(err)) == 0, err.value
        exp = guess.copy()
        ok, _ = hem.run(rho, e, exp)
        assert np.array_equal(ok2, ok) and got.tobytes() == exp.tobytes()
        cap["pressureJump"][5] = 10.0
        before = guess.copy()
        assert lib.reactive_gpu_hem_run_v2(hem.handle, A.dptr(rho), A.dptr(e), cap.ctypes.data_as(C.c_void_p), n,
                                           before.ctypes.data_as(C.c_void_p), ok2.ctypes.data_as(C.POINTER(C.c_int)),
                                           C.byref(prof), err, len(err)) == 1
        assert before.tobytes() == guess.tobytes()
    finally:
        hem.close()
