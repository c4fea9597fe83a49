"""GPU: the reference's device-resident HEM batch (reactive_gpu_hem_run_resident_v1)
on a pure-fluid handle: with capillary inputs it is the capillary recovery
(the multi-species engine made from the same image), bit for bit the host
capillary batch (reactive_gpu_hem_run_v2) on the same cells, pressure jumps
included; without them it is the plain batch, bit for bit run_v1. Results are
scattered to the named global cells, a failed cell returns its seed, and cells
the batch does not name are neither read nor written."""
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


def host_capillary(lib, hem, rho, e, cap, guess):
    """The host capillary batch (run_v2) on copies of the seeds."""
    n = len(rho)
    states, ok = guess.copy(), np.zeros(n, dtype=np.int32)
    prof = A.HemProfile(1, C.sizeof(A.HemProfile))
    err = C.create_string_buffer(1024)
    assert lib.reactive_gpu_hem_run_v2(hem.handle, A.dptr(rho), A.dptr(e), cap.ctypes.data_as(C.c_void_p), n,
                                       states.ctypes.data_as(C.c_void_p), ok.ctypes.data_as(C.POINTER(C.c_int)),
                                       C.byref(prof), err, len(err)) == 0, err.value
    return states, ok


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
    dq, de, dseed, dorder = dev(q_g), dev(e_g), dev(seed_g), dev(order)
    out = torch.zeros(total * A.HEM_OUTPUT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    lib = _lib.load()
    hem = GpuHem(capacity=n, resident=True)
    host = GpuHem(capacity=n)
    err = C.create_string_buffer(1024)
    prof = A.HemProfile(1, C.sizeof(A.HemProfile))

    def resident(capillary):
        out.zero_()
        assert lib.reactive_gpu_hem_run_resident_v1(
            hem.handle, dq.data_ptr(), de.data_ptr(), dseed.data_ptr(),
            None if capillary is None else dev(capillary).data_ptr(), dorder.data_ptr(), n, out.data_ptr(),
            C.byref(prof), err, len(err)) == 0, err.value
        return out.cpu().numpy().view(A.HEM_OUTPUT_DTYPE).copy()

    try:
        rest = np.setdiff1d(np.arange(total), order)
        for jump in (False, True):
            c = cap.copy()
            if jump:  # jumps on named cells, and one on a cell the batch does not name
                c["pressureJump"][order[::7]] = rng.uniform(0, 2e4, len(order[::7]))
                c["pressureJump"][rest[0]] = 3.5e3
            got = resident(c)
            exp, ok = host_capillary(lib, host, rho, e, np.ascontiguousarray(c[order]), guess)
            assert np.array_equal(got["success"][order], ok)
            assert got["state"][order].tobytes() == exp.tobytes()
            failed = ok == 0
            assert got["state"][order][failed].tobytes() == guess[failed].tobytes()
            assert not got[rest].view(np.uint8).any()
            assert prof.submitted == n and prof.succeeded == int(ok.sum())
            assert prof.phaseEvaluations > 0
        # without capillary inputs: the plain batch
        got = resident(None)
        exp = guess.copy()
        ok, _ = host.run(rho, e, exp)
        assert np.array_equal(got["success"][order], ok)
        assert got["state"][order].tobytes() == exp.tobytes()
        assert ok[-1] == 0 and got["state"][order[-1]].tobytes() == guess[-1:].tobytes()
        assert not got[rest].view(np.uint8).any()
        assert prof.submitted == n and prof.succeeded == int(ok.sum()) and prof.deviceFailures == n - int(ok.sum())
    finally:
        hem.close()
        host.close()
