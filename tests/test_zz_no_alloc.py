"""GPU: the allocation-free flash entry point (reactive_gpu_hem_run_static_v3).

Callers that cannot call cudaMalloc (a solver whose memory pool owns the whole
device) use this entry point; it keeps its scratch in
a static device array and takes no handle. This file runs last so that a failure
here cannot hide the other tests' results; it also passes when run alone in a
fresh process. Its output is checked against the handle-based entry point
reactive_gpu_hem_run_device_v3 on the same inputs, on two calls in a row (the
second call finds the first call's scratch contents and must not depend on them).
"""
import ctypes as C

import numpy as np
import pytest

from spuma_multiphysics_b200 import _abi as A, _lib, cases, thermo_data as td
from spuma_multiphysics_b200.hem import GpuHem

pytestmark = pytest.mark.gpu

MAX_CELLS = 4096


def _bind(lib):
    fn = lib.reactive_gpu_hem_run_static_v3
    fn.argtypes = [C.c_char_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]
    fn.restype = C.c_int
    return fn


def _device_inputs(n, seed_value, torch):
    q, e, guess = cases.flash_batch(n, seed=seed_value)
    cons = torch.zeros((5, n), dtype=torch.float64, device="cuda")
    cons[0] = torch.from_numpy(q).cuda()
    cons[4] = torch.from_numpy(e).cuda()
    seed = torch.from_numpy(guess.view(np.uint8).copy()).cuda()
    return cons, seed


def _static_call(fn, image, cons, n, seed, torch):
    state = torch.zeros_like(seed)
    transport = torch.zeros((n, 7), dtype=torch.float64, device="cuda")
    ok = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    err = C.create_string_buffer(512)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(image, len(image), cons.data_ptr(), n, n, 5, seed.data_ptr(), state.data_ptr(), transport.data_ptr(),
            ok.data_ptr(), stream, err, len(err))
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
    return state.cpu().numpy().view(A.THERMO_DTYPE), transport.cpu().numpy(), ok.cpu().numpy()


def _handle_call(hem, cons, n, seed, torch):
    state = torch.zeros_like(seed)
    transport = torch.zeros((n, 7), dtype=torch.float64, device="cuda")
    ok = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    hem.run_device(cons, n, n, 5, seed, state, transport, ok, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return state.cpu().numpy().view(A.THERMO_DTYPE), transport.cpu().numpy(), ok.cpu().numpy()


@pytest.mark.parametrize("prune", [0, 1])
def test_static_flash_matches_handle_flash_on_two_calls(prune):
    """Both closure searches: the reference's default, and stableGasPrune (its
    two queue passes with the seed-cell compaction between them, whose second
    pass solves only the cells the first pass left undecided)."""
    import torch
    fn = _bind(_lib.load())
    model = td.pure_model(stable_gas_prune=prune)
    image = td.model_bytes(model)
    for call, (n, seed_value) in enumerate([(MAX_CELLS, 101 + prune), (1500, 202 + prune)]):
        cons, seed = _device_inputs(n, seed_value, torch)
        got_state, got_tr, got_ok = _static_call(fn, image, cons, n, seed, torch)
        hem = GpuHem(model=model, capacity=n)
        ref_state, ref_tr, ref_ok = _handle_call(hem, cons, n, seed, torch)
        hem.close()
        assert np.array_equal(got_ok, ref_ok), f"call {call}: success flags differ"
        assert got_ok.sum() > 0.99 * n
        both = got_ok != 0
        # same kernels, same inputs: bitwise equal states (tolerance of the flash
        # parity tests, 1e-9 relative on p and T, is the documented bar)
        assert np.array_equal(got_state[both].view(np.uint8), ref_state[both].view(np.uint8)), f"call {call}"
        assert np.array_equal(got_tr[both], ref_tr[both])
        assert np.max(np.abs(got_state["p"][both] / ref_state["p"][both] - 1)) <= 1e-9


def test_static_flash_allocates_no_device_memory():
    """After a first call (which may load the library's device code), a call
    leaves the device's free memory unchanged: the entry point allocates nothing."""
    import torch
    fn = _bind(_lib.load())
    image = td.model_bytes(td.pure_model())
    n = 2048
    cons, seed = _device_inputs(n, 303, torch)
    state = torch.zeros_like(seed)
    transport = torch.zeros((n, 7), dtype=torch.float64, device="cuda")
    ok = torch.zeros(n, dtype=torch.int32, device="cuda")
    err = C.create_string_buffer(512)
    stream = torch.cuda.current_stream().cuda_stream
    args = (image, len(image), cons.data_ptr(), n, n, 5, seed.data_ptr(), state.data_ptr(), transport.data_ptr(),
            ok.data_ptr(), stream, err, len(err))
    assert fn(*args) == 0, err.value.decode()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        assert fn(*args) == 0, err.value.decode()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    assert int(ok.sum().item()) > 0.99 * n


def test_static_flash_rejects_oversized_batch():
    import torch
    fn = _bind(_lib.load())
    image = td.model_bytes(td.pure_model())
    n = MAX_CELLS + 1
    cons = torch.zeros((5, n), dtype=torch.float64, device="cuda")
    seed = torch.zeros(n * 176, dtype=torch.uint8, device="cuda")
    state = torch.zeros_like(seed)
    err = C.create_string_buffer(512)
    rc = fn(image, len(image), cons.data_ptr(), n, n, 5, seed.data_ptr(), state.data_ptr(), None, None,
            torch.cuda.current_stream().cuda_stream, err, len(err))
    assert rc == 1 and b"exceeds the maximum of 4096" in err.value
