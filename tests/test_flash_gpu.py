"""GPU parity of the CUDA HEM flash (reactive_gpu_hem_* in libreactive_b200.so)
against the flash oracle and the reference flash (oracle/_ref): phase labels
bit-exact, success flags equal, p and T within 1e-9 relative; the device-resident
entry point against the host-array entry point."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A, cases, thermo_data as td
from spuma_multiphysics_b200.hem import GpuHem, HemError
import flash_cases as F

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("policy,n", [("exact", 4000), ("fixed", 1000)])
def test_cuda_flash_matches_oracle_and_reference(policy, n):
    image = F.model_image()
    q, e, guess = cases.flash_batch(n, seed=1000 + n, seed_policy=policy)
    hem = GpuHem(capacity=n)
    got = guess.copy()
    ok, prof = hem.run(q, e, got)
    ref, ref_ok, _ = oracle.ref_flash_recover(image, q, e, guess)
    orc, orc_ok, _ = F.oracle_flash(oracle, image, q, e, guess)
    for other, other_ok in ((ref, ref_ok), (orc, orc_ok)):
        s = F.compare(got, ok, other, other_ok)
        assert s["success_equal"], s
        assert s["label_mismatch"] == 0, s
        assert s["p_rel"] <= F.P_T_TOL and s["T_rel"] <= F.P_T_TOL, s
        assert s["ml_rel"] <= F.STATE_TOL and s["c_rel"] <= F.STATE_TOL, s
    assert prof.submitted == n and prof.succeeded == int(ok.sum())
    assert prof.flashCandidates > 0 and prof.residualEvaluations > 0
    # failed cells keep their seed
    assert np.array_equal(got[ok == 0], guess[ok == 0])


def test_cuda_flash_edge_inputs():
    q, e, guess = cases.flash_batch(64, seed=9)
    q[0] = 0.0
    e[1] = np.nan
    q[2] = -1.0
    e[3] = -1e12
    hem = GpuHem(capacity=64)
    got = guess.copy()
    ok, _ = hem.run(q, e, got)
    ref, ref_ok, _ = oracle.ref_flash_recover(F.model_image(), q, e, guess)
    assert np.array_equal(ok != 0, ref_ok != 0)
    assert not ok[:4].any()


def test_cuda_flash_rejects_out_of_scope_models():
    m = A.HemModel()
    img = bytes(C.string_at(C.addressof(m), C.sizeof(m)))
    with pytest.raises(HemError):
        GpuHem(model=img, capacity=4)
    with pytest.raises(HemError):
        GpuHem(capacity=8).run(*cases.flash_batch(16, seed=3))


def test_cuda_flash_prune_policy():
    """stableGasPrune=1 (the reference's opt-in policy) skips the two-phase seeds
    after a stable all-gas candidate; checked against the reference flash with
    the same model flag."""
    model = F.model_image(stable_gas_prune=1)
    q, e, guess = cases.flash_batch(3000, seed=4242)
    from spuma_multiphysics_b200 import thermo_data as td
    hem = GpuHem(model=td.pure_model(stable_gas_prune=1), capacity=3000)
    got = guess.copy()
    ok, prof = hem.run(q, e, got)
    ref, ref_ok, _ = oracle.ref_flash_recover(model, q, e, guess)
    s = F.compare(got, ok, ref, ref_ok)
    assert s["success_equal"] and s["label_mismatch"] == 0, s
    assert s["p_rel"] <= F.P_T_TOL and s["T_rel"] <= F.P_T_TOL, s


@pytest.mark.parametrize("prune", [0, 1])
def test_cuda_flash_per_cell_form_matches_queue_form(prune):
    """The plain one-thread-per-cell form and the work-queue form run the same
    solvers in the same candidate order: identical success flags and phase
    labels, and states equal to rounding (the two forms are compiled with
    different inlining, so floating-point contraction may differ)."""
    import torch
    from spuma_multiphysics_b200 import thermo_data as td
    n = 3000
    q, e, guess = cases.flash_batch(n, seed=777 + prune)
    hem = GpuHem(model=td.pure_model(stable_gas_prune=prune), capacity=n)
    cons = torch.zeros((5, n), dtype=torch.float64, device="cuda")
    cons[0] = torch.from_numpy(q).cuda()
    cons[4] = torch.from_numpy(e).cuda()
    seed = torch.from_numpy(guess.view(np.uint8).copy()).cuda()
    outs = []
    for per_cell in (False, True):
        state = torch.zeros_like(seed)
        ok = torch.zeros(n, dtype=torch.int32, device="cuda")
        hem.run_device(cons, n, n, 5, seed, state, None, ok, torch.cuda.current_stream().cuda_stream, per_cell)
        torch.cuda.synchronize()
        outs.append((state.cpu().numpy(), ok.cpu().numpy()))
    assert np.array_equal(outs[0][1], outs[1][1])
    a, b = (o[0].view(A.THERMO_DTYPE) for o in outs)
    both = outs[0][1] != 0
    assert np.array_equal(cases.phase_label(a[both]), cases.phase_label(b[both]))
    for field in ("p", "T", "rho"):
        x, y = a[field][both], b[field][both]
        assert np.max(np.abs(x - y) / np.maximum(np.abs(y), 1e-300)) <= 1e-10, field


@pytest.mark.parametrize("n", [5000, 600000])
def test_cuda_flash_device_resident_matches_host_path(n):
    """The host-array batch (copies pipelined in chunks of 256Ki cells and more:
    600,000 cells take two) equals the device-resident one bit for bit; a failed
    cell keeps its seed; the profile counts the successes."""
    import torch
    q, e, guess = cases.flash_batch(n, seed=31337)
    hem = GpuHem(capacity=n)
    host = guess.copy()
    ok, prof_host = hem.run(q, e, host)
    assert prof_host.succeeded == int(np.count_nonzero(ok)) and prof_host.submitted == n
    assert np.array_equal(host[ok == 0].view(np.uint8), guess[ok == 0].view(np.uint8))
    # conserved SoA rows: rho, m (zero velocity), E = e at rest
    cons = torch.zeros((5, n + 3), dtype=torch.float64, device="cuda")
    cons[0, :n] = torch.from_numpy(q).cuda()
    cons[4, :n] = torch.from_numpy(e).cuda()
    seed = torch.from_numpy(guess.view(np.uint8).copy()).cuda()
    state = torch.zeros_like(seed)
    transport = torch.zeros((n, 7), dtype=torch.float64, device="cuda")
    success = torch.zeros(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    hem.run_device(cons, n + 3, n, 5, seed, state, transport, success, stream)
    torch.cuda.synchronize()
    dev = state.cpu().numpy().view(A.THERMO_DTYPE)
    assert np.array_equal(success.cpu().numpy(), ok)
    both = ok != 0
    assert np.array_equal(dev[both].view(np.uint8), host[both].view(np.uint8))  # bitwise identical
    tr = transport.cpu().numpy()
    assert np.array_equal(tr[both, 0], host["p"][both]) and np.array_equal(tr[both, 4], host["soundFrozen"][both])
    prof = hem.counters(stream)
    assert prof.flashCandidates > 0


def test_cuda_flash_in_place_recovery_equals_separate_output():
    """A device recovery whose seed array is also its output array (the step
    driver's second recovery of a step) gives the same bits as one into a
    separate array: the single-phase pass reads each cell's seed before it
    writes that cell's state and touches no other cell's, and the work queue
    and the restart search take their inputs from the records the pass stored.
    The batch mixes cells outside the two-phase bound (decided in the pass) and
    two-phase cells (the queue); a failed cell's output is its seed either way."""
    import torch
    n = 20000
    q, e, guess = cases.flash_batch(n, seed=9090)
    hem = GpuHem(capacity=n)
    cons = torch.zeros((5, n), dtype=torch.float64, device="cuda")
    cons[0] = torch.from_numpy(q).cuda()
    cons[4] = torch.from_numpy(e).cuda()
    seed = torch.from_numpy(guess.view(np.uint8).copy()).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.zeros_like(seed)
    tr_out = torch.zeros((n, 7), dtype=torch.float64, device="cuda")
    ok_out = torch.zeros(n, dtype=torch.int32, device="cuda")
    hem.run_device(cons, n, n, 5, seed, out, tr_out, ok_out, stream)
    same = seed.clone()
    tr_same = torch.zeros_like(tr_out)
    ok_same = torch.zeros_like(ok_out)
    hem.run_device(cons, n, n, 5, same, same, tr_same, ok_same, stream)
    torch.cuda.synchronize()
    ok = ok_out.cpu().numpy()
    assert 0 < np.count_nonzero(ok) and np.array_equal(ok, ok_same.cpu().numpy())
    assert np.array_equal(out.cpu().numpy(), same.cpu().numpy())
    assert np.array_equal(tr_out.cpu().numpy(), tr_same.cpu().numpy())
    labels = cases.phase_label(out.cpu().numpy().view(A.THERMO_DTYPE)[ok != 0])
    assert len(np.unique(labels)) > 1  # single-phase and two-phase cells both present


def test_cuda_flash_labels_match_reference_on_large_batch_sample():
    """Config-3 style batch (60% saturated two-phase states on 65,536
    temperature levels, 40% single phase), 40,000 cells: success flags and
    phase labels bit-exact against the reference flash on the host (all host
    cores), p and T within the flash tolerance."""
    n = 40000
    q, e, guess = cases.flash_batch(n, seed=20260303, saturation_levels=65536)
    model = td.model_bytes(td.pure_model())
    hem = GpuHem(capacity=n)
    got = guess.copy()
    ok, _ = hem.run(q, e, got)
    hem.close()
    ref, ref_ok, _ = oracle.ref_flash_recover(model, q, e, guess, threads=oracle.cpu_threads())
    s = F.compare(got, ok, ref, ref_ok)
    assert s["success_equal"] and s["label_mismatch"] == 0, s
    assert s["p_rel"] <= F.P_T_TOL and s["T_rel"] <= F.P_T_TOL, s


def test_cuda_flash_fails_where_the_reference_fails():
    """A near-critical state (313 K, 78 bar) from the 4,096,000-cell batch that
    the reference flash cannot recover: the CUDA flash reports the same failure
    and leaves the state unchanged."""
    q = np.array([432.822060758171])
    e = np.array([729723467.9575783])
    guess = np.zeros(1, dtype=A.THERMO_DTYPE)
    guess["p"], guess["T"], guess["rho"] = 7822403.962295835, 312.965328917707, 432.822060758171
    model = td.model_bytes(td.pure_model())
    _, ref_ok, _ = oracle.ref_flash_recover(model, q, e, guess.copy())
    hem = GpuHem(capacity=1)
    got = guess.copy()
    ok, _ = hem.run(q, e, got)
    hem.close()
    assert ref_ok[0] == 0 and ok[0] == 0
    assert got.tobytes() == guess.tobytes()
