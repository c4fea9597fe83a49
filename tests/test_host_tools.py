"""CPU: the library's parallel host helpers (include/reactive_b200_host.h) give
the numpy restatement's values bit for bit on 200,000 cells (more than one
worker chunk): the transport states and primitives of thermo states, the flash
inputs of conserved rows, and the parallel copy; null arguments return 1."""
import numpy as np

from spuma_multiphysics_b200 import _abi as A, _lib


def test_host_helpers_match_numpy():
    L = _lib.load()
    rng = np.random.default_rng(5)
    n, ns, nv = 200_000, 2, 7
    thermo = np.zeros(n, dtype=A.THERMO_DTYPE)
    for name in ("p", "T", "rho", "cv", "soundFrozen", "gasMass"):
        thermo[name] = rng.uniform(.5, 2.0, n)
    q = rng.uniform(.1, 1.0, (n, nv))
    tr = np.zeros(n, dtype=A.STATE_DTYPE)
    prim = np.zeros((n, 4))
    assert L.reactive_b200_host_transport_states_v3(thermo.ctypes.data, n, A.dptr(q), nv, ns, tr.ctypes.data,
                                                    prim.ctypes.data) == 0
    for a, b in (("p", "p"), ("T", "T"), ("rho", "rho"), ("cv", "cv"), ("sound", "soundFrozen"),
                 ("gasMass", "gasMass")):
        assert np.array_equal(tr[a], thermo[b]), a
    assert (tr["dilatation"] == 0).all()
    assert np.array_equal(prim[:, 0], thermo["rho"])
    assert np.array_equal(prim[:, 1:], q[:, ns:ns + 3] / thermo["rho"][:, None])
    masses, energy = np.zeros((n, ns)), np.zeros(n)
    assert L.reactive_b200_host_recovery_inputs_v3(A.dptr(q), n, nv, ns, A.dptr(masses), A.dptr(energy)) == 0
    rho = q[:, 0] + q[:, 1]
    m = q[:, ns:ns + 3]
    assert np.array_equal(masses, q[:, :ns])
    assert np.array_equal(energy, q[:, ns + 3] - .5 * (m[:, 0] * m[:, 0] + m[:, 1] * m[:, 1] + m[:, 2] * m[:, 2]) / rho)
    dst = np.zeros_like(thermo)
    assert L.reactive_b200_host_copy_v3(dst.ctypes.data, thermo.ctypes.data, thermo.nbytes) == 0
    assert dst.tobytes() == thermo.tobytes()
    assert L.reactive_b200_host_threads_v3() >= 1
    assert L.reactive_b200_host_copy_v3(None, thermo.ctypes.data, 8) == 1
    assert L.reactive_b200_host_recovery_inputs_v3(None, n, nv, ns, None, A.dptr(energy)) == 1
