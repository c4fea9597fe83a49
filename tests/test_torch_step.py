"""CPU: the plain PyTorch reference step used by the adjoint tests, pinned to
the transport oracle (itself pinned to the reference's CPU build) on a box with
slip and extrapolate sides, and its closure to the ideal-gas relations."""
import ctypes as C

import numpy as np
import torch

from oracle import oracle
from spuma_multiphysics_b200 import _abi as A, cases, thermo_data as td
import torch_step as TS
import transport_cases as T

DIMS = (5, 4, 3)
H = 1e-3
KINDS = (1, 2, 2, 1, 1, 2)
SPECIES = (td.N2O, td.N2)


def random_state(dims, seed=3):
    rng = np.random.default_rng(seed)
    n = int(np.prod(dims))
    ns = 2
    rho = rng.uniform(1.5, 3.0, n)
    Y0 = rng.uniform(0, 1, n)
    T = rng.uniform(280, 330, n)
    u = rng.normal(0, 25, (3, n))
    e = Y0 * td.ideal_energy(td.N2O, T) + (1 - Y0) * td.ideal_energy(td.N2, T)
    q = np.zeros((ns + 4, n))
    q[0], q[1] = rho * Y0, rho * (1 - Y0)
    q[2:5] = rho * u
    q[5] = rho * (e + .5 * (u ** 2).sum(0))
    return q, T


def test_torch_closure_recovers_temperature():
    q, T = random_state(DIMS)
    p, c = TS.closure(torch.from_numpy(q), SPECIES)
    rho = q[:2].sum(0)
    r = (q[0] / rho) * td.GAS_CONSTANT / td.N2O["W"] + (q[1] / rho) * td.GAS_CONSTANT / td.N2["W"]
    assert np.max(np.abs(p.numpy() / (rho * r * T) - 1)) < 1e-12


def test_torch_rate_matches_transport_oracle():
    q, _ = random_state(DIMS)
    p, c = TS.closure(torch.from_numpy(q), SPECIES)
    faces, volume = cases.box_faces(DIMS, H, KINDS)
    nc, ns, nv = volume.size, 2, 6
    states = np.zeros(nc, dtype=A.STATE_DTYPE)
    states["p"], states["sound"], states["rho"] = p.numpy(), c.numpy(), q[:2].sum(0)
    states["T"], states["cv"], states["gasMass"] = 300.0, 700.0, q[:2].sum(0)
    cfg = A.Config(nc, ns, nv, len(faces), 0, 0.0, 0.0, 0.0, 1.1, 2e8, 0)
    arr = (A.Face * len(faces)).from_buffer_copy(faces.tobytes())
    fixed_states = np.zeros(1, dtype=A.STATE_DTYPE)
    case = dict(config=cfg, faces=arr, volume=volume, fixed_q=np.zeros((1, nv)),
                fixed_states_ptr=C.cast(T.states_ptr(fixed_states), C.c_void_p))
    exp, _, _, _, status = oracle.transport_rhs(case, np.ascontiguousarray(q.T), states.ctypes.data_as(C.c_void_p))
    assert status == 0
    got = TS.rate(torch.from_numpy(q), p, c, DIMS, H, KINDS, ns).numpy().T
    assert T.scaled_error(got, exp) < 1e-13
