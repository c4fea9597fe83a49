"""A plain PyTorch FP64 restatement of one SSPRK2 step of the inviscid HLL
transport with the ideal-gas closure on a structured box (test reference for the
hand-written adjoint; autograd differentiates it).

Operator as src/reactiveTransport/reactiveTransportKernels.h:343-356 (HLL
coefficients, wave speeds waveFactor * c) and :180-191 (face flux), boundary
kinds 1 (slip: mirrored normal velocity and momentum) and 2 (extrapolate); the
closure as src/reactiveTransport/reactiveClosureScalar.cuh:9-57 with pr = 0
(T from e(T) = e by Newton, p = rho r T; sound^2 = cp/cv r T). The Newton runs
without autograd and is followed by one recorded Newton step, whose derivative
at the converged T is the implicit-function derivative.
"""
import torch

from spuma_multiphysics_b200.thermo_data import GAS_CONSTANT, ideal_cv, ideal_energy

WAVE = 1.1


def closure(q, species):
    ns = len(species)
    rho = q[:ns].sum(0)
    Y = q[:ns] / rho
    e_in = (q[ns + 3] - .5 * (q[ns] ** 2 + q[ns + 1] ** 2 + q[ns + 2] ** 2) / rho) / rho

    def mix(T, Yk):
        e = sum(Yk[k] * ideal_energy(sp, T, torch) for k, sp in enumerate(species))
        cv = sum(Yk[k] * ideal_cv(sp, T, torch) for k, sp in enumerate(species))
        return e, cv

    with torch.no_grad():
        T = torch.full_like(rho, 300.0)
        for _ in range(40):
            e, cv = mix(T, Y.detach())
            T = T - (e - e_in.detach()) / cv
    e, cv_c = mix(T, Y)
    T = T - (e - e_in) / cv_c.detach()
    _, cv = mix(T, Y)
    r = sum(Y[k] * (GAS_CONSTANT / sp["W"]) for k, sp in enumerate(species))
    p = rho * r * T
    c = torch.sqrt((cv + r) / cv * r * T)
    return p, c


def _hll(qL, qR, uL, uR, pL, pR, cL, cR, axis, sgn, ns):
    unL, unR = uL[axis] * sgn, uR[axis] * sgn
    aL, aR = WAVE * cL, WAVE * cR
    zero = torch.zeros_like(unL)
    left = torch.minimum(zero, torch.minimum(unL - aL, unR - aR))
    right = torch.maximum(zero, torch.maximum(unL + aL, unR + aR))
    inv = 1 / (right - left)
    advL, advR = right * (unL - left) * inv, left * (right - unR) * inv
    pM, pE = (right * pL - left * pR) * inv, (right * pL * unL - left * pR * unR) * inv
    F = advL * qL + advR * qR
    mom = torch.zeros_like(F)
    mom[ns + axis] = pM * sgn
    mom[ns + 3] = pE
    return F + mom


def rate(q, p, c, dims, h, kinds, ns):
    """L(q) (nv, cells) of the box with cells x-fastest; kinds[s] for the sides
    (-x, +x, -y, +y, -z, +z), each 1 or 2."""
    nx, ny, nz = dims
    nv = q.shape[0]
    area, vol = h * h, h ** 3
    Q = q.reshape(nv, nz, ny, nx)
    rho = Q[:ns].sum(0)
    U = Q[ns:ns + 3] / rho
    P = p.reshape(nz, ny, nx)
    S = c.reshape(nz, ny, nx)
    out = torch.zeros_like(Q)
    dim_of = {0: 3, 1: 2, 2: 1}  # axis -> tensor dimension of (nv, z, y, x)
    for axis in range(3):
        d = dim_of[axis]
        n = Q.shape[d]
        lo = lambda t, dd=d, nn=n: t.narrow(dd, 0, nn - 1)
        hi = lambda t, dd=d, nn=n: t.narrow(dd, 1, nn - 1)
        dsc = d - 1  # the same axis for scalar fields (z, y, x)
        F = _hll(lo(Q), hi(Q), lo(U), hi(U), P.narrow(dsc, 0, n - 1), P.narrow(dsc, 1, n - 1),
                 S.narrow(dsc, 0, n - 1), S.narrow(dsc, 1, n - 1), axis, 1.0, ns) * area
        out = out + torch.nn.functional.pad(-F, _pad(d, 0, 1)) + torch.nn.functional.pad(F, _pad(d, 1, 0))
        for upper in (False, True):
            idx = n - 1 if upper else 0
            qL = Q.narrow(d, idx, 1)
            uL = U.narrow(d, idx, 1)
            pL, cL = P.narrow(dsc, idx, 1), S.narrow(dsc, idx, 1)
            qR, uR = qL, uL
            if kinds[2 * axis + int(upper)] == 1:
                flip = torch.ones(nv, 1, 1, 1, dtype=q.dtype, device=q.device)
                flip[ns + axis] = -1
                qR = qL * flip
                uR = uL * flip[ns:ns + 3]
            F = _hll(qL, qR, uL, uR, pL, pL, cL, cL, axis, 1.0 if upper else -1.0, ns) * area
            out = out + torch.nn.functional.pad(-F, _pad(d, idx, n - 1 - idx))
    return (out / vol).reshape(nv, -1)


def _pad(dim, before, after):
    # F.pad takes pairs from the last dimension backwards; Q has 4 dimensions
    pads = [0] * 8
    k = 3 - dim
    pads[2 * k], pads[2 * k + 1] = before, after
    return pads


def step(q, dt, dims, h, kinds, species):
    ns = len(species)
    p, c = closure(q, species)
    q1 = q + dt * rate(q, p, c, dims, h, kinds, ns)
    p1, c1 = closure(q1, species)
    return .5 * q + .5 * (q1 + dt * rate(q1, p1, c1, dims, h, kinds, ns))
