"""Synthetic case construction on the host (seeded, reproducible).

* flash_batch: the standalone HEM workload, states generated forward from a
  seed: a share of saturated two-phase cells (T uniform, vapour quality uniform
  in [0, 1]) and single-phase cells (p log-uniform, T uniform) converted to
  (rho, e) by Peng-Robinson on the default (largest-volume) root.
* impingement: the N2O impingement cube. Uniform Cartesian face list in the
  ordering of the reference's mesh tool (tools/impinging_cartesian_mesh.py:54-127:
  internal faces sorted by (owner, neighbour), then boundary patches), two
  circular ports on x=0 and y=0 selected by face centre inside the circle
  (:12-36), boundary weights and distances as the solver assigns them
  (src/reactiveFoam/ReactiveFoam.C:1193-1204: fixed-state 0, extrapolate 1,
  internal 1 - ownerDistance/distance).
"""
import numpy as np

from . import _abi as A
from .eos import PureFluid
from .thermo_data import N2O


def flash_batch(n, seed=20260303, two_phase_share=0.6, fluid=None, seed_policy="exact", saturation_levels=0):
    """(rho, e, guess states) for n pure-fluid cells.

    seed_policy "exact": the generating (p, T, liquid mass) is the flash seed;
    "fixed": every seed is 40 bar / 293.15 K gas. saturation_levels > 0 draws the
    two-phase temperatures uniformly from that many equally spaced levels in
    [220, 305] K and solves the saturation pair once per level (for batches of
    millions of cells); 0 draws them continuously.
    """
    fluid = fluid or PureFluid(N2O)
    rng = np.random.default_rng(seed)
    n2 = int(round(two_phase_share * n))
    n1 = n - n2
    if saturation_levels:
        levels = np.linspace(220.0, 305.0, saturation_levels)
        pick = rng.integers(0, saturation_levels, n2)
        T2 = levels[pick]
        x = rng.uniform(0.0, 1.0, n2)
        ps, gs, ls = fluid.saturation(levels)
        psat = ps[pick]
        gas = {k: v[pick] for k, v in gs.items()}
        liq = {k: v[pick] for k, v in ls.items()}
    else:
        T2 = rng.uniform(220.0, 305.0, n2)
        x = rng.uniform(0.0, 1.0, n2)
        psat, gas, liq = fluid.saturation(T2)
    v2 = x / gas["rho"] + (1 - x) / liq["rho"]
    rho2 = 1 / v2
    e2 = rho2 * (x * gas["e"] + (1 - x) * liq["e"])
    ml2 = (1 - x) * rho2
    p1 = np.exp(rng.uniform(np.log(1e5), np.log(80e5), n1))
    T1 = rng.uniform(200.0, 320.0, n1)
    one = fluid.tp(T1, p1, "auto")
    rho = np.concatenate([rho2, one["rho"]])
    e = np.concatenate([e2, one["rho"] * one["e"]])
    T = np.concatenate([T2, T1])
    p = np.concatenate([psat, p1])
    ml = np.concatenate([ml2, np.zeros(n1)])
    order = rng.permutation(n)
    rho, e, T, p, ml = rho[order], e[order], T[order], p[order], ml[order]
    guess = np.zeros(n, dtype=A.THERMO_DTYPE)
    if seed_policy == "exact":
        guess["p"], guess["T"] = p, T
        guess["liquidMass"][:, 0] = ml
        guess["activeLiquids"] = (ml > 0).astype(np.int32)
    else:
        guess["p"], guess["T"] = 40e5, 293.15
    guess["rho"] = rho
    return np.ascontiguousarray(rho), np.ascontiguousarray(e), guess


def phase_label(states):
    """0 gas only, 1 liquid only, 2 two-phase (from gasMass > 0 and activeLiquids)."""
    gas = states["gasMass"] > 0
    liq = states["activeLiquids"] != 0
    return np.where(gas & liq, 2, np.where(liq, 1, 0)).astype(np.int8)


def box_faces(dims, h, side_kinds=(2, 2, 2, 2, 2, 2)):
    """Face array (numpy FACE_DTYPE) and cell volumes of a uniform nx x ny x nz
    box of cubic cells of edge h, in the mesh tool's canonical ordering
    (tools/impinging_cartesian_mesh.py:54-127): cells x-fastest; internal faces
    sorted by (owner, neighbour) with the lower cell as owner and normal +e_axis;
    then the boundary faces side by side (-x, +x, -y, +y, -z, +z), each side in
    lateral order (fast, slow) = (y, z), (x, z), (x, y).

    side_kinds[s] is one boundary kind for the whole side or an array of kinds
    in that side's lateral order (1 slip wall, 2 extrapolate, 3 fixed state with
    fixed index 0). Boundary ownerWeight: 0 fixed state, 1 extrapolate, .5 slip;
    distance h/2."""
    nx, ny, nz = dims
    area, volume = h * h, h ** 3
    cell = lambda i, j, k: i + nx * (j + ny * k)
    internal = []
    k, j, i = np.indices((nz, ny, nx - 1))
    internal.append((cell(i, j, k).ravel(), cell(i + 1, j, k).ravel(), 0))
    k, j, i = np.indices((nz, ny - 1, nx))
    internal.append((cell(i, j, k).ravel(), cell(i, j + 1, k).ravel(), 1))
    k, j, i = np.indices((nz - 1, ny, nx))
    internal.append((cell(i, j, k).ravel(), cell(i, j, k + 1).ravel(), 2))
    owners = np.concatenate([a[0] for a in internal])
    neighbours = np.concatenate([a[1] for a in internal])
    axes = np.concatenate([np.full(a[0].size, a[2]) for a in internal])
    order = np.lexsort((neighbours, owners))
    owners, neighbours, axes = owners[order], neighbours[order], axes[order]
    nint = owners.size
    b_owner, b_axis, b_sign, b_kind = [], [], [], []
    for side in range(6):
        axis, upper = side >> 1, bool(side & 1)
        lat = [d for d in range(3) if d != axis]
        slow, fast = np.indices((dims[lat[1]], dims[lat[0]]))
        coords = [None, None, None]
        coords[lat[0]], coords[lat[1]] = fast.ravel(), slow.ravel()
        coords[axis] = np.full(fast.size, dims[axis] - 1 if upper else 0)
        b_owner.append(cell(*coords))
        b_axis.append(np.full(fast.size, axis))
        b_sign.append(np.full(fast.size, 1.0 if upper else -1.0))
        b_kind.append(np.broadcast_to(np.asarray(side_kinds[side]), (fast.size,)))
    b_owner, b_axis, b_sign, b_kind = (np.concatenate(x) for x in (b_owner, b_axis, b_sign, b_kind))
    faces = np.zeros(nint + b_owner.size, dtype=A.FACE_DTYPE)
    faces["owner"][:nint] = owners
    faces["neighbour"][:nint] = neighbours
    faces["fixed"][:nint] = -1
    faces["normal"][np.arange(nint), axes] = 1.0
    faces["area"][:nint] = area
    faces["distance"][:nint] = h
    faces["ownerWeight"][:nint] = 0.5
    faces["kind"][:nint] = 0
    sl = slice(nint, None)
    faces["owner"][sl] = b_owner
    faces["neighbour"][sl] = -1
    faces["fixed"][sl] = np.where(b_kind == 3, 0, -1)
    normals = np.zeros((b_owner.size, 3))
    normals[np.arange(b_owner.size), b_axis] = b_sign
    faces["normal"][sl] = normals
    faces["area"][sl] = area
    faces["distance"][sl] = h / 2
    faces["ownerWeight"][sl] = np.where(b_kind == 3, 0.0, np.where(b_kind == 2, 1.0, 0.5))
    faces["kind"][sl] = b_kind
    return faces, np.full(nx * ny * nz, volume)


def cartesian_faces(n, edge=0.08, port_diameter=0.005, port_z=0.040, port_offset=0.006, boundary_kind=2):
    """Face array (numpy FACE_DTYPE) and cell volumes of an n^3 cube of edge
    `edge` (box_faces ordering).

    Port faces on x=0 (centre y=port_offset, z=port_z) and y=0 (centre
    x=port_offset, z=port_z) are fixed-state faces (fixed index 0); every other
    boundary face has kind `boundary_kind` (2 extrapolate: transmissive). A face
    belongs to a port when its centre lies inside the port circle
    (tools/impinging_cartesian_mesh.py:12-36,89-99).
    """
    kinds = cartesian_side_kinds(n, edge, port_diameter, port_z, port_offset, boundary_kind)
    return box_faces((n, n, n), edge / n, kinds)


def cartesian_side_kinds(n, edge=0.08, port_diameter=0.005, port_z=0.040, port_offset=0.006, boundary_kind=2):
    """The six boundary sides' kinds of cartesian_faces, each an array in that
    side's lateral order (fast, slow) = (y, z), (x, z), (x, y)."""
    h = edge / n
    r2 = (port_diameter / 2) ** 2
    kinds = []
    for side in range(6):
        axis, upper = side >> 1, bool(side & 1)
        kind = np.full(n * n, boundary_kind)
        if not upper and axis < 2:
            slow, fast = np.indices((n, n))   # z slow; the lateral axis (y on x=0, x on y=0) fast
            lateral_c = (fast.ravel() + .5) * h
            zc = (slow.ravel() + .5) * h
            kind[(lateral_c - port_offset) ** 2 + (zc - port_z) ** 2 < r2] = 3
        kinds.append(kind)
    return kinds


def impingement(n, fluid=None, seed=1234, ambient_p=40e5, ambient_T=293.15, inlet_p=56.01325e5, inlet_T=293.15,
                perturbation=0.01):
    """Initial conserved state (cell-major n^3 x 5), seed thermo states and the
    liquid inlet (fixed q and thermo) of the N2O impingement case."""
    fluid = fluid or PureFluid(N2O)
    rng = np.random.default_rng(seed)
    N = n ** 3
    gas = fluid.tp(np.array([ambient_T]), np.array([ambient_p]), "gas")
    rho0 = gas["rho"][0]
    rho = rho0 * (1 + perturbation * rng.uniform(-1, 1, N))
    T = np.full(N, ambient_T)
    props = fluid.trho(T, rho)
    q = np.zeros((N, 5))
    q[:, 0] = rho
    q[:, 4] = rho * props["e"]
    guess = np.zeros(N, dtype=A.THERMO_DTYPE)
    guess["p"], guess["T"], guess["rho"] = props["p"], T, rho
    liq = fluid.tp(np.array([inlet_T]), np.array([inlet_p]), "liquid")
    fixed_q = np.array([[liq["rho"][0], 0, 0, 0, liq["rho"][0] * liq["e"][0]]])
    fixed_guess = np.zeros(1, dtype=A.THERMO_DTYPE)
    fixed_guess["p"], fixed_guess["T"], fixed_guess["rho"] = inlet_p, inlet_T, liq["rho"][0]
    fixed_guess["liquidMass"][:, 0] = liq["rho"][0]
    fixed_guess["activeLiquids"] = 1
    return dict(q=q, guess=guess, fixed_q=fixed_q, fixed_guess=fixed_guess)


def blast_box(n=64, edge=0.064, p_drive=10e5, p_ambient=1e5, T0=300.0, radius=0.016, noise=0.005, seed=4242,
              species=None):
    """The two-species ideal-gas blast box: an n^3 cube (dx = edge/n) with a
    sphere of radius `radius` at the centre holding N2O at p_drive, N2 at
    p_ambient elsewhere, both at T0 and at rest, and a seeded uniform +-noise
    perturbation of the density. Boundaries: extrapolate (transmissive).

    Returns faces, volumes and the nominal density field rho0 (the sphere's
    pressure fixes the density through rho = p / (r T0) before the noise)."""
    from .thermo_data import GAS_CONSTANT, N2, N2O
    species = species or (N2O, N2)
    faces, volume = box_faces((n, n, n), edge / n, (2, 2, 2, 2, 2, 2))
    h = edge / n
    k, j, i = np.indices((n, n, n))
    centre = edge / 2
    r2 = ((i.ravel() + .5) * h - centre) ** 2 + ((j.ravel() + .5) * h - centre) ** 2 + \
        ((k.ravel() + .5) * h - centre) ** 2
    inside = r2 < radius ** 2
    rng = np.random.default_rng(seed)
    r_in, r_out = GAS_CONSTANT / species[0]["W"], GAS_CONSTANT / species[1]["W"]
    rho0 = np.where(inside, p_drive / (r_in * T0), p_ambient / (r_out * T0)) * (1 + noise * rng.uniform(-1, 1, n ** 3))
    return dict(faces=faces, volume=volume, inside=inside, rho0=rho0, p_drive=p_drive, p_ambient=p_ambient,
                T0=T0, species=species, n=n, h=h)


def blast_initial(box, rho0, p_drive, xp=np):
    """Conserved SoA state (nv, cells) of the blast box from the density field
    rho0 and the driver pressure (numpy, or torch tensors with xp=torch so the
    map is differentiable): inside the sphere N2O at T = p_drive / (rho0 r),
    outside N2 at T = p_ambient / (rho0 r), at rest, E = rho0 e(T)."""
    from .thermo_data import GAS_CONSTANT, ideal_energy
    sp_in, sp_out = box["species"]
    inside = box["inside"]
    if xp is not np:
        import torch
        inside = torch.as_tensor(inside, device=rho0.device)
    r_in, r_out = GAS_CONSTANT / sp_in["W"], GAS_CONSTANT / sp_out["W"]
    T_in = p_drive / (rho0 * r_in)
    T_out = box["p_ambient"] / (rho0 * r_out)
    E = xp.where(inside, rho0 * ideal_energy(sp_in, T_in, xp), rho0 * ideal_energy(sp_out, T_out, xp))
    zero = rho0 * 0
    q_in = xp.where(inside, rho0, zero)
    q_out = xp.where(inside, zero, rho0)
    return xp.stack([q_in, q_out, zero, zero, zero, E])
