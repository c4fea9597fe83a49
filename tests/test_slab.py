"""CPU: the z-slab decomposition's host logic. Each rank's local box (own layers
plus halos) is the matching sub-box of the global face list, with the global
boundary kinds and extrapolating faces only at a halo's outer side; the halo
transfers pair up; and the halo exchange over torch.distributed (gloo, world
sizes 2 and 3) fills every halo cell with its owner's q, transport state and
thermo state."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import conftest  # noqa: F401  (registers the package, also in the spawned ranks)
from spuma_multiphysics_b200 import _abi as A, cases
from spuma_multiphysics_b200.slab import SlabLayout, partition

ROOT = Path(__file__).resolve().parents[1]
PORTS = dict(port_diameter=0.005, port_z=0.006, port_offset=0.004)


def test_partition_covers_the_layers_in_order():
    for nz in (4, 7, 12, 160):
        for world in range(1, min(nz, 8) + 1):
            parts = partition(nz, world)
            assert parts[0][0] == 0 and parts[-1][1] == nz
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        partition(3, 4)
    with pytest.raises(ValueError):
        SlabLayout(6, 0, 4)  # slabs thinner than the two halo layers


def _global_faces(n, edge):
    return cases.cartesian_faces(n, edge=edge, **PORTS)


@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_local_boxes_are_sub_boxes_of_the_global_face_list(world):
    n, edge = 12, 0.012
    g_faces, g_volume = _global_faces(n, edge)
    nxy = n * n
    internal_g = {(int(f["owner"]), int(f["neighbour"])): f for f in g_faces if f["neighbour"] >= 0}
    boundary_g = {}
    for f in g_faces[g_faces["neighbour"] < 0]:
        axis = int(np.flatnonzero(f["normal"])[0])
        boundary_g[(int(f["owner"]), axis, float(f["normal"][axis]))] = f
    own_total = 0
    for rank in range(world):
        L = SlabLayout(n, rank, world)
        faces, volume = L.faces(edge, **PORTS)
        assert len(volume) == L.cells == L.nz * nxy
        assert np.array_equal(volume, g_volume[L.local])
        off = L.za * nxy
        own_total += L.own[1] - L.own[0]
        assert L.own == (L.lo * nxy, L.own[0] + (L.z1 - L.z0) * nxy)
        for f in faces:
            o = int(f["owner"]) + off
            if f["neighbour"] >= 0:
                gf = internal_g[(o, int(f["neighbour"]) + off)]
                for key in ("normal", "area", "distance", "ownerWeight", "kind", "fixed"):
                    assert np.array_equal(f[key], gf[key]), key
                continue
            axis = int(np.flatnonzero(f["normal"])[0])
            sign = float(f["normal"][axis])
            k = o // nxy
            cut = axis == 2 and ((sign < 0 and k == L.za and L.za > 0) or (sign > 0 and k == L.zb - 1 and L.zb < n))
            if cut:  # the halo's outer side: extrapolating, owned by a halo cell
                assert f["kind"] == 2 and not (L.own[0] <= int(f["owner"]) < L.own[1])
            else:
                gf = boundary_g[(o, axis, sign)]
                for key in ("area", "distance", "ownerWeight", "kind", "fixed"):
                    assert np.array_equal(f[key], gf[key]), key
    assert own_total == n ** 3
    # the port faces (kind 3) of the global list all land in some slab's own cells
    ports = {int(f["owner"]) for f in g_faces if f["kind"] == 3}
    assert ports


@pytest.mark.parametrize("world", [2, 3, 4])
def test_halo_transfers_pair_up(world):
    n = 12
    layouts = [SlabLayout(n, r, world) for r in range(world)]
    for L in layouts:
        for peer, (a, b) in L.recvs():
            (sa, sb), = [rng for p, rng in layouts[peer].sends() if p == L.rank]
            assert b - a == sb - sa == L.halo * L.nxy
            # the halo cells and the peer's sent cells are the same global cells
            assert a + L.za * L.nxy == sa + layouts[peer].za * L.nxy


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _Fields:
    """The fields a Flow exchanges, on the host."""

    def __init__(self, L, nv, fixed, fill):
        all_ = L.cells + fixed
        self.qn = torch.full((nv, all_), fill, dtype=torch.float64)
        self.q1 = torch.full((nv, all_), fill, dtype=torch.float64)
        self.tr = torch.full((all_, 7), fill, dtype=torch.float64)
        self.sn = torch.full((L.cells * A.THERMO_DTYPE.itemsize,), 0xAB, dtype=torch.uint8)
        self.s1 = torch.full((L.cells * A.THERMO_DTYPE.itemsize,), 0xCD, dtype=torch.uint8)


def _global_fields(n, nv, seed):
    rng = np.random.default_rng(seed)
    N = n ** 3
    return (rng.normal(size=(nv, N)), rng.normal(size=(nv, N)), rng.normal(size=(N, 7)),
            rng.integers(0, 256, size=N * A.THERMO_DTYPE.itemsize, dtype=np.uint8),
            rng.integers(0, 256, size=N * A.THERMO_DTYPE.itemsize, dtype=np.uint8))


def _worker(rank, world, port, n, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from spuma_multiphysics_b200.slab import DistHalo, SlabLayout
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nv, size = 5, A.THERMO_DTYPE.itemsize
        L = SlabLayout(n, rank, world)
        qn, q1, tr, sn, s1 = _global_fields(n, nv, 7)
        f = _Fields(L, nv, 1, np.nan)
        b, e = L.own
        g = slice(L.own_global.start, L.own_global.stop)
        f.qn[:, b:e] = torch.from_numpy(qn[:, g])
        f.q1[:, b:e] = torch.from_numpy(q1[:, g])
        f.tr[b:e] = torch.from_numpy(tr[g])
        f.sn[b * size:e * size] = torch.from_numpy(sn[g.start * size:g.stop * size])
        f.s1[b * size:e * size] = torch.from_numpy(s1[g.start * size:g.stop * size])
        halo = DistHalo(L)
        halo.exchange(f, 0)   # q1, tr, s1
        loc = slice(L.local.start, L.local.stop)
        ok = [np.array_equal(f.q1[:, :L.cells].numpy(), q1[:, loc]),
              np.array_equal(f.tr[:L.cells].numpy(), tr[loc]),
              np.array_equal(f.s1.numpy(), s1[loc.start * size:loc.stop * size])]
        # after stage 0 only q1/s1 (and the transport states) are complete
        ok.append(bool(np.isnan(f.qn[:, :b].numpy()).all()))
        halo.exchange(f, 1)   # qn, tr, sn
        ok += [np.array_equal(f.qn[:, :L.cells].numpy(), qn[:, loc]),
               np.array_equal(f.sn.numpy(), sn[loc.start * size:loc.stop * size]),
               bool(np.isnan(f.qn[:, L.cells:].numpy()).all())]  # fixed cells untouched
        out[rank] = ok
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_gloo(world):
    n = 8 if world == 2 else 9
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    assert sorted(out.keys()) == list(range(world))
    for r in range(world):
        assert all(out[r]), (r, out[r])
