"""Z-slab decomposition of the structured impingement box over ranks.

The reference runs one domain on one GPU; this is the decomposition of its step
(src/reactiveFoam/ReactiveFoam.C:961-1019) over several. The transport is a
one-cell stencil whose viscous and WALE terms also read both cells' velocity
gradients and eddy viscosities, so an own cell next to a slab boundary needs two
layers of its neighbour's cells: the layer it shares faces with, and the layer
behind it, from which that layer's gradient is formed. Each rank therefore steps
a box of its own z-layers plus two halo layers towards each neighbouring slab
(the box keeps the mesh tool's canonical ordering, so the structured stencils
run on it; a halo's outer face is extrapolating and only feeds halo cells).

Per stage the rank updates, recovers, bounds (CFL) and ledgers its own cells only
(`reactive_transport_owned_cells_v3`); after each recovery the halo layers'
conserved state, transport states and thermo states are replaced by the
neighbour's own cells (the halo exchange). An own cell then reads exactly the
inputs it reads in the undivided box, so the decomposed step gives the same bits
in every own cell; the CFL minimum is the minimum over ranks and the boundary
ledger the sum over ranks.

The exchange is one message per neighbour and stage: the halo layers' q (SoA
rows), transport states and 176-byte thermo states packed into one contiguous
FP64 buffer, sent with torch.distributed point-to-point operations (NCCL over
NVLink between GPUs, gloo on the host). `LocalSlabs` runs every slab of a box in
one process on one device, with the exchange as device copies.
"""
import contextlib

import numpy as np
import torch

from . import _abi as A
from .cases import box_faces, cartesian_side_kinds
from .flow import Flow, FlowError

HALO = 2
THERMO_DOUBLES = A.THERMO_DTYPE.itemsize // 8  # 22
STATE_DOUBLES = 7


def partition(nz, world):
    """Own z-layer ranges [z0, z1) of each rank: contiguous, in rank order,
    sizes differing by at most one."""
    if world < 1 or nz < world:
        raise ValueError(f"cannot split {nz} layers over {world} ranks")
    base, extra = divmod(nz, world)
    out, z = [], 0
    for r in range(world):
        size = base + (1 if r < extra else 0)
        out.append((z, z + size))
        z += size
    return out


class SlabLayout:
    """One rank's slab of an n x n x n box: own layers [z0, z1), halo layers lo
    below and hi above, the local box's cells in the global numbering (z is the
    slowest index, so a slab is one contiguous range of global cells) and the
    halo transfers."""

    def __init__(self, n, rank, world, halo=HALO):
        parts = partition(n, world)
        if world > 1 and min(b - a for a, b in parts) < halo:
            raise ValueError(f"every slab needs at least {halo} own layers ({n} layers over {world} ranks)")
        if not 0 <= rank < world:
            raise ValueError(f"rank {rank} outside [0, {world})")
        self.n, self.rank, self.world, self.halo = n, rank, world, halo
        self.z0, self.z1 = parts[rank]
        self.lo = halo if rank > 0 else 0
        self.hi = halo if rank < world - 1 else 0
        self.za, self.zb = self.z0 - self.lo, self.z1 + self.hi
        self.nxy = n * n
        self.nz = self.zb - self.za
        self.cells = self.nz * self.nxy
        self.own = (self.lo * self.nxy, (self.lo + self.z1 - self.z0) * self.nxy)
        self.local = slice(self.za * self.nxy, self.zb * self.nxy)      # the local box, global numbering
        self.own_global = slice(self.z0 * self.nxy, self.z1 * self.nxy)

    def faces(self, edge=0.08, **ports):
        """Face array and volumes of the local box: the global box's boundary
        kinds on the lateral sides and at the global z ends, extrapolating faces
        at the halo's outer side."""
        n = self.n
        kinds = []
        for side, k in enumerate(cartesian_side_kinds(n, edge, **ports)):
            axis, upper = side >> 1, bool(side & 1)
            if axis < 2:  # lateral order (fast, slow) with z slow
                kinds.append(np.asarray(k).reshape(n, n)[self.za:self.zb].ravel())
            else:
                at_end = self.zb == n if upper else self.za == 0
                kinds.append(np.asarray(k) if at_end else np.full(n * n, 2))
        return box_faces((n, n, self.nz), edge / n, kinds)

    def sends(self):
        """(peer, (begin, end)): own layers each neighbour keeps as its halo."""
        h = self.halo * self.nxy
        out = []
        if self.lo:
            out.append((self.rank - 1, (self.own[0], self.own[0] + h)))
        if self.hi:
            out.append((self.rank + 1, (self.own[1] - h, self.own[1])))
        return out

    def recvs(self):
        """(peer, (begin, end)): this slab's halo layers and who owns them."""
        out = []
        if self.lo:
            out.append((self.rank - 1, (0, self.own[0])))
        if self.hi:
            out.append((self.rank + 1, (self.own[1], self.cells)))
        return out


def stage_fields(flow, stage):
    """The fields a stage's recovery leaves: (q, thermo) = (q1, s1) after stage 0,
    (qn, sn) after stage 1."""
    return (flow.q1, flow.s1) if stage == 0 else (flow.qn, flow.sn)


def pack(flow, stage, begin, end):
    """Cells [begin, end) of the stage's q, transport states and thermo states,
    as one contiguous FP64 buffer."""
    q, s = stage_fields(flow, stage)
    return torch.cat([q[:, begin:end].reshape(-1), flow.tr[begin:end].reshape(-1),
                      s[begin * A.THERMO_DTYPE.itemsize:end * A.THERMO_DTYPE.itemsize].view(torch.float64)])


def unpack(flow, stage, begin, end, buf):
    q, s = stage_fields(flow, stage)
    count, nv = end - begin, q.shape[0]
    a, b = nv * count, (nv + STATE_DOUBLES) * count
    q[:, begin:end].copy_(buf[:a].view(nv, count))
    flow.tr[begin:end].copy_(buf[a:b].view(count, STATE_DOUBLES))
    s[begin * A.THERMO_DTYPE.itemsize:end * A.THERMO_DTYPE.itemsize].copy_(buf[b:].view(torch.uint8))


def message_doubles(flow, begin, end):
    return (flow.qn.shape[0] + STATE_DOUBLES + THERMO_DOUBLES) * (end - begin)


class DistHalo:
    """Halo exchange over torch.distributed point-to-point operations, on the
    flow's stream when it has one (NCCL waits for the stream's work and the
    stream for the transfers)."""

    def __init__(self, layout, group=None):
        self.layout, self.group = layout, group

    def exchange(self, flow, stage):
        import torch.distributed as dist
        stream = getattr(flow, "stream", None)
        ctx = torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()
        with ctx:
            ops, incoming = [], []
            for peer, (a, b) in self.layout.sends():
                ops.append(dist.P2POp(dist.isend, pack(flow, stage, a, b), peer, self.group))
            for peer, (a, b) in self.layout.recvs():
                buf = torch.empty(message_doubles(flow, a, b), dtype=torch.float64, device=flow.qn.device)
                ops.append(dist.P2POp(dist.irecv, buf, peer, self.group))
                incoming.append((a, b, buf))
            if ops:
                for req in dist.batch_isend_irecv(ops):
                    req.wait()
            for a, b, buf in incoming:
                unpack(flow, stage, a, b, buf)


class SlabFlow:
    """One rank's slab of the impingement box: a Flow over the local box (own
    layers + halos) with the owned-cell range set, stepped half by half with a
    halo exchange after each recovery. q0/guess0 are the GLOBAL cell-major
    initial state and seeds; every rank passes the same ones."""

    def __init__(self, n, rank, world, q0, guess0, fixed_q, fixed_guess, edge=0.08, ports=None, halo=HALO,
                 exchange=None, **flow_kw):
        self.layout = L = SlabLayout(n, rank, world, halo)
        faces, volume = L.faces(edge, **(ports or {}))
        self.flow = Flow(faces, volume, q0[L.local], guess0[L.local], fixed_q, fixed_guess, owned=L.own, **flow_kw)
        self.exchange = exchange if exchange is not None else (DistHalo(L) if world > 1 else None)
        self.graphs, self.graph_dt = None, None

    def capture(self, dt):
        """Capture each half step (stage, CFL, recovery) as a CUDA graph; the
        exchanges run between the replays."""
        f = self.flow
        self.graphs = []
        for stage in (0, 1):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=f.stream):
                f._launch_half(dt, stage)
            self.graphs.append(g)
        self.graph_dt = dt

    def half(self, dt, stage, graph=True):
        f = self.flow
        if graph:
            if self.graphs is None or self.graph_dt != dt:
                self.capture(dt)
            with torch.cuda.stream(f.stream):
                self.graphs[stage].replay()
        else:
            with torch.cuda.stream(f.stream):
                f._launch_half(dt, stage)

    def step(self, dt, graph=True):
        for stage in (0, 1):
            self.half(dt, stage, graph)
            if self.exchange is not None:
                self.exchange.exchange(self.flow, stage)
        self.flow.steps += 1

    def cfl(self):
        """This slab's CFL step minimum over both stages of the last step (own cells)."""
        self.flow.stream.synchronize()
        return self.flow.dt_cfl.min().item()

    def ledger(self, dt):
        return self.flow.ledger(dt)

    def close(self):
        self.graphs = None
        self.flow.close()


def global_cfl(slab, world):
    """The CFL minimum over every rank's own cells (allreduce MIN)."""
    x = slab.cfl()
    if world <= 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=slab.flow.qn.device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return t.item()


def global_ledger(slab, dt, world):
    """The boundary ledger summed over ranks (allreduce SUM)."""
    x = slab.ledger(dt)
    if world <= 1:
        return x
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(x)).to(slab.flow.qn.device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


class LocalSlabs:
    """Every slab of an n^3 box in one process on one device: the decomposed
    step with the halo exchange as device copies between the slabs' buffers
    (each slab's work on its own stream, the exchange after all of them)."""

    def __init__(self, n, world, q0, guess0, fixed_q, fixed_guess, edge=0.08, ports=None, halo=HALO, **flow_kw):
        self.world = world
        self.slabs = [SlabFlow(n, r, world, q0, guess0, fixed_q, fixed_guess, edge, ports, halo, exchange=None,
                               **flow_kw) for r in range(world)]

    def _exchange(self, stage):
        torch.cuda.synchronize()
        for dst in self.slabs:
            for peer, (a, b) in dst.layout.recvs():
                src = self.slabs[peer]
                (sa, sb), = [r for p, r in src.layout.sends() if p == dst.layout.rank]
                unpack(dst.flow, stage, a, b, pack(src.flow, stage, sa, sb))
        torch.cuda.synchronize()

    def step(self, dt, graph=True):
        for stage in (0, 1):
            for s in self.slabs:
                s.half(dt, stage, graph)
            self._exchange(stage)
        for s in self.slabs:
            s.flow.steps += 1

    def check(self, dt):
        cfl = min(s.cfl() for s in self.slabs)
        for s in self.slabs:
            f = s.flow
            b, e = f.own
            failed = int((f.success[b:e] == 0).sum().item())
            if failed:
                raise FlowError(f"HEM recovery failed in {failed} cells of slab {s.layout.rank}")
        if not (cfl > 0 and dt <= cfl * (1 + 1e-10)):
            raise FlowError(f"dt={dt} exceeds the wave/diffusion CFL step {cfl}")
        return dict(cfl_dt=cfl)

    def gather(self):
        """Own cells of every slab in global order: (q SoA nv x N, thermo bytes,
        transport states N x 7) on the device."""
        qs, ss, ts = [], [], []
        size = A.THERMO_DTYPE.itemsize
        for s in self.slabs:
            f = s.flow
            b, e = f.own
            qs.append(f.qn[:, b:e])
            ss.append(f.sn[b * size:e * size])
            ts.append(f.tr[b:e])
        return torch.cat(qs, 1), torch.cat(ss), torch.cat(ts)

    def ledger(self, dt):
        return sum(s.ledger(dt) for s in self.slabs)

    def close(self):
        for s in self.slabs:
            s.close()
