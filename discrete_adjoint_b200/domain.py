"""Domain decomposition of one mesh over several contexts (one per GPU, or several on one GPU).

The reference runs one instance on several MPI ranks and on nothing else: each rank owns a
weighted range of the elements' Hilbert keys (BSFC, src/repartition/repartition_BSFC.C:540, with
the weights of :38-40 -- 1.40 for a cell holding material, 1.35 for an empty buffer cell, 0.95
for the rest), refreshes its ghost elements every step (src/geoflow/move_data.C:28-300) and
takes dt from MPI_Allreduce(MIN) over the ranks (src/geoflow/get_coef_and_eigen.C:173).

Here:
* `partition` cuts the cells' Hilbert keys (the reference's own keys, `records.mesh_keys`) into
  contiguous ranges of equal weight;
* `decompose` builds each part's `Subdomain`: a local mesh holding the owned cells first (in the
  mesh's own order, which keeps tiles compact) and two rings of ghost cells after them -- every
  cell an owned cell's step reads (face neighbours, both fine neighbours of a hanging side) and
  every cell those read -- with neighbour entries that leave the subdomain turned into domain
  edges, plus the exchange lists: for each other part, the owned cells it holds as ghosts
  (`send`) and the ghost slots filled from it (`recv`), in matching order;
* a step of all subdomains is `da_step_bounds` on each, one MIN over the (CFL bound, -hmax) pairs,
  `da_step_apply` on each (the same dt bits everywhere), and the halo exchange
  (`da_halo_pack` -> transfer -> `da_halo_unpack`).  The owned cells then hold the undivided
  mesh's step bit for bit.

Two drivers: `LocalDomain` steps every subdomain from this process (contexts on one or several
GPUs; the MIN on the host, halos through device buffers); `run_distributed` steps this rank's
subdomain under torch.distributed -- NCCL (all-reduce of the pair and point-to-point halo
transfers of device buffers, ordered on the context's stream) or gloo (through host memory).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _ffi
from .mesh import Mesh

GEOFLOW_TINY = 1e-4  # src/header/constant.h:68
WEIGHT_WET, WEIGHT_BUFFER, WEIGHT_EMPTY = 1.40, 1.35, 0.95  # repartition_BSFC.C:38-40
GHOST_RINGS = 2


def face_neighbours(mesh: Mesh, cells: np.ndarray) -> np.ndarray:
    """Every neighbour entry (all 8 slots) of the given cells, domain edges dropped."""
    nb = mesh.nbr[:, cells].reshape(-1)
    return np.unique(nb[nb >= 0])


def lb_weights(mesh: Mesh, h: np.ndarray | None = None) -> np.ndarray:
    """The reference's load-balancing weights: a cell with h > GEOFLOW_TINY weighs 1.40, an empty
    cell next to one (the buffer zone around the flow) 1.35, any other 0.95."""
    w = np.full(mesh.n, WEIGHT_EMPTY)
    if h is None:
        return w
    wet = np.asarray(h) > GEOFLOW_TINY
    if wet.any():
        buf = np.zeros(mesh.n, dtype=bool)
        buf[face_neighbours(mesh, np.flatnonzero(wet))] = True
        w[buf & ~wet] = WEIGHT_BUFFER
    w[wet] = WEIGHT_WET
    return w


def hilbert_order(mesh: Mesh) -> np.ndarray:
    """Cells sorted by the reference's element key (the Hilbert key of the cell centre in the
    mesh's extent, src/main/hilbert.C:76-137)."""
    from . import records
    k = records.mesh_keys(mesh).astype(np.uint64)
    key64 = (k[:, 0] << np.uint64(32)) | k[:, 1]
    return np.argsort(key64, kind="stable")


def partition(mesh: Mesh, nparts: int, h: np.ndarray | None = None, order: np.ndarray | None = None) -> np.ndarray:
    """Part (0 .. nparts-1) of every cell: contiguous ranges of the Hilbert order with equal weight
    (lb_weights).  Every part gets at least one cell."""
    if nparts < 1 or nparts > mesh.n:
        raise ValueError(f"nparts must lie in [1, {mesh.n}]")
    order = hilbert_order(mesh) if order is None else np.asarray(order)
    w = lb_weights(mesh, h)[order]
    mid = np.cumsum(w) - 0.5 * w                    # weight before each cell's middle
    # part j starts at the first cell whose middle lies at or past j/nparts of the weight, moved
    # so that every part keeps at least one cell
    start = np.searchsorted(mid, np.arange(nparts) * (w.sum() / nparts), side="left")
    start[0] = 0
    for j in range(1, nparts):
        start[j] = min(max(start[j], start[j - 1] + 1), mesh.n - (nparts - j))
    sorted_part = np.zeros(mesh.n, dtype=np.int32)
    sorted_part[start[1:]] = 1
    sorted_part = np.cumsum(sorted_part).astype(np.int32)
    part = np.empty(mesh.n, dtype=np.int32)
    part[order] = sorted_part
    return part


@dataclass
class Subdomain:
    """One part of a decomposed mesh.  cells[l] is the global index of local cell l; the first
    n_owned are owned.  send[q] lists local owned cells whose values part q holds as ghosts, in
    the order of part q's recv[self.rank]; recv[q] lists local ghost cells owned by part q."""
    rank: int
    nparts: int
    cells: np.ndarray
    n_owned: int
    mesh: Mesh
    send: dict = field(default_factory=dict)
    recv: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return len(self.cells)

    def local(self, a: np.ndarray) -> np.ndarray:
        """A per-cell global array restricted to this subdomain's cells (owned, then ghosts)."""
        return np.ascontiguousarray(np.asarray(a)[..., self.cells])


def ghost_rings(mesh: Mesh, owned: np.ndarray, rings: int = GHOST_RINGS) -> list[np.ndarray]:
    """The ghost rings of a set of owned cells: ring 1 = their neighbours outside the set, ring k =
    the neighbours of ring k-1 not in any earlier ring or the set (sorted global indices)."""
    inside = np.zeros(mesh.n, dtype=bool)
    inside[owned] = True
    out, front = [], np.asarray(owned)
    for _ in range(rings):
        nb = face_neighbours(mesh, front)
        ring = nb[~inside[nb]]
        inside[ring] = True
        out.append(ring)
        front = ring
    return out


def local_mesh(mesh: Mesh, cells: np.ndarray) -> Mesh:
    """The mesh restricted to `cells` (local index = position in `cells`): neighbour entries that
    leave the set become domain edges (both slots of the side, so a hanging side stays
    consistent); every other array is the global one restricted."""
    g2l = np.full(mesh.n, -1, dtype=np.int64)
    g2l[cells] = np.arange(len(cells))
    nb = mesh.nbr[:, cells]
    loc = np.where(nb >= 0, g2l[np.maximum(nb, 0)], -1)
    # a side is kept only when both its slots stay inside and every neighbour on it names the cell
    # back across its opposite side (a coarser neighbour that lost the cell's sibling is cut too);
    # cutting one side can break that for the neighbour, so repeat until nothing changes
    n = len(cells)
    idx = np.arange(n)
    while True:
        changed = False
        for s in range(4):
            o = (s + 2) % 4
            a, b = loc[s], loc[s + 4]
            cut = (a < 0) | (b < 0)
            for e in (a, b):
                ec = np.maximum(e, 0)
                back = (loc[o][ec] == idx) | (loc[o + 4][ec] == idx)
                cut |= (e >= 0) & ~back
            cut &= (a >= 0) | (b >= 0)
            if cut.any():
                loc[s, cut] = -1
                loc[s + 4, cut] = -1
                changed = True
        if not changed:
            break
    arrays = dict(n=len(cells), max_level=mesh.max_level, nbr=loc.astype(np.int32),
                  material=mesh.material[cells], level=mesh.level[cells], ix=mesh.ix[cells], iy=mesh.iy[cells],
                  dh0_dpile=mesh.dh0_dpile[:, cells])
    for k in ("x", "y", "dx", "dy", "elevation", "h0", "hu0", "hv0"):
        arrays[k] = getattr(mesh, k)[cells]
    for k in ("zeta", "curvature", "gravity", "d_gravity"):
        arrays[k] = getattr(mesh, k)[:, cells]
    return Mesh(**arrays)


def decompose(mesh: Mesh, nparts: int, part: np.ndarray | None = None, h: np.ndarray | None = None,
              rings: int = GHOST_RINGS) -> list[Subdomain]:
    """Subdomains of `mesh` over `nparts` parts (partition() of the state h unless `part` is
    given), each with its ghost rings and exchange lists."""
    if part is None:
        part = partition(mesh, nparts, h)
    part = np.asarray(part, dtype=np.int32)
    subs = []
    for r in range(nparts):
        owned = np.flatnonzero(part == r)
        if len(owned) == 0:
            raise ValueError(f"part {r} owns no cell")
        ghosts = np.sort(np.concatenate(ghost_rings(mesh, owned, rings)))
        cells = np.concatenate([owned, ghosts])
        subs.append(Subdomain(r, nparts, cells, len(owned), local_mesh(mesh, cells)))
    for s in subs:
        g = s.cells[s.n_owned:]
        src = part[g]
        for q in np.unique(src):
            sel = np.flatnonzero(src == q)
            s.recv[int(q)] = (s.n_owned + sel).astype(np.int32)
            o = subs[q]
            pos = np.searchsorted(o.cells[:o.n_owned], g[sel])   # owned cells are sorted
            o.send[s.rank] = pos.astype(np.int32)
    return subs


def gather_owned(subs: list[Subdomain], values: list, n: int) -> np.ndarray:
    """The global array assembled from every subdomain's owned values (each [..., sub.n])."""
    first = np.asarray(values[0])
    out = np.zeros(first.shape[:-1] + (n,), dtype=first.dtype)
    for s, v in zip(subs, values):
        out[..., s.cells[:s.n_owned]] = np.asarray(v)[..., :s.n_owned]
    return out


# ------------------------------------------------------------------------------ device driver
class ContextSubdomain:
    """A subdomain's context: the mesh uploaded with its ghosts, the exchange lists and buffers
    resident on the context's GPU (torch tensors, allocated once), and the split step."""

    def __init__(self, sub: Subdomain, mat, tp=None, precision: int = _ffi.DA_PREC_FP64, device: int = 0,
                 **ctx_kw):
        import torch
        from .solver import GeoflowContext
        self.sub = sub
        self.device = device
        self.ctx = GeoflowContext(mat, tp, precision=precision, device=device, **ctx_kw)
        self.ctx.upload_mesh(sub.mesh)
        self.ctx._check(self.ctx.lib.da_set_owned(self.ctx.ctx, sub.n_owned), "da_set_owned")
        s = C.c_void_p()
        self.ctx._check(self.ctx.lib.da_get_stream(self.ctx.ctx, C.byref(s)), "da_get_stream")
        self.stream = torch.cuda.ExternalStream(s.value or 0, device=torch.device("cuda", device))
        dev = torch.device("cuda", device)
        self.real = torch.float64 if precision == _ffi.DA_PREC_FP64 else torch.float32
        self.bounds = torch.zeros(2, dtype=torch.float64, device=dev)
        self.send_idx = {q: torch.from_numpy(v).to(dev) for q, v in sub.send.items()}
        self.recv_idx = {q: torch.from_numpy(v).to(dev) for q, v in sub.recv.items()}
        self.send_buf = {q: torch.empty(3 * len(v), dtype=self.real, device=dev) for q, v in sub.send.items()}
        self.recv_buf = {q: torch.empty(3 * len(v), dtype=self.real, device=dev) for q, v in sub.recv.items()}

    def close(self):
        self.ctx.close()

    def _call(self, name, *args):
        self.ctx._check(getattr(self.ctx.lib, name)(self.ctx.ctx, *args), name)

    def set_state(self, h, hu, hv, time: float = 0.0, iteration: int = 0):
        """The global state (all cells of the undivided mesh) restricted to this subdomain."""
        self.ctx.set_state(self.sub.local(h), self.sub.local(hu), self.sub.local(hv))
        self.ctx.set_time(time, iteration)

    def get_state(self):
        return self.ctx.get_state()

    def step_bounds(self, out=None):
        """The first half of the step.  out=None: returns the (CFL bound, -hmax) pair as a host
        array (waits for it); out a float64 device tensor of this GPU: the pair goes there, ordered
        on the context's stream, and the call returns at once."""
        if out is None:
            h = np.zeros(2)
            self._call("da_step_bounds", C.c_void_p(h.ctypes.data))
            return h
        self._call("da_step_bounds", C.c_void_p(out.data_ptr()))
        return out

    def step_apply(self, bounds, stats: bool = False):
        """The second half with the combined pair (a device tensor of this GPU or a host array)."""
        import torch
        if isinstance(bounds, torch.Tensor) and bounds.is_cuda:
            ptr = C.c_void_p(bounds.data_ptr())
        else:
            host = np.ascontiguousarray(np.asarray(bounds.cpu() if hasattr(bounds, "cpu") else bounds),
                                        dtype=np.float64)
            ptr = C.c_void_p(host.ctypes.data)
        if not stats:
            self._call("da_step_apply", ptr, None)
            return None
        s = _ffi.da_step_stats()
        self._call("da_step_apply", ptr, C.byref(s))
        from .solver import StepStats
        return StepStats(s.dt, s.time, s.volume, s.hmax, s.iter)

    def pack(self, q: int):
        idx = self.send_idx[q]
        self._call("da_halo_pack", C.c_void_p(idx.data_ptr()), len(idx), C.c_void_p(self.send_buf[q].data_ptr()))
        return self.send_buf[q]

    def unpack(self, q: int, buf=None):
        idx = self.recv_idx[q]
        buf = self.recv_buf[q] if buf is None else buf
        self._call("da_halo_unpack", C.c_void_p(idx.data_ptr()), len(idx), C.c_void_p(buf.data_ptr()))

    def sync(self):
        self._call("da_sync")


class LocalDomain:
    """Every subdomain of a mesh driven from this process: one context each, on `devices`
    (round-robin; all on one GPU by default).  The MIN of the pairs is taken on the host; halos go
    through device buffers (a copy between GPUs when the two contexts sit on different ones), with
    the receiving stream waiting on an event of the sending one."""

    def __init__(self, mesh: Mesh, nparts: int, mat, tp=None, precision: int = _ffi.DA_PREC_FP64,
                 devices=(0,), part=None, h=None, rings: int = GHOST_RINGS, **ctx_kw):
        self.mesh = mesh
        self.mat = mat
        self.subs = decompose(mesh, nparts, part=part, h=h, rings=rings)
        self.doms = [ContextSubdomain(s, mat, tp, precision, devices[k % len(devices)], **ctx_kw)
                     for k, s in enumerate(self.subs)]

    def close(self):
        for d in self.doms:
            d.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_state(self, h, hu, hv, time: float = 0.0, iteration: int = 0):
        for d in self.doms:
            d.set_state(h, hu, hv, time, iteration)

    def step(self) -> float:
        """One step of every subdomain; returns its dt."""
        return float(self.run(1)[0])

    def exchange(self):
        import torch
        events = {}
        for d in self.doms:
            for q in d.sub.send:
                d.pack(q)
                ev = torch.cuda.Event()
                ev.record(d.stream)
                events[(d.sub.rank, q)] = ev
        for d in self.doms:
            for q in d.sub.recv:
                src = self.doms[q]
                d.stream.wait_event(events[(q, d.sub.rank)])
                buf = src.send_buf[d.sub.rank]
                if src.device != d.device:
                    with torch.cuda.stream(d.stream):
                        d.recv_buf[q].copy_(buf, non_blocking=True)
                    buf = d.recv_buf[q]
                d.unpack(q, buf)

    def run(self, nsteps: int) -> np.ndarray:
        """nsteps steps; returns each step's dt.  The subdomains' volumes of the last step are kept
        in self.volumes."""
        dts = np.zeros(nsteps)
        self.volumes = [0.0] * len(self.doms)
        for k in range(nsteps):
            b = np.minimum.reduce([d.step_bounds() for d in self.doms])
            last = k == nsteps - 1
            for j, d in enumerate(self.doms):
                st = d.step_apply(b, stats=(j == 0 or last))
                if st is not None:
                    dts[k] = st.dt
                    if last:
                        self.volumes[j] = st.volume
            self.exchange()
        for d in self.doms:
            d.sync()
        return dts

    def get_state(self):
        """The global state assembled from the owned cells."""
        parts = [d.get_state() for d in self.doms]
        return tuple(gather_owned(self.subs, [p[v] for p in parts], self.mesh.n) for v in range(3))


# ------------------------------------------------------------------------------ the adjoint over subdomains
ADJOINT_RINGS = 4   # a reverse step of an owned cell reads the forward state four rings out


def box_functional(m: Mesh, h, box, n_owned: int | None = None):
    """J = sum of h^2 dx dy over the cells whose centre lies in box (the first n_owned cells), and
    dJ/dU of every cell ([3][n]; the seed of the reverse sweep)."""
    inb = (m.x >= box[0]) & (m.x <= box[1]) & (m.y >= box[2]) & (m.y <= box[3])
    area = m.dx * m.dy
    lam = np.zeros((3, m.n))
    lam[0] = np.where(inb, 2.0 * h * area, 0.0)
    k = m.n if n_owned is None else n_owned
    return float(np.sum(np.where(inb[:k], h[:k] * h[:k] * area[:k], 0.0))), lam


def adjoint_run_local(dd: "LocalDomain", box, nsteps: int, dh0_dpile=None) -> dict:
    """Forward run and discrete adjoint of J = sum h^2 dx dy over a box at the final step, on the
    subdomains of a LocalDomain built with ADJOINT_RINGS ghost rings (state set, time 0).  The forward
    steps are the split step with its exchanges, each subdomain's states kept on the host; each
    reverse step runs on every subdomain through da_adjoint_step with the step's dt replayed, then
    the ghosts' lambda is refreshed from their owners.  The owned cells' lambda^0 equals the
    undivided mesh's (the same reverse steps), the parameter parts are summed over the owned cells.
    Returns J, lambda0 (the whole mesh's), dJ_dbedfrict, dJ_dintfrict, dJ_dpile, dts."""
    from .solver import adjoint_step, set_dt_replay
    states, times = [], [0.0]
    dts = []
    for _ in range(nsteps):
        states.append([d.get_state() for d in dd.doms])
        dts.append(dd.run(1)[0])
        times.append(times[-1] + dts[-1])
    lam, J = [], 0.0
    for d in dd.doms:
        u = d.get_state()
        j, seed = box_functional(d.sub.mesh, u[0], box, d.sub.n_owned)
        J += j
        lam.append(seed)
    nmat = len(dd.mat.bedfrict_deg)
    gbed, gint = np.zeros(nmat), 0.0
    glob = None
    for n in range(nsteps - 1, -1, -1):
        new = []
        for j, d in enumerate(dd.doms):
            d.ctx.set_state(*states[n][j])
            d.ctx.set_time(times[n], n)
            set_dt_replay(d.ctx, [dts[n]], n)
            ln, part = adjoint_step(d.ctx, lam[j])
            gbed += np.asarray(part.dJ_dbedfrict)
            gint += part.dJ_dintfrict
            new.append(ln)
        glob = gather_owned(dd.subs, new, dd.mesh.n)
        lam = [glob[:, s.cells] for s in dd.subs]
    for d in dd.doms:
        set_dt_replay(d.ctx, None)
    dpile = [] if dh0_dpile is None else [float(np.dot(glob[0], np.asarray(p))) for p in np.atleast_2d(dh0_dpile)]
    return {"J": J, "lambda0": glob, "dJ_dbedfrict": gbed, "dJ_dintfrict": gint, "dJ_dpile": dpile,
            "dts": np.array(dts)}


# ------------------------------------------------------------------------------ distributed driver
def exchange_distributed(dom, group=None):
    """The halo exchange of this rank's subdomain with torch.distributed point-to-point
    operations.  dom provides sub (Subdomain), pack(q) -> tensor, recv_buffer(q) -> tensor and
    unpack(q, tensor); the tensors live where the backend moves them (CUDA for NCCL, CPU for
    gloo)."""
    import torch.distributed as dist
    ops = []
    for q in sorted(dom.sub.send):
        ops.append(dist.P2POp(dist.isend, dom.pack(q), q, group))
    for q in sorted(dom.sub.recv):
        ops.append(dist.P2POp(dist.irecv, dom.recv_buffer(q), q, group))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()
    for q in sorted(dom.sub.recv):
        dom.unpack(q, dom.recv_buffer(q))


def step_distributed(dom, group=None, stats: bool = False):
    """One step of this rank's subdomain: bounds, MIN all-reduce of the pair, apply, exchange.
    dom provides bounds() -> tensor [2] (float64), apply(tensor, stats) and the exchange methods."""
    import torch.distributed as dist
    b = dom.bounds()
    dist.all_reduce(b, op=dist.ReduceOp.MIN, group=group)
    st = dom.apply(b, stats)
    exchange_distributed(dom, group)
    return st


class DistributedContext:
    """This rank's subdomain on its GPU for `step_distributed`.  Under NCCL the pair and the halo
    buffers are device tensors and every collective is issued on the context's stream (no host
    synchronisation inside a step); under gloo they go through host memory."""

    def __init__(self, sub: Subdomain, mat, tp=None, precision: int = _ffi.DA_PREC_FP64, device: int = 0,
                 backend: str = "nccl", **ctx_kw):
        import torch
        self.sub = sub
        self.cs = ContextSubdomain(sub, mat, tp, precision, device, **ctx_kw)
        self.on_device = backend == "nccl"
        if not self.on_device:
            self.host_recv = {q: torch.empty(3 * len(v), dtype=self.cs.real) for q, v in sub.recv.items()}

    def close(self):
        self.cs.close()

    def bounds(self):
        import torch
        if self.on_device:
            return self.cs.step_bounds()
        h = np.zeros(2)
        self.cs._call("da_step_bounds", C.c_void_p(h.ctypes.data))
        return torch.from_numpy(h)

    def apply(self, b, stats: bool = False):
        return self.cs.step_apply(b, stats)

    def pack(self, q):
        buf = self.cs.pack(q)
        if self.on_device:
            return buf
        self.cs.sync()
        return buf.cpu()

    def recv_buffer(self, q):
        return self.cs.recv_buf[q] if self.on_device else self.host_recv[q]

    def unpack(self, q, buf):
        if not self.on_device:
            import torch
            with torch.cuda.stream(self.cs.stream):
                self.cs.recv_buf[q].copy_(buf)
            buf = self.cs.recv_buf[q]
        self.cs.unpack(q, buf)


def run_distributed(dom, nsteps: int, group=None):
    """nsteps steps of this rank's subdomain (every rank calls it with its own, in the same order);
    under NCCL the collectives are ordered on the context's stream and only the last step waits
    for the device.  Returns the last step's stats."""
    import torch
    cs = getattr(dom, "cs", None)
    st = None
    for k in range(nsteps):
        last = k == nsteps - 1
        if cs is not None and dom.on_device:
            with torch.cuda.stream(cs.stream):
                st = step_distributed(dom, group, stats=last)
        else:
            st = step_distributed(dom, group, stats=last)
    return st
