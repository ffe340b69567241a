"""Domain decomposition on the CPU: the SFC partition, the ghost rings and exchange lists, and the
split step driven over subdomains -- in one process and as two gloo ranks -- with the oracle's
restatement of the step as each subdomain's stepper.  The decomposed run must give the owned
cells the undivided run's bits and the same dt sequence (the dt reduction of
get_coef_and_eigen.C:173 is a MIN, exact in any order)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from discrete_adjoint_b200 import TimeProps, domain, inputs, make_params


def cases():
    # hanging sides (random refinement), several materials, the frict_tiny switch at step 50
    return {
        "s11": inputs.test_case(seed=11, nx0=12, ny0=8, max_level=2, random_frac=0.4),
        "s2": inputs.test_case(seed=2),
    }


class OracleSubdomain:
    """A subdomain stepped by the oracle (the interface step_distributed / exchange_distributed
    use): bounds, apply, pack, recv_buffer, unpack."""

    def __init__(self, sub, mat, tp=None):
        self.sub = sub
        self.o = oracle.Oracle(make_params(mat, tp or TimeProps()), sub.mesh)
        m = sub.mesh
        self.h, self.hu, self.hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
        self.work = np.zeros(7 * m.n)
        self.dts = []
        self.rbuf = {q: torch.empty(3 * len(v), dtype=torch.float64) for q, v in sub.recv.items()}

    def bounds(self):
        return torch.from_numpy(self.o.step_bounds(self.sub.n_owned, self.h, self.hu, self.hv, self.work))

    def apply(self, b, stats=False):
        self.dts.append(self.o.step_apply(np.asarray(b), self.work, self.h, self.hu, self.hv))

    def pack(self, q):
        i = self.sub.send[q]
        return torch.from_numpy(np.concatenate([self.h[i], self.hu[i], self.hv[i]]))

    def recv_buffer(self, q):
        return self.rbuf[q]

    def unpack(self, q, buf):
        i = self.sub.recv[q]
        b = buf.numpy()
        n = len(i)
        self.h[i], self.hu[i], self.hv[i] = b[:n], b[n:2 * n], b[2 * n:]


def undivided(w, nsteps):
    o = oracle.Oracle(make_params(w.mat, TimeProps()), w.mesh)
    m = w.mesh
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    rc, dts, _ = o.run(h, hu, hv, nsteps)
    assert rc == 0
    return h, hu, hv, dts


@pytest.mark.parametrize("nparts", [1, 2, 3, 5])
def test_partition_is_contiguous_on_the_hilbert_order_and_balanced(nparts):
    m = cases()["s11"].mesh
    part = domain.partition(m, nparts, m.h0)
    order = domain.hilbert_order(m)
    seq = part[order]
    assert seq[0] == 0 and seq[-1] == nparts - 1
    assert np.all(np.diff(seq) >= 0) and np.all(np.diff(seq) <= 1)      # contiguous ranges, none empty
    w = domain.lb_weights(m, m.h0)
    loads = np.array([w[part == r].sum() for r in range(nparts)])
    assert loads.max() - loads.min() <= 2 * w.max()
    assert set(np.unique(w)) <= {domain.WEIGHT_WET, domain.WEIGHT_BUFFER, domain.WEIGHT_EMPTY}


def test_every_part_keeps_a_cell_when_parts_are_many():
    m = cases()["s11"].mesh
    part = domain.partition(m, m.n, m.h0)
    assert sorted(part.tolist()) == list(range(m.n))


@pytest.mark.parametrize("nparts", [2, 4])
def test_ghost_rings_cover_the_stencil_and_exchange_lists_match(nparts):
    m = cases()["s11"].mesh
    subs = domain.decompose(m, nparts, h=m.h0)
    assert sorted(np.concatenate([s.cells[:s.n_owned] for s in subs]).tolist()) == list(range(m.n))
    for s in subs:
        local = set(s.cells.tolist())
        owned = s.cells[:s.n_owned]
        ring1 = set(domain.face_neighbours(m, owned).tolist()) - set(owned.tolist())
        # every cell an owned cell's step reads is local: its neighbours and theirs
        assert ring1 <= local
        assert set(domain.face_neighbours(m, np.array(sorted(ring1), dtype=np.int64)).tolist()) <= local
        # the local neighbour table is the global one wherever a side stays inside
        lm = s.mesh
        g2l = {int(g): l for l, g in enumerate(s.cells)}
        for li in list(range(s.n_owned)) + [g2l[g] for g in ring1]:
            g = s.cells[li]
            for k in range(8):
                gn = m.nbr[k, g]
                ln = lm.nbr[k, li]
                assert (gn < 0 and ln < 0) or (ln >= 0 and s.cells[ln] == gn)
        for q, idx in s.recv.items():
            o = subs[q]
            assert np.array_equal(s.cells[idx], o.cells[o.send[s.rank]])
            assert np.all(idx >= s.n_owned) and np.all(o.send[s.rank] < o.n_owned)
        assert sum(len(v) for v in s.recv.values()) == s.n - s.n_owned


@pytest.mark.parametrize("name,nparts,nsteps", [("s11", 2, 80), ("s11", 4, 80), ("s2", 3, 70)])
def test_decomposed_oracle_run_equals_the_undivided_run(name, nparts, nsteps):
    w = cases()[name]
    m = w.mesh
    h, hu, hv, dts = undivided(w, nsteps)
    subs = domain.decompose(m, nparts, h=m.h0)
    doms = [OracleSubdomain(s, w.mat) for s in subs]
    for _ in range(nsteps):
        b = np.minimum.reduce([d.bounds().numpy() for d in doms])
        for d in doms:
            d.apply(torch.from_numpy(b))
        bufs = {(d.sub.rank, q): d.pack(q) for d in doms for q in d.sub.send}
        for d in doms:
            for q in d.sub.recv:
                d.unpack(q, bufs[(q, d.sub.rank)])
    for d in doms:
        assert d.dts == list(dts)
    H = domain.gather_owned(subs, [d.h for d in doms], m.n)
    HU = domain.gather_owned(subs, [d.hu for d in doms], m.n)
    HV = domain.gather_owned(subs, [d.hv for d in doms], m.n)
    assert np.array_equal(H, h) and np.array_equal(HU, hu) and np.array_equal(HV, hv)
    assert (h > 1e-4).sum() > 0


def test_without_the_exchange_the_run_departs():
    # the exchange is what carries the neighbours' new values: skipping it changes the result
    w = cases()["s11"]
    m = w.mesh
    h, _, _, _ = undivided(w, 40)
    subs = domain.decompose(m, 2, h=m.h0)
    doms = [OracleSubdomain(s, w.mat) for s in subs]
    for _ in range(40):
        b = np.minimum.reduce([d.bounds().numpy() for d in doms])
        for d in doms:
            d.apply(torch.from_numpy(b))
    H = domain.gather_owned(subs, [d.h for d in doms], m.n)
    assert not np.array_equal(H, h)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nsteps, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = cases()["s11"]
        subs = domain.decompose(w.mesh, world, h=w.mesh.h0)
        d = OracleSubdomain(subs[rank], w.mat)
        for _ in range(nsteps):
            domain.step_distributed(d)
        s = subs[rank]
        q.put((rank, s.cells[:s.n_owned], d.h[:s.n_owned], d.hu[:s.n_owned], d.hv[:s.n_owned], d.dts))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_step_the_split_mesh_as_the_undivided_one():
    nsteps, world = 70, 2
    w = cases()["s11"]
    h, hu, hv, dts = undivided(w, nsteps)
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, nsteps, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=150) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    seen = np.zeros(w.mesh.n, dtype=bool)
    for rank, cells, hh, hhu, hhv, rdts in res:
        assert rdts == list(dts)
        assert np.array_equal(hh, h[cells]) and np.array_equal(hhu, hu[cells]) and np.array_equal(hhv, hv[cells])
        seen[cells] = True
    assert seen.all()


def oracle_reverse(mesh, mat, states, dts, lam_end, keep=0):
    """The oracle's reverse sweep (exact transpose: keep=0) over stored states; returns lambda^0."""
    o = oracle.Oracle(make_params(mat, TimeProps()), mesh)
    lam = lam_end
    for n in range(len(dts) - 1, -1, -1):
        ft = mat.frict_tiny_early if n < mat.frict_tiny_iters else mat.frict_tiny_late
        lam = o.adjoint_step_ref(*states[n], dts[n], ft, lam, keep=keep)
    return lam


@pytest.mark.parametrize("name,nparts", [("s11", 3), ("s2", 4)])
def test_decomposed_oracle_adjoint_equals_the_undivided(name, nparts):
    # the reverse sweep on subdomains with ADJOINT_RINGS ghost rings (each reverse step on every
    # subdomain from its stored forward states, then the ghosts' lambda from their owners) against
    # the undivided sweep, across the frict_tiny switch
    rings = domain.ADJOINT_RINGS
    w = cases()[name]
    m = w.mesh
    nsteps = 56
    box = (float(np.percentile(m.x, 30)), float(np.percentile(m.x, 70)),
           float(np.percentile(m.y, 30)), float(np.percentile(m.y, 70)))
    # undivided
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    u = [m.h0.copy(), m.hu0.copy(), m.hv0.copy()]
    states, dts = [], []
    for _ in range(nsteps):
        states.append(tuple(a.copy() for a in u))
        rc, dt, _ = o.run(*u, 1)
        dts.append(float(dt[0]))
    _, seed = domain.box_functional(m, u[0], box)
    lam_ref = oracle_reverse(m, w.mat, states, dts, seed)
    assert np.abs(lam_ref).max() > 0
    # subdomains: forward with exchanges, states kept per subdomain
    subs = domain.decompose(m, nparts, h=m.h0, rings=rings)
    doms = [OracleSubdomain(s, w.mat) for s in subs]
    local_states = []
    for _ in range(nsteps):
        local_states.append([(d.h.copy(), d.hu.copy(), d.hv.copy()) for d in doms])
        b = np.minimum.reduce([d.bounds().numpy() for d in doms])
        for d in doms:
            d.apply(torch.from_numpy(b))
        bufs = {(d.sub.rank, q): d.pack(q) for d in doms for q in d.sub.send}
        for d in doms:
            for q in d.sub.recv:
                d.unpack(q, bufs[(q, d.sub.rank)])
    assert doms[0].dts == dts
    lam = [domain.box_functional(d.sub.mesh, d.h, box, d.sub.n_owned)[1] for d in doms]
    os_ = [oracle.Oracle(make_params(w.mat, TimeProps()), s.mesh) for s in subs]
    for n in range(nsteps - 1, -1, -1):
        ft = w.mat.frict_tiny_early if n < w.mat.frict_tiny_iters else w.mat.frict_tiny_late
        new = [o_.adjoint_step_ref(*local_states[n][j], dts[n], ft, lam[j], keep=0) for j, o_ in enumerate(os_)]
        glob = domain.gather_owned(subs, new, m.n)
        lam = [glob[:, s.cells] for s in subs]
    assert np.array_equal(glob, lam_ref)
