"""Domain decomposition on the device: subdomain contexts stepped through da_step_bounds /
da_step_apply with halo exchanges (da_halo_pack / da_halo_unpack) give the owned cells the
undivided mesh's bits and dt sequence -- from one process (LocalDomain: every subdomain's context
on this GPU) and from two processes (run_distributed over gloo, both ranks on this GPU; their
kernels never wait on each other, the ranks meet only in host collectives)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from discrete_adjoint_b200 import GeoflowContext, TimeProps, _ffi, domain, inputs, make_params

pytestmark = pytest.mark.gpu


def undivided_device(w, nsteps, precision=_ffi.DA_PREC_FP64):
    """The undivided mesh stepped one da_forward_step at a time (the two launches the subdomains use)."""
    m = w.mesh
    with GeoflowContext(w.mat, TimeProps(), precision=precision) as c:
        c.upload_mesh(m)
        c.set_state(m.h0, m.hu0, m.hv0)
        dts = [c.step().dt for _ in range(nsteps)]
        return c.get_state(), dts


def small():
    return inputs.test_case(seed=11, nx0=12, ny0=8, max_level=2, random_frac=0.4)


@pytest.mark.parametrize("nparts", [2, 3, 4])
def test_fp64_subdomains_equal_the_undivided_run_and_the_oracle(nparts):
    w = small()
    m = w.mesh
    nsteps = 80   # past the frict_tiny switch at step 50
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    rc, odts, _ = o.run(h, hu, hv, nsteps)
    assert rc == 0
    with domain.LocalDomain(m, nparts, w.mat, h=m.h0) as dd:
        dd.set_state(m.h0, m.hu0, m.hv0)
        dts = dd.run(nsteps)
        H, HU, HV = dd.get_state()
        vol = sum(dd.volumes)
    assert np.array_equal(dts, odts)
    assert np.array_equal(H, h) and np.array_equal(HU, hu) and np.array_equal(HV, hv)
    v_ref = float(np.sum(m.dx * m.dy * h))
    assert abs(vol - v_ref) <= 1e-12 * v_ref


def test_fp32_split_subdomains_equal_the_undivided_fp32_run():
    w = small()
    m = w.mesh
    (h, hu, hv), dts = undivided_device(w, 60, _ffi.DA_PREC_FP32_SPLIT)
    with domain.LocalDomain(m, 3, w.mat, precision=_ffi.DA_PREC_FP32_SPLIT, h=m.h0) as dd:
        dd.set_state(m.h0, m.hu0, m.hv0)
        ddts = dd.run(60)
        H, HU, HV = dd.get_state()
    assert np.array_equal(ddts, dts)
    assert np.array_equal(H, h) and np.array_equal(HU, hu) and np.array_equal(HV, hv)


def test_headline_mesh_in_four_subdomains():
    # the 1M-cell plane-and-runout workload, split along the Hilbert curve into 4 subdomains
    w = inputs.workload3()
    m = w.mesh
    (h, hu, hv), dts = undivided_device(w, 40)
    with domain.LocalDomain(m, 4, w.mat, h=m.h0) as dd:
        assert all(len(d.sub.send) > 0 for d in dd.doms)
        dd.set_state(m.h0, m.hu0, m.hv0)
        ddts = dd.run(40)
        H, HU, HV = dd.get_state()
    assert np.array_equal(ddts, dts)
    assert np.array_equal(H, h) and np.array_equal(HU, hu) and np.array_equal(HV, hv)


def test_ghosted_context_refuses_whole_steps_and_reports_bad_halo_indices():
    w = small()
    m = w.mesh
    sub = domain.decompose(m, 2, h=m.h0)[0]
    cs = domain.ContextSubdomain(sub, w.mat)
    try:
        cs.set_state(m.h0, m.hu0, m.hv0)
        lib, ctx = cs.ctx.lib, cs.ctx.ctx
        s = _ffi.da_step_stats()
        import ctypes as C
        assert lib.da_forward_step(ctx, C.byref(s)) == _ffi.DA_ERR_UNSUPPORTED
        assert lib.da_forward_run(ctx, 3, C.byref(s)) == _ffi.DA_ERR_UNSUPPORTED
        # an owned cell as an unpack target: skipped by the kernel and reported at the next wait
        q = next(iter(sub.recv))
        bad = torch.zeros(len(sub.recv[q]), dtype=torch.int32, device="cuda")
        rc = lib.da_halo_unpack(ctx, C.c_void_p(bad.data_ptr()), len(bad), C.c_void_p(cs.recv_buf[q].data_ptr()))
        assert rc == 0
        assert lib.da_sync(ctx) == _ffi.DA_ERR_INVALID
        # a host buffer is refused before any launch
        hb = np.zeros(3 * len(bad))
        assert lib.da_halo_pack(ctx, C.c_void_p(bad.data_ptr()), len(bad), C.c_void_p(hb.ctypes.data)) == \
            _ffi.DA_ERR_INVALID
    finally:
        cs.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nsteps, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    d = None
    try:
        w = small()
        subs = domain.decompose(w.mesh, world, h=w.mesh.h0)
        d = domain.DistributedContext(subs[rank], w.mat, backend="gloo")
        d.cs.set_state(w.mesh.h0, w.mesh.hu0, w.mesh.hv0)
        st = domain.run_distributed(d, nsteps)
        h, hu, hv = d.cs.get_state()
        s = subs[rank]
        q.put((rank, s.cells[:s.n_owned], h[:s.n_owned], hu[:s.n_owned], hv[:s.n_owned], st.time, st.iter))
    finally:
        if d is not None:
            d.close()
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_processes_over_gloo_step_the_split_mesh():
    nsteps, world = 60, 2
    w = small()
    (h, hu, hv), dts = undivided_device(w, nsteps)
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, nsteps, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, cells, hh, hhu, hhv, t, it in res:
        assert it == nsteps and t == pytest.approx(sum(dts), rel=1e-12)
        assert np.array_equal(hh, h[cells]) and np.array_equal(hhu, hu[cells]) and np.array_equal(hhv, hv[cells])


def test_subdomain_adjoint_equals_the_undivided():
    # the reverse sweep over subdomain contexts with four ghost rings (da_adjoint_step with the
    # step's dt replayed, the ghosts' lambda refreshed from their owners) against the same
    # reverse steps on the undivided mesh (one part): lambda^0 bit for bit, J and the parameter
    # gradients to rounding (sums over the parts); and against the fused checkpointed sweep
    from discrete_adjoint_b200 import adjoint_run
    w = small()
    m = w.mesh
    nsteps = 56   # across the frict_tiny switch
    box = (float(np.percentile(m.x, 30)), float(np.percentile(m.x, 70)),
           float(np.percentile(m.y, 30)), float(np.percentile(m.y, 70)))
    res = []
    for nparts in (1, 3):
        with domain.LocalDomain(m, nparts, w.mat, h=m.h0, rings=domain.ADJOINT_RINGS) as dd:
            dd.set_state(m.h0, m.hu0, m.hv0)
            res.append(domain.adjoint_run_local(dd, box, nsteps, m.dh0_dpile))
    a, b = res
    assert np.array_equal(a["dts"], b["dts"])
    assert np.array_equal(a["lambda0"], b["lambda0"]) and np.abs(a["lambda0"]).max() > 0
    rel = lambda x, y: abs(x - y) / max(abs(y), 1e-300)  # noqa: E731
    assert rel(b["J"], a["J"]) < 1e-12 and rel(b["dJ_dintfrict"], a["dJ_dintfrict"]) < 1e-10
    assert all(rel(x, y) < 1e-10 for x, y in zip(b["dJ_dbedfrict"], a["dJ_dbedfrict"]))
    assert all(rel(x, y) < 1e-12 for x, y in zip(b["dJ_dpile"], a["dJ_dpile"]))
    with GeoflowContext(w.mat, TimeProps()) as c:
        c.upload_mesh(m)
        c.set_state(m.h0, m.hu0, m.hv0)
        g = adjoint_run(c, box, nsteps, 8, m.dh0_dpile, want_lambda0=True)
    scale = np.abs(g.lambda0).max()
    assert np.abs(g.lambda0 - b["lambda0"]).max() <= 1e-12 * scale
    assert rel(b["J"], g.J) < 1e-12 and rel(b["dJ_dintfrict"], g.dJ_dintfrict) < 1e-9
