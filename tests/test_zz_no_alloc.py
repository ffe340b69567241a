"""The entry point that allocates nothing, da_forward_step_noalloc, against da_forward_step.

It serves callers that may not allocate device memory (a plugin whose host application owns
the GPU's memory, a real-time loop that forbids allocation): they pass device buffers they
already hold and the step's temporaries live in the library's fixed device array.  This test
holds its buffers in torch tensors (the test may allocate; the entry point does not), calls the
entry point through the C ABI twice in a row, the second call on the first call's output, and
requires the same bits as two steps of a context.  It also checks the size limit.
"""
import ctypes as C

import numpy as np
import pytest

from discrete_adjoint_b200 import GeoflowContext, TimeProps, _ffi, inputs, make_params

pytestmark = pytest.mark.gpu


def dev(a, dtype):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def dptr(t):
    return C.cast(C.c_void_p(t.data_ptr()), _ffi.PD)


def test_noalloc_step_matches_context_step_twice():
    import torch
    lib = _ffi.load()
    w = inputs.test_case(seed=3)
    m = w.mesh
    p = make_params(w.mat, TimeProps())
    keep = dict(nbr=dev(m.nbr.reshape(-1), np.int32), x=dev(m.x, np.float64), y=dev(m.y, np.float64),
                dx=dev(m.dx, np.float64), dy=dev(m.dy, np.float64), g=dev(m.gravity.reshape(-1), np.float64),
                dg=dev(m.d_gravity.reshape(-1), np.float64), cv=dev(m.curvature.reshape(-1), np.float64),
                mat=dev(m.material, np.int32))
    soa = _ffi.da_mesh_soa(m.n, C.cast(C.c_void_p(keep["nbr"].data_ptr()), _ffi.PI32), dptr(keep["x"]),
                           dptr(keep["y"]), dptr(keep["dx"]), dptr(keep["dy"]), dptr(keep["g"]), dptr(keep["dg"]),
                           dptr(keep["cv"]), C.cast(C.c_void_p(keep["mat"].data_ptr()), _ffi.PI32))
    U = [dev(a, np.float64) for a in (m.h0, m.hu0, m.hv0)]
    V = [torch.empty_like(a) for a in U]
    torch.cuda.synchronize()
    stats = []
    t, it = 0.0, 0
    for k in range(2):
        s = _ffi.da_step_stats()
        rc = lib.da_forward_step_noalloc(C.byref(p), C.byref(soa), dptr(U[0]), dptr(U[1]), dptr(U[2]),
                                         dptr(V[0]), dptr(V[1]), dptr(V[2]), t, it, None, C.byref(s))
        assert rc == 0, lib.da_strerror(rc)
        stats.append(s)
        t, it = s.time, s.iter
        U, V = V, U
    got = [a.cpu().numpy() for a in U]

    with GeoflowContext(w.mat, TimeProps()) as ctx:
        ctx.upload_mesh(m)
        ctx.set_state(m.h0, m.hu0, m.hv0)
        ref_stats = [ctx.step(), ctx.step()]
        ref = ctx.get_state()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    for s, r in zip(stats, ref_stats):
        assert s.dt == r.dt and s.time == r.time and s.iter == r.iter
        assert abs(s.volume - r.volume) <= 1e-12 * abs(r.volume)

    # beyond the fixed scratch: rejected before any device access
    big = _ffi.da_mesh_soa(soa.n_cells, soa.nbr, soa.x, soa.y, soa.dx, soa.dy, soa.gravity, soa.d_gravity,
                           soa.curvature, soa.material)
    big.n_cells = (1 << 20) + 1
    s = _ffi.da_step_stats()
    rc = lib.da_forward_step_noalloc(C.byref(p), C.byref(big), dptr(U[0]), dptr(U[1]), dptr(U[2]), dptr(V[0]),
                                     dptr(V[1]), dptr(V[2]), 0.0, 0, None, C.byref(s))
    assert rc == _ffi.DA_ERR_UNSUPPORTED
