"""The reference's element keys and forward solution records (include/da_mesh.h).

TITAN2D's dual solver stores each step's forward state in a gz file solution_<rank>_<step>
(src/datstr/dualmesh.C:82-147) keyed by the elements' Hilbert keys; these read and write the same
files for a flattened mesh, so a forward run on the device can hand its states to the reference's
dual solver and back."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _ffi


def solution_name(rank: int, step: int) -> str:
    """The reference's file name of one step's record (dualmesh.C:95)."""
    return "solution_%04d_%08d" % (rank, step)


def cell_keys(x, y, xrange, yrange) -> np.ndarray:
    """[n][2] uint32 keys of cells with centres (x, y) in a table spanning xrange x yrange."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    xr = np.ascontiguousarray(xrange, dtype=np.float64)
    yr = np.ascontiguousarray(yrange, dtype=np.float64)
    out = np.zeros((len(x), 2), dtype=np.uint32)
    st = _ffi.load().da_cell_keys(len(x), _ffi.dptr(x), _ffi.dptr(y), _ffi.dptr(xr), _ffi.dptr(yr),
                                  out.ctypes.data_as(C.POINTER(C.c_uint32)))
    if st:
        raise _ffi.DAError(st, "da_cell_keys")
    return out


def mesh_keys(mesh) -> np.ndarray:
    """Keys of a mesh's cells in the table spanning the mesh's extent."""
    xr = (float(np.min(mesh.x - 0.5 * mesh.dx)), float(np.max(mesh.x + 0.5 * mesh.dx)))
    yr = (float(np.min(mesh.y - 0.5 * mesh.dy)), float(np.max(mesh.y + 0.5 * mesh.dy)))
    return cell_keys(mesh.x, mesh.y, xr, yr)


def write_solution(path: str, keys: np.ndarray, h, hu, hv):
    k = np.ascontiguousarray(keys, dtype=np.uint32)
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (h, hu, hv)]
    st = _ffi.load().da_write_solution(os.fsencode(path), len(k), k.ctypes.data_as(C.POINTER(C.c_uint32)),
                                       *[_ffi.dptr(v) for v in a])
    if st:
        raise _ffi.DAError(st, f"da_write_solution {path}")


def read_solution(path: str, keys: np.ndarray):
    """(h, hu, hv, number of cells without a record)."""
    k = np.ascontiguousarray(keys, dtype=np.uint32)
    n = len(k)
    h, hu, hv = np.zeros(n), np.zeros(n), np.zeros(n)
    miss = C.c_int32(0)
    st = _ffi.load().da_read_solution(os.fsencode(path), n, k.ctypes.data_as(C.POINTER(C.c_uint32)),
                                      _ffi.dptr(h), _ffi.dptr(hu), _ffi.dptr(hv), C.byref(miss))
    if st:
        raise _ffi.DAError(st, f"da_read_solution {path}")
    return h, hu, hv, miss.value


def record_forward(ctx, nsteps: int, directory: str, keys: np.ndarray, rank: int = 0, step0: int = 0):
    """Steps the context nsteps times and writes the state before each step as the reference's
    dual solver records it (record_solution, dualmesh.C:35-80: step k holds U^k)."""
    for k in range(nsteps):
        h, hu, hv = ctx.get_state()
        write_solution(os.path.join(directory, solution_name(rank, step0 + k)), keys, h, hu, hv)
        ctx.step()


# ---------------------------------------------------------------------------- restart files
def write_restart(path: str, mesh, h, hu, hv, time: float = 0.0, iteration: int = 0, dt_hist=(),
                  bedfrict=None, adjiter: int = 0, min_dx=(0.0, 0.0), min_gen: float = 0.0,
                  maxh=(0, 0.0), solrec_last_step: int = 0):
    """restart_<rank> of the reference (save_forward, src/main/restart.C:21-125) for a mesh built
    by this package (its level / ix / iy give the node lattice) and a state: the reference's
    loadrun rebuilds the tables from it and its step() continues the run."""
    hd = _ffi.da_restart_header()
    hd.min_dx[0], hd.min_dx[1] = min_dx
    hd.min_gen = min_gen
    hd.maxh_iter, hd.maxh_hmax = int(maxh[0]), float(maxh[1])
    hd.iter, hd.adjiter, hd.time = int(iteration), int(adjiter), float(time)
    hd.solrec_last_step = int(solrec_last_step)
    dts = np.ascontiguousarray(dt_hist, dtype=np.float64)
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (h, hu, hv)]
    bf = None if bedfrict is None else np.ascontiguousarray(bedfrict, dtype=np.float64)
    st = _ffi.load().da_write_restart(os.fsencode(path), C.byref(hd), _ffi.dptr(dts) if len(dts) else None,
                                      len(dts), C.byref(mesh.soa()), _ffi.iptr(mesh.level), _ffi.iptr(mesh.ix),
                                      _ffi.iptr(mesh.iy), _ffi.dptr(mesh.zeta), _ffi.dptr(mesh.elevation),
                                      _ffi.dptr(bf) if bf is not None else None, *[_ffi.dptr(v) for v in a])
    if st:
        raise _ffi.DAError(st, f"da_write_restart {path}")


def read_restart(path: str) -> dict:
    """The active elements of a reference restart file as a flattened mesh in key order: a dict
    with 'mesh' (Mesh), 'keys', 'h', 'hu', 'hv', 'iter', 'adjiter', 'time', 'dt' (the history)
    and the file's other header fields."""
    from .mesh import Mesh
    lib = _ffi.load()
    hd = _ffi.da_restart_header()
    n, ndt = C.c_int32(0), C.c_int32(0)
    st = lib.da_read_restart(os.fsencode(path), C.byref(hd), C.byref(n), C.byref(ndt), None, None)
    if st:
        raise _ffi.DAError(st, f"da_read_restart {path}")
    N = n.value
    arr = {"keys": np.zeros((N, 2), np.uint32), "nbr": np.zeros((8, N), np.int32), "level": np.zeros(N, np.int32),
           "material": np.zeros(N, np.int32), "x": np.zeros(N), "y": np.zeros(N), "dx": np.zeros(N),
           "dy": np.zeros(N), "elevation": np.zeros(N), "zeta": np.zeros((2, N)), "curvature": np.zeros((2, N)),
           "d_gravity": np.zeros((2, N)), "gravity": np.zeros((3, N)), "h": np.zeros(N), "hu": np.zeros(N),
           "hv": np.zeros(N)}
    dts = np.zeros(max(ndt.value, 1))
    cells = _ffi.da_restart_cells(
        arr["keys"].ctypes.data_as(C.POINTER(C.c_uint32)), _ffi.iptr(arr["nbr"]), _ffi.iptr(arr["level"]),
        _ffi.iptr(arr["material"]), *[_ffi.dptr(arr[k]) for k in ("x", "y", "dx", "dy", "elevation", "zeta",
                                                                   "curvature", "d_gravity", "gravity", "h", "hu",
                                                                   "hv")])
    st = lib.da_read_restart(os.fsencode(path), C.byref(hd), C.byref(n), C.byref(ndt), _ffi.dptr(dts),
                             C.byref(cells))
    if st:
        raise _ffi.DAError(st, f"da_read_restart {path}")
    mesh = Mesh(n=N, nbr=arr["nbr"], material=arr["material"], level=arr["level"], x=arr["x"], y=arr["y"],
                dx=arr["dx"], dy=arr["dy"], elevation=arr["elevation"], zeta=arr["zeta"],
                curvature=arr["curvature"], gravity=arr["gravity"], d_gravity=arr["d_gravity"],
                h0=arr["h"], hu0=arr["hu"], hv0=arr["hv"])
    return {"mesh": mesh, "keys": arr["keys"], "h": arr["h"], "hu": arr["hu"], "hv": arr["hv"],
            "iter": hd.iter, "adjiter": hd.adjiter, "time": hd.time, "dt": dts[:ndt.value],
            "min_dx": tuple(hd.min_dx), "min_gen": hd.min_gen, "maxh": (hd.maxh_iter, hd.maxh_hmax),
            "solrec_last_step": hd.solrec_last_step, "n_nodes": hd.n_nodes, "n_elements": hd.n_elements,
            "n_unresolved": hd.n_unresolved, "xrange": tuple(hd.xrange), "yrange": tuple(hd.yrange)}


def write_outline(path: str, dxy, xrange, yrange, grid: np.ndarray):
    """outline_<rank> beside a restart file (restart.C:104-121): grid is [ny][nx]."""
    g = np.ascontiguousarray(grid, dtype=np.float64)
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (dxy, xrange, yrange)]
    st = _ffi.load().da_write_outline(os.fsencode(path), *[_ffi.dptr(v) for v in a], g.shape[1], g.shape[0],
                                      _ffi.dptr(g))
    if st:
        raise _ffi.DAError(st, f"da_write_outline {path}")
