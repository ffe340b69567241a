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
