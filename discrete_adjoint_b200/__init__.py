"""B200-native finite-volume step and discrete adjoint of the TITAN2D-derived granular-flow
solver (haghakhani/discrete_adjoint), behind a C ABI (include/discrete_adjoint.h).

The device path is the in-tree shared library libda_b200.so; importing a context without
it raises (there is no CPU fallback).
"""
from . import _ffi
from .ensemble import Ensemble, Member
from .mesh import DEM, Mesh, MeshSpec, Pile
from .solver import (GeoflowContext, Gradient, MatProps, StepStats, TimeProps, adjoint_run, adjoint_step,
                     make_params, set_dt_replay, step)

__all__ = ["_ffi", "Ensemble", "Member", "DEM", "Mesh", "MeshSpec", "Pile", "GeoflowContext", "Gradient", "MatProps", "StepStats",
           "TimeProps", "adjoint_run", "adjoint_step", "make_params", "set_dt_replay", "step"]
