"""Loading helpers for the golden fixtures made by tests/golden/make_golden.py."""
import glob
import os

import numpy as np

from discrete_adjoint_b200.mesh import Mesh
from discrete_adjoint_b200.solver import MatProps

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixtures():
    return sorted(glob.glob(os.path.join(GOLDEN, "fwd_*.npz")))


def load(path):
    z = np.load(path)
    mesh = Mesh(**{k[5:]: z[k] for k in z.files if k.startswith("mesh_")})
    ref = {k[4:]: z[k] for k in z.files if k.startswith("ref_")}
    mat = MatProps(intfrict_deg=float(z["intfrict_deg"]), bedfrict_deg=[float(b) for b in z["bedfrict_deg"]])
    return mesh, mat, int(z["nsteps"]), ref


def load_stats(path):
    """(mesh, mat, nsteps, npz) of a stats_* fixture."""
    z = np.load(path)
    mesh = Mesh(**{k[5:]: z[k] for k in z.files if k.startswith("mesh_")})
    mat = MatProps(intfrict_deg=float(z["intfrict_deg"]), bedfrict_deg=[float(b) for b in z["bedfrict_deg"]])
    return mesh, mat, int(z["nsteps"]), z
