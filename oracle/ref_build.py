"""Recipe: compile the reference's own step() and adjoint numerics into oracle/_ref/ref_harness.

TEST INFRASTRUCTURE ONLY (the checker, never the product).  Reads the reference sources where
they lie under /root/reference/src and writes only into oracle/_ref/.  The reference's own
build system (autotools, MPI, HDF5, Fortran) is not used: this recipe compiles the few
translation units on the step() path directly with g++, against
  - oracle/ref/include/mpi.h + mpi_stub.cpp   (single rank),
  - oracle/ref/include/hdf5.h + hdf5_stub.cpp (no-op),
  - oracle/ref/fortran_c.cpp                  (C restatements of getcoef.f, eigen.f, predict.f),
  - oracle/ref/lapack_c.cpp                   (dgesv, LAPACK's LU solve, restated).
Two translation units miss the `template` keyword at dependent member-template calls
(src/geoflow/edge_states.C:61, src/datstr/element2.C:4308-4324), which g++ rejects; they are
preprocessed into oracle/_ref/ and the keyword is inserted there before compiling.  No source
is copied into the repository.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's sources: the checkout this container mounts, or DA_REFERENCE_SRC
REF = os.environ.get("DA_REFERENCE_SRC", "/root/reference/src")
OUT = os.path.join(HERE, "_ref")
EXE = os.path.join(OUT, "ref_harness")
ADAPTER = os.path.join(OUT, "adapter_check")
STUBS = os.path.join(HERE, "ref")

# translation units on the step() path (geoflow, datstr, the update kernel, helpers)
UNITS = [
    "geoflow/step.C", "geoflow/slopes.C", "geoflow/get_coef_and_eigen.C", "geoflow/edge_states.C",
    "geoflow/corrector.C", "geoflow/stats.C", "geoflow/move_data.C", "geoflow/flux_srcs.C",
    "datstr/element2.C", "datstr/node.C", "datstr/hashtab2.C", "datstr/dualmesh.C", "datstr/jacobian.C",
    "adjoint/residual.C", "useful/useful_lib.C", "main/compare_key.C", "main/hilbert.C",
    # the reference's adjoint of one step (the harness's 'DAJ1' mode)
    "adjoint/dual_grid_routines.C", "adjoint/calc_jacobain.C", "adjoint/compute_jacobian_elem.C",
    "adjoint/calc_adjoint.C", "adjoint/debug_routines.C",
    # restart files (the harness's 'DAS1' / 'DAL1' modes)
    "main/restart.C",
    # the DWR estimate on the error grid (the harness's 'DAE1' mode)
    "adjoint/bilinear_interp.C", "adjoint/error_compute.C", "adjoint/error_grid_routines.C",
]
PATCH = {
    "geoflow/edge_states.C": [(r"Curr_El->calc_edge_states<T>\(", "Curr_El->template calc_edge_states<T>(")],
    "datstr/element2.C": [(r"reserve->get_side_neighbor<T>\(", "reserve->template get_side_neighbor<T>(")],
}
# The reference instantiates Element::calc_edge_states<Element> only through a function that
# calls it on an uninitialised pointer (element2.C:4335-4354), which an optimising compiler may
# drop; the harness build adds an explicit instantiation instead.
APPEND = {
    "datstr/element2.C": "\ntemplate void Element::calc_edge_states<Element>(HashTable*, HashTable*, "
                         "std::vector<Element*>*, std::vector<Element*>*, MatProps*, int, double, int*, double*);\n",
}
CXX = ["g++", "-O2", "-std=gnu++14", "-fpermissive", "-w", "-ffp-contract=off", "-fno-fast-math", "-DSUNOS",
       "-I" + os.path.join(STUBS, "include"), "-I" + os.path.join(REF, "header")]


def available() -> bool:
    return os.path.isdir(REF)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False) -> str | None:
    if not available():
        return EXE if os.path.exists(EXE) else None
    os.makedirs(OUT, exist_ok=True)
    objs = []
    for u in UNITS:
        src = os.path.join(REF, u)
        obj = os.path.join(OUT, u.replace("/", "__") + ".o")
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) > os.path.getmtime(src):
            continue
        if u in PATCH:
            ii = os.path.join(OUT, u.replace("/", "__") + ".ii")
            _run(CXX + ["-E", src, "-o", ii], verbose)
            text = open(ii).read()
            for pat, rep in PATCH[u]:
                text, k = re.subn(pat, rep, text)
                if k == 0:
                    raise RuntimeError(f"patch {pat} did not apply to {u}")
            text += APPEND.get(u, "")
            open(ii, "w").write(text)
            _run(CXX + ["-c", ii, "-o", obj], verbose)
        else:
            _run(CXX + ["-c", src, "-o", obj], verbose)
    own = []
    for f in ("mpi_stub.cpp", "hdf5_stub.cpp", "fortran_c.cpp", "lapack_c.cpp", "link_stubs.cpp",
              "harness_tables.cpp", "ref_harness.cpp"):
        src = os.path.join(STUBS, f)
        obj = os.path.join(OUT, f + ".o")
        own.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < os.path.getmtime(src):
            _run(CXX + ["-c", src, "-o", obj], verbose)
    _run(["g++", "-o", EXE] + own + objs + ["-lz", "-lm"], verbose)
    build_adapter(own, objs, verbose, force)
    return EXE


def build_adapter(own, objs, verbose=False, force=False):
    """oracle/_ref/adapter_check: the drop-in adapter (the element-table flattening and the step()
    replacement a maintainer adds to the reference) compiled against the reference's headers,
    linked with the reference's objects and the product library (when it has been built)."""
    root = os.path.dirname(HERE)
    lib_dir = os.path.join(root, "discrete_adjoint_b200")
    if not os.path.exists(os.path.join(lib_dir, "libda_b200.so")):
        return None
    src = os.path.join(STUBS, "adapter_check.cpp")
    obj = os.path.join(OUT, "adapter_check.cpp.o")
    if force or not os.path.exists(obj) or os.path.getmtime(obj) < os.path.getmtime(src):
        _run(CXX + ["-I" + os.path.join(root, "include"), "-c", src, "-o", obj], verbose)
    harness_objs = [o for o in own if not o.endswith("ref_harness.cpp.o")]
    _run(["g++", "-o", ADAPTER] + harness_objs + [obj] + objs +
         ["-L" + lib_dir, "-l:libda_b200.so", "-Wl,-rpath,$ORIGIN/../../discrete_adjoint_b200", "-lz", "-lm"],
         verbose)
    return ADAPTER


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
