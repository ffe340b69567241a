// Shared by the oracle's programs that rebuild the reference's tables from a flattened mesh
// (ref_harness.cpp, adapter_check.cpp).  TEST INFRASTRUCTURE ONLY.
//
// Input format of a flattened mesh (little endian), after a 6-word header
// (magic, n, max_level, n_materials, a count, a flag):
//   double intfrict, epsilon, gravity_scale, gamma, maxtime, bedfrict[16]
//   int32 nbr[8n] level[n] ix[n] iy[n] material[n]
//   double x[n] y[n] dx[n] dy[n] zeta[2n] gravity[3n] d_gravity[2n] curvature[2n]
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <hdf5.h>
#include <mpi.h>

#include "hpfem.h"

namespace harness {

template <class T>
void rd(FILE *f, T *p, size_t n) {
    if (std::fread(p, sizeof(T), n, f) != n) {
        std::fprintf(stderr, "oracle harness: short read\n");
        std::exit(2);
    }
}
template <class T>
void wr(FILE *f, const T *p, size_t n) {
    std::fwrite(p, sizeof(T), n, f);
}

struct MeshIn {
    int n = 0, L = 0, nmat = 0, nsteps = 0, flag = 0;
    double sc[5], bed[16];
    std::vector<int32_t> nbr, level, ix, iy, mat;
    std::vector<double> x, y, dx, dy, zeta, grav, dgrav, curv;
};
void read_mesh(FILE *f, const int32_t hdr[6], MeshIn &m);

// MatProps (properties.h:527-640) of the mesh's materials; ids are 1-based in the reference
struct Props {
    std::vector<double> bedin;
    std::vector<char *> names;
    MatProps *matprops = nullptr;
};
void make_props(const MeshIn &m, Props &pr);

// The reference's Node and Element hash tables of a flattened mesh with state (h, hu, hv)
struct Tables {
    HashTable *NodeTable = nullptr, *El_Table = nullptr;
    std::vector<Element *> els;   // the element of each flattened cell
    double dkr[2], XR[2], YR[2];  // key and coordinate ranges of the element keys
};
Tables build_tables(const MeshIn &m, const double *h, const double *hu, const double *hv, MatProps &matprops,
                    bool ref_static);
// A SolRec over the element keys of t
SolRec *solrec_for(const Tables &t, int n);

}  // namespace harness
