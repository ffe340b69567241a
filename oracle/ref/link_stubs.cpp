// Definitions that the step() translation units reference but that live in parts of the
// reference the harness does not build (driver globals, GIS, MPI packing, adaptation, the
// dual/error meshes).  None is reached on the step() path; each aborts loudly if it is.
// Test infrastructure only.
#include <sys/sysinfo.h>
#include <sys/types.h>
#include <unistd.h>
#include <zlib.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include <hdf5.h>
#include <mpi.h>

#include "hpfem.h"
#include "GMFG_hdfapi.h"

#define NOT_ON_PATH(name)                                                      \
    do {                                                                       \
        std::fprintf(stderr, "ref_harness: %s is not on the step() path\n", name); \
        std::abort();                                                          \
    } while (0)

// driver globals (src/main/hpfem.C, src/repartition/new_datatype.C)
double min_gen, min_dx[2];
double doubleKeyRange;
Mat3x3 ZERO_MATRIX;
MPI_Datatype NSOLTYPE, ELEMTYPE, JACTYPE, DUALELEMTYPE, ERRELEMTYPE, TRANSKEYS, NEIGHTYPE, LB_VERT_TYPE;

// calc_stats (src/geoflow/stats.C:224-229) samples the terrain slope for a volume-averaged
// statistic that the harness does not report; it gets zero resolution and slope.
int Get_max_resolution(double *r) {
    *r = 0.0;
    return 0;
}
int Get_elevation(double, double, double, double *) { NOT_ON_PATH("Get_elevation"); }
int Get_slope(double, double, double, double *sx, double *sy) {
    *sx = *sy = 0.0;
    return 0;
}
int Get_curvature(double, double, double, double *, double *) { NOT_ON_PATH("Get_curvature"); }
int Get_raster_id(double, double, double, int *) { NOT_ON_PATH("Get_raster_id"); }
void construct_el(Element *, ElemPack *, HashTable *, int, double *) { NOT_ON_PATH("construct_el"); }
void Pack_element(void *, ElemPack *, HashTable *, int) { NOT_ON_PATH("Pack_element"); }
void initial_H_adapt(HashTable *, HashTable *, int, MatProps *, PileProps *, FluxProps *, TimeProps *, int) {
    NOT_ON_PATH("initial_H_adapt");
}
void ElemBackgroundCheck(HashTable *, HashTable *, unsigned *, FILE *) { NOT_ON_PATH("ElemBackgroundCheck"); }
void ElemBackgroundCheck2(HashTable *, HashTable *, void *, FILE *) { NOT_ON_PATH("ElemBackgroundCheck2"); }
void SetTransPack(TRANSKEY &, unsigned *, unsigned *, unsigned (*)[2]) { NOT_ON_PATH("SetTransPack"); }
hid_t GH5_open_zip_sol_file(const char *, char) { NOT_ON_PATH("GH5_open_zip_sol_file"); }
hid_t GH5_open_group(hid_t, const char *) { NOT_ON_PATH("GH5_open_group"); }
void GH5_write_zero_keys(hid_t, int, std::vector<unsigned> &) { NOT_ON_PATH("GH5_write_zero_keys"); }
void GH5_write_non_zero_keys_sol(hid_t, int, std::vector<unsigned> &, std::vector<double> &) {
    NOT_ON_PATH("GH5_write_non_zero_keys_sol");
}
