/*
 * da_mesh.h -- host-side mesh and input preparation (C ABI).
 *
 * The reference builds its mesh with the preprocessor (src/preproc) and adapts it
 * with src/adapt; both stay on the host and out of the GPU path.  This module gives
 * a host-only stand-in that produces the same kind of flattened mesh the hot path
 * consumes: a 2:1-balanced quadtree over a rectangular domain, cells in Morton
 * (space-filling-curve) order, neighbour and hanging-neighbour tables, and the
 * static per-cell fields that the reference computes once per adapt:
 *   gravity vector     Element::calc_gravity_vector  src/datstr/element2.C:3545-3564
 *   d gravity          Element::calc_d_gravity       src/datstr/element2.C:3574-3653
 *   slope, curvature   Get_slope / Get_curvature     src/gisapi/GisApi.C:705-838
 *   initial pile       elliptical_pile_height        src/main/init_piles.C:167-277
 * Nothing here touches a GPU.
 */
#ifndef DA_MESH_H
#define DA_MESH_H

#include <stdint.h>
#include "discrete_adjoint.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Elevation raster, GRASS layout (row 0 is the northern edge, src/gisapi/GisApi.C:153-193). */
typedef struct da_dem {
    int32_t nrows, ncols;
    double xmin, ymin;         /* south-west corner */
    double res;                /* post spacing */
    const float *elev;         /* [nrows*ncols] */
    const int32_t *mat;        /* optional [nrows*ncols] 0-based material ids, or NULL */
} da_dem;

/* One pile (PileProps, src/header/properties.h:199-270); paraboloid shape. */
typedef struct da_pile_spec {
    double xc, yc;             /* centre */
    double height;             /* PileProps::pileheight */
    double major, minor;       /* radii */
    double rot_deg;            /* orientation of the major axis */
    double vx, vy;             /* initial velocity */
} da_pile_spec;

typedef struct da_mesh_spec {
    double xmin, ymin;         /* domain south-west corner */
    double dx0, dy0;           /* base (level 0) cell size */
    int32_t nx0, ny0;          /* base grid */
    int32_t max_level;         /* finest level (<= 20) */
    int32_t uniform;           /* 1: every cell at max_level */
    double refine_margin;      /* pile ellipses are grown by this distance before refining */
    int32_t n_boxes;           /* extra axis-aligned refinement boxes */
    const double *boxes;       /* [4*n_boxes] xmin,xmax,ymin,ymax */
    double random_frac;        /* fraction of cells refined at random (tests: hanging nodes everywhere) */
    uint64_t seed;
    int32_t extra_level;       /* 1: after balancing, every leaf is split once more (the error grid of
                                * the dual-weighted-residual estimate, uniform_refine.C:24-130) */
    int32_t pad;
} da_mesh_spec;

/* Host-owned mesh.  All arrays have n_cells entries per component. */
typedef struct da_mesh_host {
    int32_t n_cells;
    int32_t max_level;
    int32_t n_piles;
    int32_t *level;            /* [n] */
    int32_t *ix, *iy;          /* [n] integer cell coordinates at their level */
    int32_t *nbr;              /* [8][n] */
    double *x, *y, *dx, *dy;   /* [n] */
    double *elevation;         /* [n] */
    double *zeta;              /* [2][n] terrain slope dz/dx, dz/dy */
    double *curvature;         /* [2][n] */
    double *gravity;           /* [3][n] */
    double *d_gravity;         /* [2][n] */
    int32_t *material;         /* [n] */
    double *h0, *hu0, *hv0;    /* [n] initial state */
    double *dh0_dpile;         /* [n_piles][n] d h0 / d pile height */
} da_mesh_host;

/* Builds the mesh.  gravity_scale and length_scale follow MatProps (1 for SI runs). */
int da_mesh_build(const da_mesh_spec *spec, const da_dem *dem, const da_pile_spec *piles,
                  int32_t n_piles, double length_scale, double gravity_scale,
                  da_mesh_host **out);
void da_mesh_free(da_mesh_host *m);
/* Fills a da_mesh_soa view whose pointers alias the host mesh. */
int da_mesh_view(const da_mesh_host *m, da_mesh_soa *view);

/* ---- the reference's element keys and forward solution records (host) ---------------------
 * da_cell_keys: the key TITAN2D gives an element with centre (x, y) in a table spanning xrange x
 * yrange (Element::gen_my_sons_key, src/datstr/element2.C:4360-4420, through fhsfc2d_ of
 * src/main/hilbert.C): the 2-D Hilbert code of the normalised centre, 2 x uint32 per cell.
 * da_write_solution / da_read_solution: the dual solver's gz record of one step's forward state,
 * solution_<rank>_<step> (SolRec::wrtie_sol_to_disk / read_sol_from_disk, src/datstr/dualmesh.C:
 * 82-147, 234-297): zero records (depth not positive) by key, then key + (h, hu, hv).  Reading maps
 * records to cells by key (an unknown key is DA_ERR_INVALID); cells without a record get a zero
 * state and are counted in n_missing (may be NULL). */
int da_cell_keys(int32_t n, const double *x, const double *y, const double xrange[2], const double yrange[2],
                 uint32_t *keys);
int da_write_solution(const char *path, int32_t n, const uint32_t *keys, const double *h, const double *hu,
                      const double *hv);
int da_read_solution(const char *path, int32_t n, const uint32_t *keys, double *h, double *hu, double *hv,
                     int32_t *n_missing);

/* ---- the reference's restart files (host) --------------------------------------------------
 * restart_<rank> as save_forward writes it and loadrun reads it (src/main/restart.C:21-239): the
 * driver's min_dx / min_gen, MaxH_Functional's iteration and hmax, TimeProps (iter, adjiter, time,
 * the dt history), the node table, the element table and the SolRec table header, one gzip stream.
 *
 * da_write_restart: the tables of a flattened quadtree mesh (level, ix, iy of each cell at its own
 * level, as the mesh builder gives them) with its state, in the reference's layout -- nodes on the
 * lattice of half the finest cell with their CORNER / SIDE / BUBBLE / S_C_CON / S_S_CON info,
 * Hilbert keys of the coordinates, positive_x_side 1, every cell NOTRECADAPTED -- so that the
 * reference's loadrun rebuilds them and its step() continues the run.  zeta, elevation, bedfrict
 * (per material, radians; effect_bedfrict and its tangent) may be NULL (zeros).  Node elevations
 * are written as 0.
 * da_read_restart: the active elements (adapted flag > 0) in key order as a flattened mesh: call
 * with out NULL to get *n_cells and *n_dt, then with arrays of at least those sizes (*n_cells and
 * *n_dt in: the capacities).  A neighbour that is not in the file (another rank's) is -1 and
 * counted in n_unresolved.
 * da_write_outline: outline_<rank> (restart.C:104-121): dxy, x and y ranges, ny rows of nx
 * maximum depths. */
typedef struct da_restart_header {
    double min_dx[2];
    double min_gen;
    int32_t maxh_iter;
    double maxh_hmax;
    int32_t iter;               /* TimeProps::iter */
    int32_t adjiter;            /* TimeProps::adjiter */
    double time;                /* TimeProps::time (dimensionless) */
    int32_t solrec_last_step;   /* SolRec::last_solution_time_step */
    /* filled by da_read_restart */
    int32_t n_nodes, n_elements, n_unresolved;
    double xrange[2], yrange[2];  /* the element table's */
} da_restart_header;

typedef struct da_restart_cells {  /* any pointer may be NULL (not returned) */
    uint32_t *keys;                /* [n][2] */
    int32_t *nbr;                  /* [8][n], the layout of da_mesh_soa.nbr */
    int32_t *level, *material;     /* generation; material from 0 */
    double *x, *y, *dx, *dy, *elevation;
    double *zeta, *curvature, *d_gravity;  /* [2][n] */
    double *gravity;               /* [3][n] */
    double *h, *hu, *hv;
} da_restart_cells;

int da_write_restart(const char *path, const da_restart_header *hd, const double *dt_hist, int32_t n_dt,
                     const da_mesh_soa *m, const int32_t *level, const int32_t *ix, const int32_t *iy,
                     const double *zeta, const double *elevation, const double *bedfrict, const double *h,
                     const double *hu, const double *hv);
int da_read_restart(const char *path, da_restart_header *hd, int32_t *n_cells, int32_t *n_dt, double *dt_hist,
                    const da_restart_cells *out);
int da_write_outline(const char *path, const double dxy[2], const double xrange[2], const double yrange[2],
                     int32_t nx, int32_t ny, const double *map);

#ifdef __cplusplus
}
#endif

#endif /* DA_MESH_H */
