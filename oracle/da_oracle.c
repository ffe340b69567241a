/*
 * da_oracle.c -- CPU restatement of the reference's forward step (order_flag = 1).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: only the
 * tests, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may
 * load it.  The product library never links or calls it.
 *
 * It follows the reference's structure rather than the device kernels' structure:
 * whole-mesh passes in the order of step() (src/geoflow/step.C:29-275), fluxes stored
 * on edge "nodes" and written by the owning cell exactly as Element::calc_edge_states
 * does (src/datstr/element2.C:2745-3072), then boundary_flux (element2.C:3374-3411),
 * then the corrector (src/geoflow/corrector.C:36-193 -> update_states,
 * src/adjoint/residual.C:162-275).  Expression order matches the reference; build
 * with -ffp-contract=off so that no multiply-add is fused.
 *
 * Pinning: tests/golden/ holds fixtures produced by the reference's own compiled
 * numerics (oracle/ref_harness.C over the reference sources); test_oracle_golden.py
 * checks this restatement against them.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/discrete_adjoint.h"

#define TINY 1.e-4 /* GEOFLOW_TINY, src/header/constant.h:68 */

/* c_sgn, c_dmin1, dabs: src/header/geoflow.h:90-147 */
static double c_sgn(double zz) {
    double sgn;
    if (zz > TINY)
        sgn = 1;
    else if (zz < -TINY)
        sgn = -1;
    else
        sgn = 0;
    return sgn;
}
static double c_dmin1_2(double d1, double d2) {
    if (d1 > d2) d1 = d2;
    return d1;
}
static double c_dmin1_3(double d1, double d2, double d3) {
    if (d1 > d2) d1 = d2;
    if (d1 > d3) d1 = d3;
    return d1;
}
static double dabs(double dd) {
    if (dd < 0.) dd = -dd;
    return dd;
}
/* max/min: src/datstr/element2.C:1059-1071 */
static double rmax(double x, double y) { return x > y ? x : y; }
static double rmin(double x, double y) { return x > y ? y : x; }
/* sgn(zz, tiny): src/geoflow/sgn.f:19-33 */
static double fsgn(double zz, double tiny) {
    if (dabs(zz) < tiny) return 0.0;
    if (zz >= tiny) return 1.0;
    return -1.0;
}
/* tiny_sgn: src/adjoint/residual.C:153-160 */
static double tiny_sgn(double num, double tiny) {
    if (dabs(num) < tiny)
        return 0.;
    else if (num > tiny)
        return 1.;
    else
        return -1.;
}

static int is_boundary(const da_mesh_soa *m, int i) {
    int n = m->n_cells;
    for (int s = 0; s < 4; ++s)
        if (m->nbr[(size_t)s * n + i] < 0) return 1;
    return 0;
}

/* Element::get_slopes, src/datstr/element2.C:830-939.  slopes: [6][n], x part then y part. */
void orc_slopes(const da_params *p, const da_mesh_soa *m, const double *h, const double *hu,
                const double *hv, double *slopes) {
    const int n = m->n_cells;
    const double *U[3] = {h, hu, hv};
    for (int i = 0; i < n; ++i) {
        if (is_boundary(m, i)) {
            for (int j = 0; j < 6; ++j) slopes[(size_t)j * n + i] = 0;
            continue;
        }
        for (int dir = 0; dir < 2; ++dir) {
            const int sp = dir, sm = dir + 2;
            const int ep = m->nbr[(size_t)sp * n + i], em = m->nbr[(size_t)sm * n + i];
            const int ep2r = m->nbr[(size_t)(sp + 4) * n + i], em2r = m->nbr[(size_t)(sm + 4) * n + i];
            const int ep2 = (ep2r != ep) ? ep2r : -1; /* S_C_CON on the side midpoint */
            const int em2 = (em2r != em) ? em2r : -1;
            const double *co = dir == 0 ? m->x : m->y;
            const double dxp = co[ep] - co[i];
            const double dxm = co[i] - co[em];
            for (int j = 0; j < 3; ++j) {
                double dp = (U[j][ep] - U[j][i]) / dxp;
                if (ep2 >= 0) dp = .5 * (dp + (U[j][ep2] - U[j][i]) / dxp);
                double dm = (U[j][i] - U[j][em]) / dxm;
                if (em2 >= 0) dm = .5 * (dm + (U[j][i] - U[j][em2]) / dxm);
                const double dc = (dp * dxm + dm * dxp) / (dxm + dxp);
                slopes[(size_t)(j + 3 * dir) * n + i] =
                    .5 * (c_sgn(dp) + c_sgn(dm)) * c_dmin1_3(p->gamma * dabs(dp), p->gamma * dabs(dm), dabs(dc));
            }
        }
    }
}

/* k active/passive for one material: gmfggetcoef, src/geoflow/getcoef.f:19-66.
 * The result depends on the state only through sgn(vel) and two guards, so the
 * three signed values are formed once per material. */
static double coef_signed(double bedfrict, double intfrict, double s) {
    const double cosphi = cos(intfrict);
    const double tandel = tan(bedfrict);
    return (2.0 / (cosphi * cosphi)) * (1.0 - s * sqrt(dabs(1.0 - (1.0 + tandel * tandel) * (cosphi * cosphi)))) - 1.0;
}

double orc_kact_cell(const da_params *p, int mat, double h, double hu, double hv, const double *dudx,
                     const double *dudy) {
    double kactx;
    if (h > TINY) {
        const double vel = dudx[1] / h - hu * dudx[0] / (h * h) + dudy[2] / h - hv * dudy[0] / (h * h);
        kactx = coef_signed(p->bedfrict[mat], p->intfrict, fsgn(vel, TINY));
        if (dabs(hu / h) < TINY && dabs(hv / h) < TINY) kactx = 1.0;
        if (kactx < 0.0) kactx = 0.0;
    } else {
        kactx = 1.0;
    }
    return kactx * p->epsilon;
}

/* get_coef_and_eigen, src/geoflow/get_coef_and_eigen.C:86-166 (+ eigen.f:19-49).
 * kact: [n].  Returns via min_dxe (min over wet cells of min(dx,dy)/evalue, init 1e7),
 * hmax; returns DA_ERR_EIGEN if a wave speed exceeds 1e9. */
static int coef_eigen_owned(const da_params *p, const da_mesh_soa *m, int n_owned, const double *h,
                            const double *hu, const double *hv, const double *slopes, double *kact,
                            double *min_dxe_out, double *hmax_out) {
    const int n = m->n_cells;
    double min_dx_dy_evalue = 10000000, hmax = 0;
    int status = DA_OK;
    for (int i = 0; i < n; ++i) {
        if (h[i] > TINY) {
            const int own = i < n_owned;  /* ghosts of a subdomain enter no reduction */
            if (own && hmax < h[i]) hmax = h[i];
            double dudx[3], dudy[3];
            for (int j = 0; j < 3; ++j) {
                dudx[j] = slopes[(size_t)j * n + i];
                dudy[j] = slopes[(size_t)(j + 3) * n + i];
            }
            kact[i] = orc_kact_cell(p, m->material[i], h[i], hu[i], hv[i], dudx, dudy);
            const double vx = hu[i] / h[i], vy = hv[i] / h[i];
            const double gz = m->gravity[(size_t)2 * n + i];
            double k = kact[i];
            if (k < 0.0) k = 0;
            const double evx = dabs(vx) + sqrt(k * gz * h[i]);
            const double evy = dabs(vy) + sqrt(k * gz * h[i]);
            const double evalue = evx > evy ? evx : evy;
            if (evalue > 1000000000.) status = DA_ERR_EIGEN;
            if (own) min_dx_dy_evalue = c_dmin1_2(c_dmin1_2(m->dx[i], m->dy[i]) / evalue, min_dx_dy_evalue);
        } else {
            kact[i] = p->epsilon;
        }
    }
    *min_dxe_out = min_dx_dy_evalue;
    *hmax_out = hmax;
    return status;
}

int orc_coef_eigen(const da_params *p, const da_mesh_soa *m, const double *h, const double *hu,
                   const double *hv, const double *slopes, double *kact, double *min_dxe_out,
                   double *hmax_out) {
    return coef_eigen_owned(p, m, m->n_cells, h, hu, hv, slopes, kact, min_dxe_out, hmax_out);
}

/* dt of get_coef_and_eigen.C:168-179 followed by TimeProps::incrtime (properties.h:397-410).
 * Returns the clipped dt; *time is advanced. */
double orc_dt(const da_params *p, double min_dxe, double hmax, double *time) {
    double g0 = 0.5 * min_dxe;
    double g1 = -0.9 * sqrt(hmax * (p->epsilon) * (p->gravity_scale) / 9.8);
    double dt = 0.5 * c_dmin1_2(g0, -g1);
    if (dt == 0.0) dt = 0.5 * p->influx_dt;
    if (*time + dt > p->next_output) dt = p->next_output - *time;
    if (*time + dt > p->next_save) dt = p->next_save - *time;
    if (*time + dt > p->max_time) dt = p->max_time - *time;
    *time += dt;
    return dt;
}

/* xdirflux / ydirflux with dz = 0 (order 1): src/datstr/element2.C:1810-1996.
 * hfv[0..2][0..2]: state, physical flux, wave speeds. */
static void dirflux(int dir, double h, double hu, double hv, double kact, double gz, double hfv[3][3]) {
    if (h < TINY) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) hfv[a][b] = 0.;
        return;
    }
    hfv[0][0] = h;
    hfv[0][1] = hu;
    hfv[0][2] = hv;
    if (dir == 0) {
        const double Vel = hfv[0][1] / hfv[0][0];
        const double a = sqrt(kact * hfv[0][0] * gz);
        hfv[1][0] = hfv[0][1];
        hfv[1][1] = hfv[0][1] * Vel + 0.5 * a * a * hfv[0][0];
        hfv[1][2] = hfv[0][2] * Vel;
        hfv[2][0] = Vel - a;
        hfv[2][1] = Vel;
        hfv[2][2] = Vel + a;
    } else {
        const double a = sqrt(kact * hfv[0][0] * gz);
        const double Vel = hfv[0][2] / hfv[0][0];
        hfv[1][0] = hfv[0][2];
        hfv[1][1] = hfv[0][1] * Vel;
        hfv[1][2] = hfv[0][2] * Vel + 0.5 * a * a * hfv[0][0];
        hfv[2][0] = Vel - a;
        hfv[2][1] = Vel;
        hfv[2][2] = Vel + a;
    }
}

/* riemannflux, src/datstr/element2.C:2228-2264 (HLL with Davis speeds). */
static void riemannflux(double hfvl[3][3], double hfvr[3][3], double flux[3]) {
    if ((hfvl[0][0] == 0.) && (hfvr[0][0] == 0.)) {
        for (int v = 0; v < 3; ++v) flux[v] = 0.;
        return;
    }
    double sl, sr;
    if (hfvl[0][0] == 0.) {
        sl = rmin(0, 2.0 * hfvr[2][0] - hfvr[2][1]);
        sr = rmax(0, 2.0 * hfvr[2][2] - hfvr[2][1]);
    } else if (hfvr[0][0] == 0.) {
        sl = rmin(0, 2.0 * hfvl[2][0] - hfvl[2][1]);
        sr = rmax(0, 2.0 * hfvl[2][2] - hfvl[2][1]);
    } else {
        sl = rmin(0, rmin(hfvl[2][0], hfvr[2][0]));
        sr = rmax(0, rmax(hfvl[2][2], hfvr[2][2]));
    }
    if (sl >= 0.0)
        for (int v = 0; v < 3; ++v) flux[v] = hfvl[1][v];
    else if (sr <= 0.0)
        for (int v = 0; v < 3; ++v) flux[v] = hfvr[1][v];
    else
        for (int v = 0; v < 3; ++v)
            flux[v] = (sr * hfvl[1][v] - sl * hfvr[1][v] + sl * sr * (hfvr[0][v] - hfvl[0][v])) / (sr - sl);
}

/* flux on the side-midpoint node of (cell, side): F[(side*3 + var)*n + cell] */
#define FN(F, n, cell, side, var) (F)[((size_t)(side) * 3 + (var)) * (n) + (cell)]

static void cell_hfv(const da_mesh_soa *m, const double *h, const double *hu, const double *hv,
                     const double *kact, int c, int dir, double hfv[3][3]) {
    dirflux(dir, h[c], hu[c], hv[c], kact[c], m->gravity[(size_t)2 * m->n_cells + c], hfv);
}

/* Element::calc_edge_states (single process: only +x/+y sides are owned), then
 * boundary_flux for the domain-edge cells.  F: [4][3][n]. */
void orc_edge_fluxes(const da_params *p, const da_mesh_soa *m, const double *h, const double *hu,
                     const double *hv, const double *kact, double *F) {
    (void)p;
    const int n = m->n_cells;
    double hfv[3][3], hfv1[3][3], hfv2[3][3], f[3];
    for (int i = 0; i < n; ++i) {
        for (int side = 0; side < 2; ++side) {
            const int zp = side, zm = side + 2;
            const int e1 = m->nbr[(size_t)zp * n + i];
            if (e1 < 0) continue; /* boundary: handled by boundary_flux */
            const int e2 = m->nbr[(size_t)(zp + 4) * n + i];
            cell_hfv(m, h, hu, hv, kact, i, side, hfv);
            cell_hfv(m, h, hu, hv, kact, e1, side, hfv1);
            riemannflux(hfv, hfv1, f);
            for (int v = 0; v < 3; ++v) FN(F, n, i, zp, v) = f[v];
            if (e2 != e1) {
                /* Case III, node S_C_CON: two finer neighbours; store both fine-side fluxes
                 * on their own nodes, then average onto this cell's node. */
                double f2[3];
                cell_hfv(m, h, hu, hv, kact, e2, side, hfv2);
                riemannflux(hfv, hfv2, f2);
                for (int v = 0; v < 3; ++v) {
                    FN(F, n, e1, zm, v) = f[v];
                    FN(F, n, e2, zm, v) = f2[v];
                    FN(F, n, i, zp, v) = 0.5 * (FN(F, n, e1, zm, v) + FN(F, n, e2, zm, v));
                }
            } else {
                const int b1 = m->nbr[(size_t)zm * n + e1], b2 = m->nbr[(size_t)(zm + 4) * n + e1];
                if (b1 == i && b2 == i) {
                    /* Case I: conforming, one shared node */
                    for (int v = 0; v < 3; ++v) FN(F, n, e1, zm, v) = f[v];
                } else {
                    /* Case II, node S_S_CON: this cell is one of two finer cells facing a coarser
                     * one; the sibling's flux is formed here too and both are averaged onto the
                     * coarse cell's node. */
                    const int sib = (b1 == i) ? b2 : b1;
                    double fs[3];
                    cell_hfv(m, h, hu, hv, kact, sib, side, hfv2);
                    riemannflux(hfv2, hfv1, fs);
                    for (int v = 0; v < 3; ++v) {
                        FN(F, n, sib, zp, v) = fs[v];
                        FN(F, n, e1, zm, v) = 0.5 * (f[v] + fs[v]);
                    }
                }
            }
        }
    }
    /* boundary_flux: x list first, then y list (edge_states.C:69-73) */
    for (int side = 0; side < 2; ++side)
        for (int i = 0; i < n; ++i) {
            const int zp = side, zm = side + 2;
            if (m->nbr[(size_t)zp * n + i] < 0)
                for (int v = 0; v < 3; ++v) FN(F, n, i, zp, v) = FN(F, n, i, zm, v);
            if (m->nbr[(size_t)zm * n + i] < 0)
                for (int v = 0; v < 3; ++v) FN(F, n, i, zm, v) = FN(F, n, i, zp, v);
        }
}

/* correct() -> update_states(), src/geoflow/corrector.C:36-193, src/adjoint/residual.C:162-275.
 * prev = state at the start of the step (update_prev_state_vars, step.C:194-195).
 * sgn_out [4][n] (orgSrcSgn) and stop_out [2][n] may be NULL.  Returns DA_ERR_NAN on NaN/Inf. */
int orc_correct(const da_params *p, const da_mesh_soa *m, const double *ph, const double *phu,
                const double *phv, const double *slopes, const double *kact, const double *F, double dt,
                double frict_tiny, double *h, double *hu, double *hv, double *sgn_out, int32_t *stop_out) {
    const int n = m->n_cells;
    const double sin_int_fric = sin(p->intfrict);
    int status = DA_OK;
    for (int i = 0; i < n; ++i) {
        const double prev[3] = {ph[i], phu[i], phv[i]};
        const double dtdx = dt / m->dx[i];
        const double dtdy = dt / m->dy[i];
        /* corrector.C:95-109: kact of a wet cell, epsilon otherwise */
        const double kactxyelem = (prev[0] > TINY) ? kact[i] : p->epsilon;
        const double bedfrict = p->bedfrict[m->material[i]];
        const double dx_[3] = {slopes[i], slopes[(size_t)n + i], slopes[(size_t)2 * n + i]};
        const double dy_[3] = {slopes[(size_t)3 * n + i], slopes[(size_t)4 * n + i], slopes[(size_t)5 * n + i]};
        const double *g = m->gravity, *dg = m->d_gravity, *cv = m->curvature;
        const double gravity[3] = {g[i], g[(size_t)n + i], g[(size_t)2 * n + i]};
        const double dgdx[2] = {dg[i], dg[(size_t)n + i]};
        const double curvature[2] = {cv[i], cv[(size_t)n + i]};
        double velocity[2], kactxy0, st[3];
        double orgSrcSgn[4] = {0, 0, 0, 0};
        int stop[2] = {0, 0};
        if (prev[0] > TINY) {
            kactxy0 = kactxyelem;
            velocity[0] = prev[1] / prev[0];
            velocity[1] = prev[2] / prev[0];
        } else {
            kactxy0 = 0.;
            velocity[0] = velocity[1] = 0.;
        }
        for (int v = 0; v < 3; ++v)
            st[v] = prev[v] - dtdx * (FN(F, n, i, 0, v) - FN(F, n, i, 2, v)) -
                    dtdy * (FN(F, n, i, 1, v) - FN(F, n, i, 3, v));
        if (st[0] < 0.) st[0] = 0;
        if (prev[0] > TINY) {
            const double h_inv = 1. / prev[0];
            double tmp = h_inv * (dy_[1] - velocity[0] * dy_[0]);
            orgSrcSgn[0] = tiny_sgn(tmp, frict_tiny);
            orgSrcSgn[2] = tiny_sgn(velocity[0], frict_tiny);
            tmp = h_inv * (dx_[2] - velocity[1] * dx_[0]);
            orgSrcSgn[1] = tiny_sgn(tmp, frict_tiny);
            orgSrcSgn[3] = tiny_sgn(velocity[1], frict_tiny);

            double s1 = gravity[0] * prev[0];
            double s2 = orgSrcSgn[0] * prev[0] * kactxy0 * (gravity[2] * dy_[0] + dgdx[1] * prev[0]) * sin_int_fric;
            const double tan_bed_fric = tan(bedfrict);
            double s3 = orgSrcSgn[2] * rmax(gravity[2] * prev[0] + velocity[0] * prev[1] * curvature[0], 0.0) *
                        tan_bed_fric;
            if (s3 == 0. && orgSrcSgn[2]) stop[0] = 1;
            st[1] += dt * (s1 - s2 - s3);

            s1 = gravity[1] * prev[0];
            s2 = orgSrcSgn[1] * prev[0] * kactxy0 * (gravity[2] * dx_[0] + dgdx[0] * prev[0]) * sin_int_fric;
            s3 = orgSrcSgn[3] * rmax(gravity[2] * prev[0] + velocity[1] * prev[2] * curvature[1], 0.0) *
                 tan_bed_fric;
            if (s3 == 0. && orgSrcSgn[3]) stop[1] = 1;
            st[2] += dt * (s1 - s2 - s3);
        }
        for (int v = 0; v < 3; ++v)
            if (isnan(st[v]) || isinf(st[v])) status = DA_ERR_NAN;
        h[i] = st[0];
        hu[i] = st[1];
        hv[i] = st[2];
        if (sgn_out)
            for (int k = 0; k < 4; ++k) sgn_out[(size_t)k * n + i] = orgSrcSgn[k];
        if (stop_out) {
            stop_out[i] = stop[0];
            stop_out[(size_t)n + i] = stop[1];
        }
    }
    return status;
}

/* One step() with order_flag = 1 (step.C:29-275).  State arrays are updated in place.
 * *time and *iter are TimeProps::time / ::iter; frict_tiny follows hpfem.C:232-235.
 * stats may be NULL; work must hold 14*n doubles (slopes 6n, kact n, prev 3n... see below). */
int orc_forward_step(const da_params *p, const da_mesh_soa *m, double *h, double *hu, double *hv,
                     double *time, int64_t *iter, da_step_stats *stats) {
    const int n = m->n_cells;
    double *slopes = (double *)malloc(sizeof(double) * 6 * (size_t)n);
    double *kact = (double *)malloc(sizeof(double) * (size_t)n);
    double *F = (double *)calloc(12 * (size_t)n, sizeof(double));
    double *prev = (double *)malloc(sizeof(double) * 3 * (size_t)n);
    if (!slopes || !kact || !F || !prev) {
        free(slopes); free(kact); free(F); free(prev);
        return DA_ERR_OOM;
    }
    const double frict_tiny = (*iter < p->frict_tiny_iters) ? p->frict_tiny_early : p->frict_tiny_late;
    orc_slopes(p, m, h, hu, hv, slopes);
    double min_dxe, hmax;
    int st = orc_coef_eigen(p, m, h, hu, hv, slopes, kact, &min_dxe, &hmax);
    const double dt = orc_dt(p, min_dxe, hmax, time);
    *iter += 1;
    orc_edge_fluxes(p, m, h, hu, hv, kact, F);
    memcpy(prev, h, sizeof(double) * n);
    memcpy(prev + n, hu, sizeof(double) * n);
    memcpy(prev + 2 * (size_t)n, hv, sizeof(double) * n);
    int st2 = orc_correct(p, m, prev, prev + n, prev + 2 * (size_t)n, slopes, kact, F, dt, frict_tiny, h, hu, hv,
                          NULL, NULL);
    if (stats) {
        double vol = 0.0;
        for (int i = 0; i < n; ++i) vol += m->dx[i] * m->dy[i] * h[i];
        stats->dt = dt;
        stats->time = *time;
        stats->volume = vol;
        stats->hmax = hmax;
        stats->iter = *iter;
    }
    free(slopes); free(kact); free(F); free(prev);
    if (st != DA_OK) return st;
    return st2;
}

int orc_forward_run(const da_params *p, const da_mesh_soa *m, double *h, double *hu, double *hv,
                    double *time, int64_t *iter, int nsteps, double *dt_hist, da_step_stats *last) {
    for (int k = 0; k < nsteps; ++k) {
        da_step_stats s;
        int st = orc_forward_step(p, m, h, hu, hv, time, iter, &s);
        if (dt_hist) dt_hist[k] = s.dt;
        if (last) *last = s;
        if (st != DA_OK) return st;
    }
    return DA_OK;
}

/* The two halves of one step on a subdomain whose cells [n_owned, n) are ghost copies of other
 * subdomains' cells (the domain-decomposed step: the ranks' CFL bounds meet in
 * MPI_Allreduce(MIN), get_coef_and_eigen.C:173, between the halves).
 * orc_step_bounds: slopes and k act/pass of every cell into work (7n doubles: slopes 6n, kact n);
 *   bounds[0] = min over the owned wet cells of min(dx,dy)/eigen (1e7 if none), bounds[1] = -hmax.
 * orc_step_apply: dt from the combined bounds (orc_dt), then the fluxes and the corrector of
 *   orc_forward_step from the same work array; *dt_out receives dt. */
int orc_step_bounds(const da_params *p, const da_mesh_soa *m, int n_owned, const double *h, const double *hu,
                    const double *hv, double *work, double *bounds) {
    const int n = m->n_cells;
    double *slopes = work, *kact = work + 6 * (size_t)n;
    orc_slopes(p, m, h, hu, hv, slopes);
    double min_dxe, hmax;
    const int st = coef_eigen_owned(p, m, n_owned, h, hu, hv, slopes, kact, &min_dxe, &hmax);
    bounds[0] = min_dxe;
    bounds[1] = -hmax;
    return st;
}

int orc_step_apply(const da_params *p, const da_mesh_soa *m, const double *bounds, const double *work,
                   double *h, double *hu, double *hv, double *time, int64_t *iter, double *dt_out) {
    const int n = m->n_cells;
    const double *slopes = work, *kact = work + 6 * (size_t)n;
    double *F = (double *)calloc(12 * (size_t)n, sizeof(double));
    double *prev = (double *)malloc(sizeof(double) * 3 * (size_t)n);
    if (!F || !prev) {
        free(F); free(prev);
        return DA_ERR_OOM;
    }
    const double frict_tiny = (*iter < p->frict_tiny_iters) ? p->frict_tiny_early : p->frict_tiny_late;
    const double dt = orc_dt(p, bounds[0], -bounds[1], time);
    *iter += 1;
    orc_edge_fluxes(p, m, h, hu, hv, kact, F);
    memcpy(prev, h, sizeof(double) * n);
    memcpy(prev + n, hu, sizeof(double) * n);
    memcpy(prev + 2 * (size_t)n, hv, sizeof(double) * n);
    const int st = orc_correct(p, m, prev, prev + n, prev + 2 * (size_t)n, slopes, kact, F, dt, frict_tiny, h, hu,
                               hv, NULL, NULL);
    if (dt_out) *dt_out = dt;
    free(F); free(prev);
    return st;
}

/* One step with a given dt (no CFL reduction): slopes, k act/pass, fluxes and the corrector of
 * orc_forward_step, frict_tiny by *iter as there.  The error grid's step of the DWR estimate takes
 * the coarse step's dt (error_grid_routines.C:13-55, error_compute.C:24-119). */
int orc_step_frozen(const da_params *p, const da_mesh_soa *m, double dt, double *h, double *hu, double *hv,
                    int64_t iter) {
    const int n = m->n_cells;
    double *work = (double *)malloc(sizeof(double) * 7 * (size_t)n);
    if (!work) return DA_ERR_OOM;
    double b[2];
    int st = orc_step_bounds(p, m, n, h, hu, hv, work, b);
    double *F = (double *)calloc(12 * (size_t)n, sizeof(double));
    double *prev = (double *)malloc(sizeof(double) * 3 * (size_t)n);
    if (!F || !prev) {
        free(work); free(F); free(prev);
        return DA_ERR_OOM;
    }
    const double frict_tiny = (iter < p->frict_tiny_iters) ? p->frict_tiny_early : p->frict_tiny_late;
    orc_edge_fluxes(p, m, h, hu, hv, work + 6 * (size_t)n, F);
    memcpy(prev, h, sizeof(double) * n);
    memcpy(prev + n, hu, sizeof(double) * n);
    memcpy(prev + 2 * (size_t)n, hv, sizeof(double) * n);
    const int st2 = orc_correct(p, m, prev, prev + n, prev + 2 * (size_t)n, work, work + 6 * (size_t)n, F, dt,
                                frict_tiny, h, hu, hv, NULL, NULL);
    free(work); free(F); free(prev);
    return st ? st : st2;
}
