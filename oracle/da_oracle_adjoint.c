/*
 * da_oracle_adjoint.c -- CPU restatement of the reference's discrete adjoint of one step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker for the CUDA adjoint, never linked by the product).
 *
 * It follows the reference's own structure, not the device kernels':
 *   - the forward state enters as the dual solver reads it back from its records (SolRec:
 *     a zero record for every cell with h <= 0, src/datstr/dualmesh.C:35-80);
 *   - slopes of that state with the depth-slope sensitivities hslope_sens
 *     (DualElem::get_slopes_prev, dualmesh.C:1393-1626) and k act/pass by gmfggetcoef
 *     (update_dual_grid, src/adjoint/dual_grid_routines.C:15-93);
 *   - flux Jacobians of every edge (dual_xdirflux / dual_ydirflux, src/datstr/element2.C:1858-2041;
 *     dual_riemannflux, dualmesh.C:1628-1843), stored per cell, direction, side and contributor
 *     with the hanging-edge averages and the boundary copies of DualElem::calc_flux /
 *     boundary_flux (dualmesh.C:1853-2279, FluxJac::set in src/header/matrix.h:215-245);
 *   - nine 3x3 blocks per cell (calc_jacobian, src/adjoint/calc_jacobain.C:40-153;
 *     set_fluxes_hsens :187-330; calc_jacobian_elem, src/adjoint/compute_jacobian_elem.C:15-121);
 *   - the adjoint gather lambda^{n-1}_i = -sum_e lambda^n_e . J_e[which(i)] with the flush of
 *     entries below 1e-16 (calc_adjoint_elem, src/adjoint/calc_adjoint.C:74-167).
 * Neighbour slots use the reference's absolute side numbering with positive_x_side = 1 (the
 * orientation the harness gives every element), so blocks are summed in the reference's order.
 * Build with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/discrete_adjoint.h"

#define TINY 1.e-4 /* GEOFLOW_TINY, src/header/constant.h:68 */

double orc_kact_cell(const da_params *p, int mat, double h, double hu, double hv, const double *dudx,
                     const double *dudy);

typedef double M3[3][3];

/* The reference's approximations of the exact transpose, each of which orc_adjoint_step_var can
 * keep or drop (orc_adjoint_step_ref keeps all of them):
 *   Q_RECORD    the state is read back from the dual solver's records, zero where h <= 0
 *               (record_solution, dualmesh.C:35-80), so a dry cell's momenta enter its
 *               neighbours' slopes (and so their sign tests) as zero;
 *   Q_VOID      blocks with respect to a cell whose record is zero are zero, its own block
 *               included (calc_jacobain.C:109-113, void_neigh_elem :155-166);
 *   Q_STOP      a neighbour's depth-slope term is dropped where the basal friction of that
 *               direction stopped (compute_jacobian_elem.C:48-55);
 *   Q_SLOPEFAC  depth-slope sensitivities without the limiter's sign factor .5 (c_sgn(dp) +
 *               c_sgn(dm)) and without gamma (hslope_sens, dualmesh.C:1484-1532);
 *   Q_DRYVDIFF  the HLL state-difference term sl sr / (sr - sl) I kept for a dry side, whose
 *               flux does not depend on its state (dual_riemannflux, dualmesh.C:1789-1799);
 *   Q_SRTIE     a tie between the two sides' fastest right-going speeds is taken from the left
 *               side (dualmesh.C:1755-1773);
 *   Q_FLUSH     adjoint entries below 1e-16 are set to zero (calc_adjoint.C:155-158). */
#define Q_RECORD 1
#define Q_VOID 2
#define Q_STOP 4
#define Q_SLOPEFAC 8
#define Q_DRYVDIFF 16
#define Q_SRTIE 32
#define Q_FLUSH 64
#define Q_ALL 127

static double dabs(double dd) { return dd < 0. ? -dd : dd; }
static double c_sgn(double zz) { /* geoflow.h:90-100 */
    if (zz > TINY) return 1;
    if (zz < -TINY) return -1;
    return 0;
}
static double c_dmin1_3(double d1, double d2, double d3) {
    if (d1 > d2) d1 = d2;
    if (d1 > d3) d1 = d3;
    return d1;
}
static double tiny_sgn(double num, double tiny) { /* residual.C:153-160 */
    if (dabs(num) < tiny) return 0.;
    if (num > tiny) return 1.;
    return -1.;
}
static void m_zero(M3 a) { memset(a, 0, sizeof(M3)); }
static void m_copy(M3 d, M3 s) { memcpy(d, s, sizeof(M3)); }
/* FluxJac::set(side, dir, index, jac1, jac2): (jac1 + jac2) * .5 */
static void m_avg(M3 d, M3 a, M3 b) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) d[i][j] = (a[i][j] + b[i][j]) * .5;
}

/* relative side r (0 +x, 1 +y, 2 -x, 3 -y) of absolute side a with positive_x_side = 1 */
static int rel_of_abs(int a) { return (a + 3) % 4; }

/* neighbour slot a (0..7, absolute) of cell c: the cell, or -1 at the domain boundary */
static int nb_abs(const da_mesh_soa *m, int c, int a) {
    const int n = m->n_cells, r = rel_of_abs(a & 3);
    return m->nbr[(size_t)(r + (a & 4)) * n + c];
}
/* neigh_proc of slot a: -1 boundary, -2 a repeated first neighbour, 0 a neighbour */
static int nproc_abs(const da_mesh_soa *m, int c, int a) {
    const int n = m->n_cells, r = rel_of_abs(a & 3);
    const int e1 = m->nbr[(size_t)r * n + c];
    if (a < 4) return e1 < 0 ? -1 : 0;
    const int e2 = m->nbr[(size_t)(r + 4) * n + c];
    return (e1 < 0 || e2 == e1) ? -2 : 0;
}
/* Element::which_neighbor (element2.C:574-583): first slot holding key with neigh_proc >= 0 */
static int which_neighbor(const da_mesh_soa *m, int e, int c) {
    for (int a = 0; a < 8; ++a)
        if (nb_abs(m, e, a) == c && nproc_abs(m, e, a) >= 0) return a;
    return 8;
}

/* dual_xdirflux / dual_ydirflux (element2.C:1858-2041): hfv, d flux / d U, d speeds / d U */
static void dual_dirflux(int dir, const double U[3], double kact, double gz, M3 hfv, M3 fj, M3 sj) {
    m_zero(hfv);
    m_zero(fj);
    m_zero(sj);
    if (U[0] < TINY) return;
    for (int i = 0; i < 3; ++i) hfv[0][i] = U[i];
    if (dir == 0) {
        const double h_inv = 1. / hfv[0][0];
        const double Vel = hfv[0][1] * h_inv;
        const double a = sqrt(kact * hfv[0][0] * gz);
        hfv[1][0] = hfv[0][1];
        hfv[1][1] = hfv[0][1] * Vel + 0.5 * a * a * hfv[0][0];
        hfv[1][2] = hfv[0][2] * Vel;
        hfv[2][0] = Vel - a;
        hfv[2][1] = Vel;
        hfv[2][2] = Vel + a;
        fj[0][1] = 1.;
        fj[1][0] = a * a - Vel * Vel;
        fj[1][1] = 2 * Vel;
        fj[2][0] = -Vel * hfv[0][2] * h_inv;
        fj[2][1] = hfv[0][2] * h_inv;
        fj[2][2] = Vel;
        sj[0][0] = -.5 * a * h_inv - Vel * h_inv;
        sj[0][1] = h_inv;
        sj[1][0] = -Vel * h_inv;
        sj[1][1] = h_inv;
        sj[2][0] = .5 * a * h_inv - Vel * h_inv;
        sj[2][1] = h_inv;
    } else {
        const double a = sqrt(kact * hfv[0][0] * gz);
        const double h_inv = 1. / hfv[0][0];
        const double Vel = hfv[0][2] * h_inv;
        hfv[1][0] = hfv[0][2];
        hfv[1][1] = hfv[0][1] * Vel;
        hfv[1][2] = hfv[0][2] * Vel + 0.5 * a * a * hfv[0][0];
        hfv[2][0] = Vel - a;
        hfv[2][1] = Vel;
        hfv[2][2] = Vel + a;
        fj[0][2] = 1.;
        fj[1][0] = -Vel * hfv[0][1] * h_inv;
        fj[1][1] = Vel;
        fj[1][2] = hfv[0][1] * h_inv;
        fj[2][0] = a * a - Vel * Vel;
        fj[2][2] = 2 * Vel;
        sj[0][0] = -.5 * a * h_inv - Vel * h_inv;
        sj[0][2] = h_inv;
        sj[1][0] = -Vel * h_inv;
        sj[1][2] = h_inv;
        sj[2][0] = .5 * a * h_inv - Vel * h_inv;
        sj[2][2] = h_inv;
    }
}

/* dual_riemannflux (dualmesh.C:1628-1843): d F_HLL / d U_left, d U_right */
static void dual_riemann(M3 hl, M3 hr, M3 fjl, M3 fjr, M3 sjl, M3 sjr, M3 jl, M3 jr, int keep) {
    m_zero(jl);
    m_zero(jr);
    if (hl[0][0] == 0. && hr[0][0] == 0.) return;
    double sl, sr, dsl_l[3], dsl_r[3], dsr_l[3], dsr_r[3];
    if (hl[0][0] == 0.) {
        for (int i = 0; i < 3; ++i) dsr_l[i] = dsl_l[i] = 0.;
        sl = fmin(0., 2. * hr[2][0] - hr[2][1]);
        for (int i = 0; i < 3; ++i) dsl_r[i] = sl == 0 ? 0. : 2 * sjr[0][i] - sjr[1][i];
        sr = fmax(0., 2. * hr[2][2] - hr[2][1]);
        for (int i = 0; i < 3; ++i) dsr_r[i] = sr == 0 ? 0. : 2 * sjr[2][i] - sjr[1][i];
    } else if (hr[0][0] == 0.) {
        for (int i = 0; i < 3; ++i) dsr_r[i] = dsl_r[i] = 0.;
        sl = fmin(0., 2. * hl[2][0] - hl[2][1]);
        for (int i = 0; i < 3; ++i) dsl_l[i] = sl == 0 ? 0. : 2 * sjl[0][i] - sjl[1][i];
        sr = fmax(0., 2. * hl[2][2] - hl[2][1]);
        for (int i = 0; i < 3; ++i) dsr_l[i] = sr == 0 ? 0. : 2 * sjl[2][i] - sjl[1][i];
    } else {
        sl = fmin(0., fmin(hl[2][0], hr[2][0]));
        if (sl == 0) {
            for (int i = 0; i < 3; ++i) dsl_l[i] = dsl_r[i] = 0.;
        } else if (sl == hl[2][0]) {
            for (int i = 0; i < 3; ++i) {
                dsl_r[i] = 0.;
                dsl_l[i] = sjl[0][i];
            }
        } else {
            for (int i = 0; i < 3; ++i) {
                dsl_l[i] = 0.;
                dsl_r[i] = sjr[0][i];
            }
        }
        sr = fmax(0., fmax(hl[2][2], hr[2][2]));
        if (sr == 0) {
            for (int i = 0; i < 3; ++i) dsr_l[i] = dsr_r[i] = 0.;
        } else if (sr == hl[2][2] && ((keep & Q_SRTIE) || hl[2][2] != hr[2][2])) {
            for (int i = 0; i < 3; ++i) {
                dsr_r[i] = 0.;
                dsr_l[i] = sjl[2][i];
            }
        } else {
            for (int i = 0; i < 3; ++i) {
                dsr_l[i] = 0.;
                dsr_r[i] = sjr[2][i];
            }
        }
    }
    if (sl >= 0.) {
        m_copy(jl, fjl);
    } else if (sr <= 0.) {
        m_copy(jr, fjr);
    } else {
        const double inv = 1. / (sr - sl);
        double vd[3], flux[3], dfsr[3], dfsl[3];
        for (int i = 0; i < 3; ++i) vd[i] = hr[0][i] - hl[0][i];
        for (int i = 0; i < 3; ++i) flux[i] = (sr * hl[1][i] - sl * hr[1][i] + sl * sr * vd[i]) * inv;
        for (int i = 0; i < 3; ++i) {
            dfsr[i] = (hl[1][i] + sl * vd[i] - flux[i]) * inv;
            dfsl[i] = (-hr[1][i] + sr * vd[i] + flux[i]) * inv;
        }
        const double dfr = -sl * inv, dfl = sr * inv;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double vr = i == j ? sr * sl * inv : 0., vl = i == j ? -sr * sl * inv : 0.;
                if (!(keep & Q_DRYVDIFF)) {
                    if (hr[0][0] == 0.) vr = 0.;
                    if (hl[0][0] == 0.) vl = 0.;
                }
                jr[i][j] = dfsr[i] * dsr_r[j] + dfsl[i] * dsl_r[j] + dfr * fjr[i][j] + vr;
                jl[i][j] = dfsr[i] * dsr_l[j] + dfsl[i] * dsl_l[j] + dfl * fjl[i][j] + vl;
            }
    }
}

/* calc_jacobian_elem (compute_jacobian_elem.C:15-121) */
static void jacobian_elem(M3 J, M3 jnx, M3 jpx, M3 jny, M3 jpy, const double prev[3], const double dx_[3],
                          const double dy_[3], const double curv[2], const double g[3], const double dg[2],
                          const double dh_sens[2], double int_fric, double bedfrict, double kact, int eff, double dtdx,
                          double dtdy, double dt, const int stop_in[2], const double sgn[4], int keep) {
    const int stop_n[2] = {(keep & Q_STOP) ? stop_in[0] : 0, (keep & Q_STOP) ? stop_in[1] : 0};
    const int *stop = stop_in;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) J[i][j] = +dtdx * (jpx[i][j] - jnx[i][j]) + dtdy * (jpy[i][j] - jny[i][j]);
    if (eff == 0)
        for (int i = 0; i < 3; ++i) J[i][i] -= 1.;
    if (prev[0] > TINY) {
        const double sin_int_fric = sin(int_fric);
        const double alpha = sin_int_fric * sgn[0] * kact;
        const double betta = sin_int_fric * sgn[1] * kact;
        if (eff > 0) {
            if (!stop_n[0]) J[1][0] -= -dt * prev[0] * alpha * g[2] * dh_sens[1];
            if (!stop_n[1]) J[2][0] -= -dt * prev[0] * betta * g[2] * dh_sens[0];
        } else {
            const double velocity[2] = {prev[1] / prev[0], prev[2] / prev[0]};
            const double vx_sq = velocity[0] * velocity[0], vy_sq = velocity[1] * velocity[1];
            const double tan_bed_frict = tan(bedfrict);
            J[1][0] -= dt * (g[0] - alpha * prev[0] * (2 * dg[1] + g[2] * dh_sens[1]) - alpha * g[2] * dy_[0]);
            if (sgn[2] != 0. && !stop[0]) {
                J[1][0] -= -dt * sgn[2] * tan_bed_frict * (g[2] - vx_sq * curv[0]);
                J[1][1] -= -dt * sgn[2] * tan_bed_frict * (2 * velocity[0] * curv[0]);
                J[1][2] -= 0.;
            }
            J[2][0] -= dt * (g[1] - betta * prev[0] * (2 * dg[0] + g[2] * dh_sens[0]) - betta * g[2] * dx_[0]);
            if (sgn[3] != 0. && !stop[1]) {
                J[2][0] -= -dt * sgn[3] * tan_bed_frict * (g[2] - vy_sq * curv[1]);
                J[2][1] -= 0.;
                J[2][2] -= -dt * sgn[3] * tan_bed_frict * (2 * velocity[1] * curv[1]);
            }
        }
    }
}

/* the stop flags and friction signs of update_states (residual.C:162-275) */
static void src_signs(const double prev[3], const double dx_[3], const double dy_[3], const double g[3],
                      const double curv[2], double bedfrict, double fric_tiny, int stop[2], double sgn[4]) {
    stop[0] = stop[1] = 0;
    sgn[0] = sgn[1] = sgn[2] = sgn[3] = 0.;
    if (!(prev[0] > TINY)) return;
    const double velocity[2] = {prev[1] / prev[0], prev[2] / prev[0]};
    const double h_inv = 1. / prev[0];
    double tmp = h_inv * (dy_[1] - velocity[0] * dy_[0]);
    sgn[0] = tiny_sgn(tmp, fric_tiny);
    sgn[2] = tiny_sgn(velocity[0], fric_tiny);
    tmp = h_inv * (dx_[2] - velocity[1] * dx_[0]);
    sgn[1] = tiny_sgn(tmp, fric_tiny);
    sgn[3] = tiny_sgn(velocity[1], fric_tiny);
    const double tan_bed_fric = tan(bedfrict);
    const double px = g[2] * prev[0] + velocity[0] * prev[1] * curv[0];
    const double s3x = sgn[2] * (px > 0.0 ? px : 0.0) * tan_bed_fric;
    if (s3x == 0. && sgn[2]) stop[0] = 1;
    const double py = g[2] * prev[0] + velocity[1] * prev[2] * curv[1];
    const double s3y = sgn[3] * (py > 0.0 ? py : 0.0) * tan_bed_fric;
    if (s3y == 0. && sgn[3]) stop[1] = 1;
}

/* DualElem::get_slopes_prev (dualmesh.C:1393-1626) for one direction of cell i: the limited
 * slopes of the recorded state in that direction (d[3]) with reciprocal products as the dual
 * solver forms them, and hs[5], d (dh/dx) / d h of self, m1, p1, m2, p2 */
static void dual_slopes_dir(const da_mesh_soa *m, const double *P[3], int i, int dir, double gamma, double d[3],
                            double hs[5], int keep) {
    const int n = m->n_cells;
    const int ep = m->nbr[(size_t)dir * n + i], em = m->nbr[(size_t)(dir + 2) * n + i];
    const int ep2r = m->nbr[(size_t)(dir + 4) * n + i], em2r = m->nbr[(size_t)(dir + 6) * n + i];
    const int ep2 = ep2r != ep ? ep2r : -1, em2 = em2r != em ? em2r : -1;
    const double *co = dir == 0 ? m->x : m->y;
    const double dxp = co[ep] - co[i], dxm = co[i] - co[em];
    const double inv_dxp = 1 / dxp, inv_dxm = 1 / dxm, inv_s = 1 / (dxm + dxp);
    for (int j = 0; j < 3; ++j) {
        const double *V = P[j];
        double dp = (V[ep] - V[i]) * inv_dxp;
        if (ep2 >= 0) dp = .5 * (dp + (V[ep2] - V[i]) * inv_dxp);
        double dm = (V[i] - V[em]) * inv_dxm;
        if (em2 >= 0) dm = .5 * (dm + (V[i] - V[em2]) * inv_dxm);
        const double dc = (dp * dxm + dm * dxp) * inv_s;
        const double mn = c_dmin1_3(gamma * dabs(dp), gamma * dabs(dm), dabs(dc));
        d[j] = .5 * (c_sgn(dp) + c_sgn(dm)) * mn;
        if (j != 0) continue;
        for (int k = 0; k < 5; ++k) hs[k] = 0.;
        if (.5 * (c_sgn(dp) + c_sgn(dm)) == 0) continue;
        /* the exact derivative carries the limiter's sign factor and gamma as well */
        const double fac = .5 * (c_sgn(dp) + c_sgn(dm));
        const double sg_dp = dp > 0 ? 1. : (dp < 0 ? -1. : 0.), sg_dm = dm > 0 ? 1. : (dm < 0 ? -1. : 0.);
        const double sg_dc = dc > 0 ? 1. : (dc < 0 ? -1. : 0.);
        double q = 1.;
        if (mn == gamma * dabs(dp)) {
            hs[0] = -inv_dxp;
            hs[2] = inv_dxp;
            if (ep2 >= 0) hs[2] = hs[4] = .5 * inv_dxp;
            q = fac * gamma * sg_dp;
        } else if (mn == gamma * dabs(dm)) {
            hs[0] = inv_dxm;
            hs[1] = -inv_dxm;
            if (em2 >= 0) hs[1] = hs[3] = -.5 * inv_dxm;
            q = fac * gamma * sg_dm;
        } else {
            q = fac * sg_dc;
            hs[0] = inv_dxm - inv_dxp;
            hs[1] = -inv_dxm;
            hs[2] = inv_dxp;
            if (ep2 >= 0) hs[2] = hs[4] = .5 * inv_dxp;
            if (em2 >= 0) hs[1] = hs[3] = -.5 * inv_dxm;
            hs[1] *= dxp * inv_s;
            hs[2] *= dxm * inv_s;
            hs[3] *= dxp * inv_s;
            hs[4] *= dxm * inv_s;
        }
        if (!(keep & Q_SLOPEFAC))
            for (int k = 0; k < 5; ++k) hs[k] *= q;
    }
}

/* FJ index: cell c, direction side (0 x, 1 y), dir (0 minus, 1 plus), contributor k (0 self,
 * 1 first neighbour, 2 second neighbour) */
#define FJ(c, side, dir, k) fj[(((size_t)(c) * 2 + (side)) * 2 + (dir)) * 3 + (k)]

/*
 * One reverse step of the reference's dual solver.  (h, hu, hv): the forward state U^{n-1} the
 * step starts from (as the forward computed it); dt: that step's time step; frict_tiny: its
 * threshold (calc_jacobain.C:82-85); lam_next [3][n]: the adjoint of U^n; lam_out [3][n]: the
 * adjoint of U^{n-1} with a zero functional sensitivity.  Returns DA_OK or DA_ERR_OOM.
 */
static int adjoint_step_ccw(const da_params *p, const da_mesh_soa *m, const double *h, const double *hu,
                            const double *hv, double dt, double frict_tiny, const double *lam_next, double *lam_out,
                            int keep);

/* The reference keeps a side's two finer neighbours in the counter-clockwise order of the element's
 * boundary (adapt/refine2.C:590-805): +x lower then upper, +y right then left, -x upper then lower,
 * -y left then right; the flattened table lists the lower / left one first.  The dual solver sums
 * its blocks in slot order, so the step below runs on the table with the +y and -x pairs in the
 * reference's order. */
int orc_adjoint_step_var(const da_params *p, const da_mesh_soa *m, const double *h, const double *hu,
                         const double *hv, double dt, double frict_tiny, const double *lam_next, double *lam_out,
                         int keep) {
    const int n = m->n_cells;
    int32_t *nb = (int32_t *)malloc(sizeof(int32_t) * 8 * (size_t)n);
    if (!nb) return DA_ERR_OOM;
    memcpy(nb, m->nbr, sizeof(int32_t) * 8 * (size_t)n);
    for (int r = 1; r <= 2; ++r)
        for (int c = 0; c < n; ++c) {
            const int32_t t = nb[(size_t)r * n + c];
            nb[(size_t)r * n + c] = nb[(size_t)(r + 4) * n + c];
            nb[(size_t)(r + 4) * n + c] = t;
        }
    da_mesh_soa mc = *m;
    mc.nbr = nb;
    const int st = adjoint_step_ccw(p, &mc, h, hu, hv, dt, frict_tiny, lam_next, lam_out, keep);
    free(nb);
    return st;
}

static int adjoint_step_ccw(const da_params *p, const da_mesh_soa *m, const double *h, const double *hu,
                            const double *hv, double dt, double frict_tiny, const double *lam_next, double *lam_out,
                            int keep) {
    const int n = m->n_cells;
    double *P = (double *)malloc(sizeof(double) * 3 * (size_t)n);
    double *S = (double *)malloc(sizeof(double) * 6 * (size_t)n);
    double *kact = (double *)malloc(sizeof(double) * (size_t)n);
    double *hs = (double *)malloc(sizeof(double) * 10 * (size_t)n);
    M3 *fj = (M3 *)calloc((size_t)n * 12, sizeof(M3));
    M3 *jac = (M3 *)calloc((size_t)n * 9, sizeof(M3));
    if (!P || !S || !kact || !hs || !fj || !jac) {
        free(P); free(S); free(kact); free(hs); free(fj); free(jac);
        return DA_ERR_OOM;
    }
    double *Ph = P, *Phu = P + n, *Phv = P + 2 * (size_t)n;
    /* the dual solver's record of U^{n-1}: a zero record where h <= 0 */
    for (int i = 0; i < n; ++i) {
        const int rec = h[i] > 0. || !(keep & Q_RECORD);
        Ph[i] = rec ? h[i] : 0.;
        Phu[i] = rec ? hu[i] : 0.;
        Phv[i] = rec ? hv[i] : 0.;
    }
    const double *PV[3] = {Ph, Phu, Phv};
    for (int i = 0; i < n; ++i) {
        int bc = 0;
        for (int s4 = 0; s4 < 4; ++s4) bc |= m->nbr[(size_t)s4 * n + i] < 0;
        double d[2][3] = {{0., 0., 0.}, {0., 0., 0.}};
        for (int k = 0; k < 10; ++k) hs[(size_t)i * 10 + k] = 0.;
        if (!bc)
            for (int dir = 0; dir < 2; ++dir)
                dual_slopes_dir(m, PV, i, dir, p->gamma, d[dir], &hs[(size_t)i * 10 + dir * 5], keep);
        for (int j = 0; j < 3; ++j) {
            S[(size_t)j * n + i] = d[0][j];
            S[(size_t)(j + 3) * n + i] = d[1][j];
        }
        kact[i] = orc_kact_cell(p, m->material[i], Ph[i], Phu[i], Phv[i], d[0], d[1]);
    }
    const double *gz = m->gravity + 2 * (size_t)n;
    /* DualElem::calc_flux for each cell and direction, then boundary_flux (edge_states.C:79-120) */
    for (int i = 0; i < n; ++i) {
        const double Ui[3] = {Ph[i], Phu[i], Phv[i]};
        for (int side = 0; side < 2; ++side) {
            const int zp = side;
            const int e1 = m->nbr[(size_t)zp * n + i];
            if (e1 < 0) continue;
            M3 hfv, fjv, sjv, hfv1, fj1, sj1, hfv2, fj2, sj2, jc, jn1, jn2, jres;
            const double U1[3] = {Ph[e1], Phu[e1], Phv[e1]};
            dual_dirflux(side, Ui, kact[i], gz[i], hfv, fjv, sjv);
            dual_dirflux(side, U1, kact[e1], gz[e1], hfv1, fj1, sj1);
            dual_riemann(hfv, hfv1, fjv, fj1, sjv, sj1, jc, jn1, keep);
            m_copy(FJ(i, side, 1, 0), jc);
            m_copy(FJ(i, side, 1, 1), jn1);
            m_zero(FJ(i, side, 1, 2));
            m_copy(FJ(e1, side, 0, 0), jn1);
            m_copy(FJ(e1, side, 0, 1), jc);
            m_zero(FJ(e1, side, 0, 2));
            const int e2r = m->nbr[(size_t)(zp + 4) * n + i];
            const int lvl_coarser = m->nbr[(size_t)(zp + 2) * n + e1] != m->nbr[(size_t)(zp + 6) * n + e1];
            if (e2r != e1) {
                /* S_C_CON: two finer neighbours */
                const int e2 = e2r;
                const double U2[3] = {Ph[e2], Phu[e2], Phv[e2]};
                dual_dirflux(side, U2, kact[e2], gz[e2], hfv2, fj2, sj2);
                dual_riemann(hfv, hfv2, fjv, fj2, sjv, sj2, jres, jn2, keep);
                M3 z;
                m_zero(z);
                m_avg(FJ(i, side, 1, 0), jc, jres);
                m_avg(FJ(i, side, 1, 1), jn1, z);
                m_avg(FJ(i, side, 1, 2), jn2, z);
                m_copy(FJ(e2, side, 0, 0), jn2);
                m_copy(FJ(e2, side, 0, 1), jres);
                m_zero(FJ(e2, side, 0, 2));
            } else if (lvl_coarser) {
                /* S_S_CON: this cell is one of two finer cells facing e1 */
                const int zel = which_neighbor(m, e1, i);
                const int e2 = nb_abs(m, e1, (zel + 4) % 8);
                const double U2[3] = {Ph[e2], Phu[e2], Phv[e2]};
                dual_dirflux(side, U1, kact[e1], gz[e1], hfv1, fj1, sj1);
                dual_dirflux(side, U2, kact[e2], gz[e2], hfv2, fj2, sj2);
                dual_riemann(hfv2, hfv1, fj2, fj1, sj2, sj1, jn2, jres, keep);
                M3 z;
                m_zero(z);
                m_avg(FJ(e1, side, 0, 0), jn1, jres);
                if (zel < 4) {
                    m_avg(FJ(e1, side, 0, 1), jc, z);
                    m_avg(FJ(e1, side, 0, 2), jn2, z);
                } else {
                    m_avg(FJ(e1, side, 0, 1), jn2, z);
                    m_avg(FJ(e1, side, 0, 2), jc, z);
                }
            }
        }
    }
    for (int side = 0; side < 2; ++side)
        for (int i = 0; i < n; ++i) {
            const int bp = m->nbr[(size_t)side * n + i] < 0, bm = m->nbr[(size_t)(side + 2) * n + i] < 0;
            /* each cell of the list runs boundary_flux once per boundary side it was listed for */
            for (int rep = 0; rep < bp + bm; ++rep) {
                if (bp)
                    for (int k = 0; k < 3; ++k) m_copy(FJ(i, side, 1, k), FJ(i, side, 0, k));
                if (bm)
                    for (int k = 0; k < 3; ++k) m_copy(FJ(i, side, 0, k), FJ(i, side, 1, k));
            }
        }
    /* calc_jacobian */
    for (int i = 0; i < n; ++i) {
        const double prev[3] = {Ph[i], Phu[i], Phv[i]};
        const double dx_[3] = {S[i], S[(size_t)n + i], S[(size_t)2 * n + i]};
        const double dy_[3] = {S[(size_t)3 * n + i], S[(size_t)4 * n + i], S[(size_t)5 * n + i]};
        const double g[3] = {m->gravity[i], m->gravity[(size_t)n + i], m->gravity[(size_t)2 * n + i]};
        const double dg[2] = {m->d_gravity[i], m->d_gravity[(size_t)n + i]};
        const double cv[2] = {m->curvature[i], m->curvature[(size_t)n + i]};
        const double bedfrict = p->bedfrict[m->material[i]];
        int stop[2];
        double sgn[4];
        src_signs(prev, dx_, dy_, g, cv, bedfrict, frict_tiny, stop, sgn);
        const double dtdx = dt / m->dx[i], dtdy = dt / m->dy[i];
        const double *hsi = &hs[(size_t)i * 10];
        for (int eff = 0; eff < 9; ++eff) {
            M3 *J = &jac[(size_t)i * 9 + eff];
            const int a = eff - 1;
            int zero = 0;
            if (eff == 0 && prev[0] == 0. && (keep & Q_VOID)) zero = 1;
            if (eff > 4 && nproc_abs(m, i, a) == -2) zero = 1;
            if (eff != 0 && !zero) {
                const int e = nb_abs(m, i, a);
                if (e < 0 || (Ph[e] == 0. && (keep & Q_VOID))) zero = 1;
            }
            if (eff > 0 && nproc_abs(m, i, a) == -1) zero = 1;
            if (zero) {
                m_zero(*J);
                continue;
            }
            M3 Z;
            m_zero(Z);
            double (*jnx)[3] = Z, (*jpx)[3] = Z, (*jny)[3] = Z, (*jpy)[3] = Z;
            double dh[2] = {0., 0.};
            if (eff == 0) {
                jnx = FJ(i, 0, 0, 0);
                jpx = FJ(i, 0, 1, 0);
                jny = FJ(i, 1, 0, 0);
                jpy = FJ(i, 1, 1, 0);
                dh[0] = hsi[0];
                dh[1] = hsi[5];
            } else {
                const int r = rel_of_abs(a & 3), idx = eff <= 4 ? 1 : 2;
                const int boundary = m->nbr[(size_t)((r + 2) % 4) * n + i] < 0;
                const int hp = eff <= 4 ? 2 : 4, hm = eff <= 4 ? 1 : 3;
                if (r == 0) {
                    dh[0] = hsi[hp];
                    jpx = FJ(i, 0, 1, idx);
                    if (boundary) jnx = FJ(i, 0, 0, idx);
                } else if (r == 2) {
                    dh[0] = hsi[hm];
                    jnx = FJ(i, 0, 0, idx);
                    if (boundary) jpx = FJ(i, 0, 1, idx);
                } else if (r == 1) {
                    dh[1] = hsi[5 + hp];
                    jpy = FJ(i, 1, 1, idx);
                    if (boundary) jny = FJ(i, 1, 0, idx);
                } else {
                    dh[1] = hsi[5 + hm];
                    jny = FJ(i, 1, 0, idx);
                    if (boundary) jpy = FJ(i, 1, 1, idx);
                }
            }
            jacobian_elem(*J, jnx, jpx, jny, jpy, prev, dx_, dy_, cv, g, dg, dh, p->intfrict, bedfrict, kact[i], eff,
                          dtdx, dtdy, dt, stop, sgn, keep);
        }
    }
    /* calc_adjoint_elem */
    for (int i = 0; i < n; ++i) {
        double ac[3] = {0., 0., 0.};
        for (int eff = 0; eff < 9; ++eff) {
            if (eff == 0) {
                M3 *J = &jac[(size_t)i * 9];
                for (int k = 0; k < 3; ++k)
                    for (int l = 0; l < 3; ++l) ac[k] += lam_next[(size_t)l * n + i] * (*J)[l][k];
                continue;
            }
            const int a = eff - 1;
            if (!(eff <= 4 || nproc_abs(m, i, a) > -2)) continue;
            const int e = nb_abs(m, i, a);
            if (e < 0) continue;
            const int jacind = which_neighbor(m, e, i) + 1;
            M3 *J = &jac[(size_t)e * 9 + jacind];
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l) ac[k] += lam_next[(size_t)l * n + e] * (*J)[l][k];
        }
        for (int j = 0; j < 3; ++j) {
            double v = 0. - ac[j];
            if ((keep & Q_FLUSH) && fabs(v) < 1e-16) v = 0.;
            lam_out[(size_t)j * n + i] = v;
        }
    }
    free(P); free(S); free(kact); free(hs); free(fj); free(jac);
    return DA_OK;
}

/* The reference's own adjoint step: every approximation kept. */
int orc_adjoint_step_ref(const da_params *p, const da_mesh_soa *m, const double *h, const double *hu,
                         const double *hv, double dt, double frict_tiny, const double *lam_next, double *lam_out) {
    return orc_adjoint_step_var(p, m, h, hu, hv, dt, frict_tiny, lam_next, lam_out, Q_ALL);
}
