/*
 * da_oracle_split.c -- CPU model of the FP32 / FP64 precision split of the forward step.
 *
 * TEST INFRASTRUCTURE ONLY: it measures, against the FP64 restatement in da_oracle.c, how a
 * precision split of the reference's step (order_flag = 1, src/geoflow/step.C:29-275) drifts; the
 * product never links it.  The split modelled here keeps the state in FP64 and accumulates the
 * corrector in FP64 (U^{n+1} = U^n - dt/dx dF - dt/dy dG + dt S with the differences and sums in
 * FP64), while every flux and source term is computed in FP32: the limited slopes
 * (Element::get_slopes, src/datstr/element2.C:830-939), k act/pass (getcoef.f), the Davis wave
 * speeds and the CFL bound (eigen.f), the physical fluxes and the HLL flux (element2.C:1810-2264),
 * and the gravity, internal- and basal-friction sources with their sign tests
 * (update_states, src/adjoint/residual.C:162-275).  The dt reduction, the time and the clipping stay
 * FP64.  Built with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/discrete_adjoint.h"

#define TINYF 1.e-4f

static float fabsf_(float v) { return v < 0.f ? -v : v; }
static float c_sgnf(float z) { return z > TINYF ? 1.f : (z < -TINYF ? -1.f : 0.f); }
static float tiny_sgnf(float v, float t) { return fabsf_(v) < t ? 0.f : (v > t ? 1.f : -1.f); }
static int fsgnf(float z, float t) { return fabsf_(z) < t ? 0 : (z >= t ? 1 : -1); }
static float rmaxf(float x, float y) { return x > y ? x : y; }
static float rminf(float x, float y) { return x > y ? y : x; }

/* k act/pass of the three sgn(vel) branches of one material (getcoef.f), in FP32 */
static float kact_f(const da_params *p, int mat, float h, float hu, float hv, const float *sx, const float *sy) {
    if (!(h > TINYF)) return (float)p->epsilon;
    const float vel = sx[1] / h - hu * sx[0] / (h * h) + sy[2] / h - hv * sy[0] / (h * h);
    const float c = cosf((float)p->intfrict), t = tanf((float)p->bedfrict[mat]);
    float k = (2.f / (c * c)) * (1.f - (float)fsgnf(vel, TINYF) * sqrtf(fabsf_(1.f - (1.f + t * t) * (c * c)))) - 1.f;
    if (fabsf_(hu / h) < TINYF && fabsf_(hv / h) < TINYF) k = 1.f;
    if (k < 0.f) k = 0.f;
    return k * (float)p->epsilon;
}

static void dirflux_f(int dir, float h, float hu, float hv, float k, float gz, float o[3][3]) {
    memset(o, 0, sizeof(float) * 9);
    if (h < TINYF) return;
    o[0][0] = h; o[0][1] = hu; o[0][2] = hv;
    const float a = sqrtf(k * h * gz);
    const float vel = (dir == 0 ? hu : hv) / h;
    if (dir == 0) {
        o[1][0] = hu; o[1][1] = hu * vel + 0.5f * a * a * h; o[1][2] = hv * vel;
    } else {
        o[1][0] = hv; o[1][1] = hu * vel; o[1][2] = hv * vel + 0.5f * a * a * h;
    }
    o[2][0] = vel - a; o[2][1] = vel; o[2][2] = vel + a;
}

static void riemann_f(float l[3][3], float r[3][3], float f[3]) {
    if (l[0][0] == 0.f && r[0][0] == 0.f) {
        f[0] = f[1] = f[2] = 0.f;
        return;
    }
    float sl, sr;
    if (l[0][0] == 0.f) {
        sl = rminf(0.f, 2.f * r[2][0] - r[2][1]);
        sr = rmaxf(0.f, 2.f * r[2][2] - r[2][1]);
    } else if (r[0][0] == 0.f) {
        sl = rminf(0.f, 2.f * l[2][0] - l[2][1]);
        sr = rmaxf(0.f, 2.f * l[2][2] - l[2][1]);
    } else {
        sl = rminf(0.f, rminf(l[2][0], r[2][0]));
        sr = rmaxf(0.f, rmaxf(l[2][2], r[2][2]));
    }
    for (int v = 0; v < 3; ++v) {
        if (sl >= 0.f) f[v] = l[1][v];
        else if (sr <= 0.f) f[v] = r[1][v];
        else f[v] = (sr * l[1][v] - sl * r[1][v] + sl * sr * (r[0][v] - l[0][v])) / (sr - sl);
    }
}

/* One step with the split described above.  State arrays FP64, updated in place. */
int orc_forward_step_split(const da_params *p, const da_mesh_soa *m, double *h, double *hu, double *hv, double *time,
                           int64_t *iter, double *dt_out) {
    const int n = m->n_cells;
    float *S = (float *)malloc(sizeof(float) * 6 * (size_t)n);
    float *K = (float *)malloc(sizeof(float) * (size_t)n);
    float *F = (float *)calloc((size_t)12 * n, sizeof(float));
    double *U0 = (double *)malloc(sizeof(double) * 3 * (size_t)n);
    if (!S || !K || !F || !U0) {
        free(S); free(K); free(F); free(U0);
        return DA_ERR_OOM;
    }
    const double *Ud[3] = {h, hu, hv};
    /* slopes (FP32) */
    for (int i = 0; i < n; ++i) {
        int bc = 0;
        for (int s = 0; s < 4; ++s) bc |= m->nbr[(size_t)s * n + i] < 0;
        for (int d = 0; d < 2; ++d) {
            for (int j = 0; j < 3; ++j) S[(size_t)(j + 3 * d) * n + i] = 0.f;
            if (bc) continue;
            const int ep = m->nbr[(size_t)d * n + i], em = m->nbr[(size_t)(d + 2) * n + i];
            const int ep2r = m->nbr[(size_t)(d + 4) * n + i], em2r = m->nbr[(size_t)(d + 6) * n + i];
            const double *co = d == 0 ? m->x : m->y;
            const float dxp = (float)(co[ep] - co[i]), dxm = (float)(co[i] - co[em]);
            for (int j = 0; j < 3; ++j) {
                const float vi = (float)Ud[j][i];
                float dp = ((float)Ud[j][ep] - vi) / dxp;
                if (ep2r != ep) dp = .5f * (dp + ((float)Ud[j][ep2r] - vi) / dxp);
                float dm = (vi - (float)Ud[j][em]) / dxm;
                if (em2r != em) dm = .5f * (dm + (vi - (float)Ud[j][em2r]) / dxm);
                const float dc = (dp * dxm + dm * dxp) / (dxm + dxp);
                float mn = (float)p->gamma * fabsf_(dp);
                if (mn > (float)p->gamma * fabsf_(dm)) mn = (float)p->gamma * fabsf_(dm);
                if (mn > fabsf_(dc)) mn = fabsf_(dc);
                S[(size_t)(j + 3 * d) * n + i] = .5f * (c_sgnf(dp) + c_sgnf(dm)) * mn;
            }
        }
    }
    /* k act/pass and the CFL bound (FP32 per cell, FP64 reduction and dt) */
    double min_dxe = 10000000, hmax = 0;
    for (int i = 0; i < n; ++i) {
        const float hf = (float)h[i], huf = (float)hu[i], hvf = (float)hv[i];
        const float sx[3] = {S[i], S[(size_t)n + i], S[(size_t)2 * n + i]};
        const float sy[3] = {S[(size_t)3 * n + i], S[(size_t)4 * n + i], S[(size_t)5 * n + i]};
        K[i] = kact_f(p, m->material[i], hf, huf, hvf, sx, sy);
        if (h[i] > 1e-4) {
            if (hmax < h[i]) hmax = h[i];
            const float gz = (float)m->gravity[(size_t)2 * n + i];
            const float c = sqrtf(K[i] * gz * hf);
            const float ex = fabsf_(huf / hf) + c, ey = fabsf_(hvf / hf) + c;
            const double ev = (double)(ex > ey ? ex : ey);
            const double v = (m->dx[i] < m->dy[i] ? m->dx[i] : m->dy[i]) / ev;
            if (v < min_dxe) min_dxe = v;
        }
    }
    double g0 = 0.5 * min_dxe, g1 = 0.9 * sqrt(hmax * p->epsilon * p->gravity_scale / 9.8);
    double dt = 0.5 * (g0 < g1 ? g0 : g1);
    if (dt == 0.0) dt = 0.5 * p->influx_dt;
    if (*time + dt > p->next_output) dt = p->next_output - *time;
    if (*time + dt > p->next_save) dt = p->next_save - *time;
    if (*time + dt > p->max_time) dt = p->max_time - *time;
    *time += dt;
    const float ft = (*iter < p->frict_tiny_iters) ? (float)p->frict_tiny_early : (float)p->frict_tiny_late;
    *iter += 1;
    /* each cell's four side fluxes (FP32), hanging sides averaged */
    for (int i = 0; i < n; ++i) {
        float hi[3][3];
        for (int s = 0; s < 4; ++s) {
            const int d = s & 1;
            const int e1 = m->nbr[(size_t)s * n + i];
            float f[3] = {0.f, 0.f, 0.f};
            dirflux_f(d, (float)h[i], (float)hu[i], (float)hv[i], K[i], (float)m->gravity[(size_t)2 * n + i], hi);
            if (e1 >= 0) {
                const int e2 = m->nbr[(size_t)(s + 4) * n + i];
                const int ne = e2 != e1 ? 2 : 1;
                for (int q = 0; q < ne; ++q) {
                    const int e = q ? e2 : e1;
                    float he[3][3], fq[3];
                    dirflux_f(d, (float)h[e], (float)hu[e], (float)hv[e], K[e], (float)m->gravity[(size_t)2 * n + e], he);
                    if (s < 2) riemann_f(hi, he, fq); else riemann_f(he, hi, fq);
                    for (int v = 0; v < 3; ++v) f[v] += ne == 2 ? 0.5f * fq[v] : fq[v];
                }
            }
            for (int v = 0; v < 3; ++v) F[((size_t)s * 3 + v) * n + i] = f[v];
        }
        /* domain boundary: the flux of the opposite side (boundary_flux) */
        for (int d = 0; d < 2; ++d) {
            const int bp = m->nbr[(size_t)d * n + i] < 0, bm = m->nbr[(size_t)(d + 2) * n + i] < 0;
            for (int v = 0; v < 3; ++v) {
                if (bp) F[((size_t)d * 3 + v) * n + i] = F[((size_t)(d + 2) * 3 + v) * n + i];
                if (bm) F[((size_t)(d + 2) * 3 + v) * n + i] = F[((size_t)d * 3 + v) * n + i];
            }
        }
    }
    memcpy(U0, h, sizeof(double) * n);
    memcpy(U0 + n, hu, sizeof(double) * n);
    memcpy(U0 + 2 * (size_t)n, hv, sizeof(double) * n);
    const float sin_int = sinf((float)p->intfrict);
    for (int i = 0; i < n; ++i) {
        const double prev[3] = {U0[i], U0[(size_t)n + i], U0[(size_t)2 * n + i]};
        const double dtdx = dt / m->dx[i], dtdy = dt / m->dy[i];
        double st[3];
        for (int v = 0; v < 3; ++v)
            st[v] = prev[v] - dtdx * ((double)F[((size_t)0 * 3 + v) * n + i] - (double)F[((size_t)2 * 3 + v) * n + i]) -
                    dtdy * ((double)F[((size_t)1 * 3 + v) * n + i] - (double)F[((size_t)3 * 3 + v) * n + i]);
        if (st[0] < 0.) st[0] = 0;
        if (prev[0] > 1e-4) {
            const float hp = (float)prev[0], up = (float)prev[1], vp = (float)prev[2];
            const float vx = up / hp, vy = vp / hp, hinv = 1.f / hp;
            const float sx0 = S[i], sx2 = S[(size_t)2 * n + i], sy0 = S[(size_t)3 * n + i], sy1 = S[(size_t)4 * n + i];
            const float sg0 = tiny_sgnf(hinv * (sy1 - vx * sy0), ft), sg2 = tiny_sgnf(vx, ft);
            const float sg1 = tiny_sgnf(hinv * (sx2 - vy * sx0), ft), sg3 = tiny_sgnf(vy, ft);
            const float gx = (float)m->gravity[i], gy = (float)m->gravity[(size_t)n + i];
            const float gz = (float)m->gravity[(size_t)2 * n + i];
            const float dgx = (float)m->d_gravity[i], dgy = (float)m->d_gravity[(size_t)n + i];
            const float cx = (float)m->curvature[i], cy = (float)m->curvature[(size_t)n + i];
            const float tb = tanf((float)p->bedfrict[m->material[i]]);
            const float k = K[i];
            const float s1x = gx * hp;
            const float s2x = sg0 * hp * k * (gz * sy0 + dgy * hp) * sin_int;
            const float s3x = sg2 * rmaxf(gz * hp + vx * up * cx, 0.f) * tb;
            st[1] += dt * (double)(s1x - s2x - s3x);
            const float s1y = gy * hp;
            const float s2y = sg1 * hp * k * (gz * sx0 + dgx * hp) * sin_int;
            const float s3y = sg3 * rmaxf(gz * hp + vy * vp * cy, 0.f) * tb;
            st[2] += dt * (double)(s1y - s2y - s3y);
        }
        h[i] = st[0];
        hu[i] = st[1];
        hv[i] = st[2];
    }
    if (dt_out) *dt_out = dt;
    free(S); free(K); free(F); free(U0);
    return DA_OK;
}
