// Host-side mesh and input preparation: 2:1-balanced quadtree, Morton order,
// neighbour/hanging tables and the static per-cell fields of the flow model.
//
// The reference builds and adapts its mesh on the host (src/preproc, src/adapt);
// this file is the stand-in that feeds the device path.  The per-cell fields follow:
//   calc_gravity_vector  src/datstr/element2.C:3545-3564
//   calc_d_gravity       src/datstr/element2.C:3574-3653
//   calculate_slope      src/gisapi/GisApi.C:1295-1346   (Sobel / 8h on the DEM posts)
//   Get_elevation/Get_slope/Get_curvature  src/gisapi/GisApi.C:648-838 (bilinear sampling)
//   elliptical_pile_height src/main/init_piles.C:167-277 (9-node weighted paraboloid)
#include "da_mesh.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

constexpr double kTiny = 1.e-4;  // GEOFLOW_TINY, src/header/constant.h:68

inline uint64_t leaf_key(int l, int64_t i, int64_t j) {
    return (uint64_t(l) << 58) | (uint64_t(i) << 29) | uint64_t(j);
}

inline uint64_t spread_bits(uint64_t v) {  // 29-bit -> even bits
    v &= 0x1FFFFFFFull;
    v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
    v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
    v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v;
}

inline uint64_t splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct Leaf {
    int l;
    int64_t i, j;
};

// ---------------------------------------------------------------- terrain sampling
struct Terrain {
    int nrows = 0, ncols = 0;
    double xmin = 0, ymax = 0, res = 1;
    std::vector<float> elev, xslope, yslope, xcurv, ycurv;
    const int32_t *mat = nullptr;

    float &at(std::vector<float> &g, int r, int c) { return g[size_t(r) * ncols + c]; }
    float get(const std::vector<float> &g, int r, int c) const { return g[size_t(r) * ncols + c]; }

    // Sobel gradient of grid g into gx, gy (rows run north -> south, so d/dy = (north - south)).
    void sobel(const std::vector<float> &g, std::vector<float> &gx, std::vector<float> &gy) {
        gx.assign(size_t(nrows) * ncols, 0.f);
        gy.assign(size_t(nrows) * ncols, 0.f);
        const float inv = 8.f * float(res);
        for (int r = 1; r < nrows - 1; ++r)
            for (int c = 1; c < ncols - 1; ++c) {
                at(gx, r, c) = ((get(g, r - 1, c + 1) - get(g, r - 1, c - 1)) +
                                2.f * (get(g, r, c + 1) - get(g, r, c - 1)) +
                                (get(g, r + 1, c + 1) - get(g, r + 1, c - 1))) / inv;
                at(gy, r, c) = ((get(g, r - 1, c - 1) - get(g, r + 1, c - 1)) +
                                2.f * (get(g, r - 1, c) - get(g, r + 1, c)) +
                                (get(g, r - 1, c + 1) - get(g, r + 1, c + 1))) / inv;
            }
        // replicate the outermost rows/columns from their inner neighbours
        for (int c = 1; c < ncols - 1; ++c) {
            at(gx, 0, c) = get(gx, 1, c); at(gx, nrows - 1, c) = get(gx, nrows - 2, c);
            at(gy, 0, c) = get(gy, 1, c); at(gy, nrows - 1, c) = get(gy, nrows - 2, c);
        }
        for (int r = 0; r < nrows; ++r) {
            at(gx, r, 0) = get(gx, r, 1); at(gx, r, ncols - 1) = get(gx, r, ncols - 2);
            at(gy, r, 0) = get(gy, r, 1); at(gy, r, ncols - 1) = get(gy, r, ncols - 2);
        }
    }

    void prepare() {
        sobel(elev, xslope, yslope);
        std::vector<float> dummy;
        sobel(xslope, xcurv, dummy);  // d2z/dx2
        sobel(yslope, dummy, ycurv);  // d2z/dy2
    }

    double bilinear(const std::vector<float> &g, double x, double y) const {
        // x, y in post units measured from (xmin, ymax) eastwards / southwards
        if (x < 0) x = 0;
        if (y < 0) y = 0;
        if (x > ncols - 1) x = ncols - 1;
        if (y > nrows - 1) y = nrows - 1;
        int c = int(x), r = int(y);
        if (c >= ncols - 1) c = ncols - 2;
        if (r >= nrows - 1) r = nrows - 2;
        double fx = x - c, fy = y - r;
        double p1 = get(g, r, c) * (1.0 - fy) + get(g, r + 1, c) * fy;
        double p2 = get(g, r, c + 1) * (1.0 - fy) + get(g, r + 1, c + 1) * fy;
        return p1 * (1.0 - fx) + p2 * fx;
    }

    void sample(double xw, double yw, double *elev_out, double *zx, double *zy, double *kx,
                double *ky, int *material) const {
        double x = (xw - xmin) / res, y = (ymax - yw) / res;
        *elev_out = bilinear(elev, x, y);
        *zx = bilinear(xslope, x, y);
        *zy = bilinear(yslope, x, y);
        *kx = bilinear(xcurv, x, y);
        *ky = bilinear(ycurv, x, y);
        int c = int(std::floor(x + 0.5)), r = int(std::floor(y + 0.5));
        c = std::min(std::max(c, 0), ncols - 1);
        r = std::min(std::max(r, 0), nrows - 1);
        *material = mat ? mat[size_t(r) * ncols + c] : 0;
    }
};

struct MeshBuild {
    const da_mesh_spec &s;
    std::unordered_set<uint64_t> leaves;

    explicit MeshBuild(const da_mesh_spec &spec) : s(spec) {}

    int64_t nx(int l) const { return int64_t(s.nx0) << l; }
    int64_t ny(int l) const { return int64_t(s.ny0) << l; }
    double cdx(int l) const { return std::ldexp(s.dx0, -l); }
    double cdy(int l) const { return std::ldexp(s.dy0, -l); }

    bool want_refine(const Leaf &c, const da_pile_spec *piles, int n_piles) const {
        if (c.l >= s.max_level) return false;
        if (s.uniform) return true;
        const double x0 = s.xmin + c.i * cdx(c.l), x1 = x0 + cdx(c.l);
        const double y0 = s.ymin + c.j * cdy(c.l), y1 = y0 + cdy(c.l);
        for (int p = 0; p < n_piles; ++p) {
            const double r = std::max(piles[p].major, piles[p].minor) + s.refine_margin;
            const double qx = std::min(std::max(piles[p].xc, x0), x1);
            const double qy = std::min(std::max(piles[p].yc, y0), y1);
            if ((qx - piles[p].xc) * (qx - piles[p].xc) + (qy - piles[p].yc) * (qy - piles[p].yc) <= r * r)
                return true;
        }
        for (int b = 0; b < s.n_boxes; ++b) {
            const double *bx = s.boxes + 4 * b;
            if (x1 > bx[0] && x0 < bx[1] && y1 > bx[2] && y0 < bx[3]) return true;
        }
        if (s.random_frac > 0) {
            const uint64_t h = splitmix(s.seed ^ leaf_key(c.l, c.i, c.j));
            if (double(h >> 11) * (1.0 / 9007199254740992.0) < s.random_frac) return true;
        }
        return false;
    }

    void refine_leaf(const Leaf &c) {
        leaves.erase(leaf_key(c.l, c.i, c.j));
        for (int q = 0; q < 4; ++q) leaves.insert(leaf_key(c.l + 1, 2 * c.i + (q & 1), 2 * c.j + (q >> 1)));
    }

    // Level of the leaf that contains cell (l, i, j), or -1 if that region is finer.
    int containing_level(int l, int64_t i, int64_t j) const {
        for (int lp = l; lp >= 0; --lp)
            if (leaves.count(leaf_key(lp, i >> (l - lp), j >> (l - lp)))) return lp;
        return -1;
    }

    void build(const da_pile_spec *piles, int n_piles) {
        std::vector<Leaf> work;
        for (int64_t j = 0; j < s.ny0; ++j)
            for (int64_t i = 0; i < s.nx0; ++i) {
                leaves.insert(leaf_key(0, i, j));
                work.push_back({0, i, j});
            }
        while (!work.empty()) {
            Leaf c = work.back();
            work.pop_back();
            if (want_refine(c, piles, n_piles)) {
                refine_leaf(c);
                for (int q = 0; q < 4; ++q) work.push_back({c.l + 1, 2 * c.i + (q & 1), 2 * c.j + (q >> 1)});
            }
        }
        balance();
    }

    // 2:1 balance across faces: no leaf may touch a face neighbour more than one level coarser.
    void balance() {
        static const int DI[4] = {1, 0, -1, 0}, DJ[4] = {0, 1, 0, -1};
        for (;;) {
            std::unordered_set<uint64_t> marks;
            for (uint64_t k : leaves) {
                const int l = int(k >> 58);
                if (l < 2) continue;
                const int64_t i = int64_t((k >> 29) & 0x1FFFFFFFull), j = int64_t(k & 0x1FFFFFFFull);
                for (int d = 0; d < 4; ++d) {
                    const int64_t ni = i + DI[d], nj = j + DJ[d];
                    if (ni < 0 || nj < 0 || ni >= nx(l) || nj >= ny(l)) continue;
                    const int lp = containing_level(l, ni, nj);
                    if (lp >= 0 && lp < l - 1) marks.insert(leaf_key(lp, ni >> (l - lp), nj >> (l - lp)));
                }
            }
            if (marks.empty()) break;
            for (uint64_t k : marks)
                refine_leaf({int(k >> 58), int64_t((k >> 29) & 0x1FFFFFFFull), int64_t(k & 0x1FFFFFFFull)});
        }
    }
};

template <class T>
T *alloc(size_t n) {
    T *p = static_cast<T *>(std::calloc(n ? n : 1, sizeof(T)));
    if (!p) throw std::bad_alloc();
    return p;
}

}  // namespace

extern "C" int da_mesh_build(const da_mesh_spec *spec, const da_dem *dem, const da_pile_spec *piles,
                             int32_t n_piles, double length_scale, double gravity_scale,
                             da_mesh_host **out) {
    if (!spec || !out || spec->nx0 <= 0 || spec->ny0 <= 0 || spec->max_level < 0 || spec->max_level > 20 ||
        spec->dx0 <= 0 || spec->dy0 <= 0 || n_piles < 0 || n_piles > DA_MAX_PILES ||
        (n_piles > 0 && !piles) || (spec->n_boxes > 0 && !spec->boxes) || length_scale <= 0 ||
        gravity_scale <= 0)
        return DA_ERR_INVALID;
    if ((int64_t(std::max(spec->nx0, spec->ny0)) << (spec->max_level + (spec->extra_level ? 1 : 0))) >=
        (int64_t(1) << 29))
        return DA_ERR_INVALID;
    if (dem && (dem->nrows < 4 || dem->ncols < 4 || !dem->elev || dem->res <= 0)) return DA_ERR_INVALID;
    *out = nullptr;
    da_mesh_host *m = nullptr;
    try {
        MeshBuild mb(*spec);
        mb.build(piles, n_piles);
        if (spec->extra_level) {
            // every leaf once more: 2:1 balance is kept, levels go up to max_level + 1
            std::vector<uint64_t> all(mb.leaves.begin(), mb.leaves.end());
            for (uint64_t k : all)
                mb.refine_leaf({int(k >> 58), int64_t((k >> 29) & 0x1FFFFFFFull), int64_t(k & 0x1FFFFFFFull)});
        }

        // ---- Morton order of the leaves (lower-left corner at the finest level)
        const int L = spec->max_level + (spec->extra_level ? 1 : 0);
        std::vector<std::pair<uint64_t, uint64_t>> order;
        order.reserve(mb.leaves.size());
        for (uint64_t k : mb.leaves) {
            const int l = int(k >> 58);
            const uint64_t i = (k >> 29) & 0x1FFFFFFFull, j = k & 0x1FFFFFFFull;
            const uint64_t mk = spread_bits(i << (L - l)) | (spread_bits(j << (L - l)) << 1);
            order.emplace_back(mk, k);
        }
        std::sort(order.begin(), order.end());
        const int32_t n = int32_t(order.size());
        std::unordered_map<uint64_t, int32_t> index;
        index.reserve(size_t(n) * 2);
        for (int32_t c = 0; c < n; ++c) index.emplace(order[c].second, c);

        m = alloc<da_mesh_host>(1);
        m->n_cells = n;
        m->max_level = L;
        m->n_piles = n_piles;
        m->level = alloc<int32_t>(n);
        m->ix = alloc<int32_t>(n);
        m->iy = alloc<int32_t>(n);
        m->nbr = alloc<int32_t>(size_t(8) * n);
        m->x = alloc<double>(n); m->y = alloc<double>(n);
        m->dx = alloc<double>(n); m->dy = alloc<double>(n);
        m->elevation = alloc<double>(n);
        m->zeta = alloc<double>(size_t(2) * n);
        m->curvature = alloc<double>(size_t(2) * n);
        m->gravity = alloc<double>(size_t(3) * n);
        m->d_gravity = alloc<double>(size_t(2) * n);
        m->material = alloc<int32_t>(n);
        m->h0 = alloc<double>(n); m->hu0 = alloc<double>(n); m->hv0 = alloc<double>(n);
        m->dh0_dpile = alloc<double>(size_t(std::max(n_piles, 1)) * n);

        // ---- geometry and neighbour tables
        static const int DI[4] = {1, 0, -1, 0}, DJ[4] = {0, 1, 0, -1};
        for (int32_t c = 0; c < n; ++c) {
            const uint64_t k = order[c].second;
            const int l = int(k >> 58);
            const int64_t i = int64_t((k >> 29) & 0x1FFFFFFFull), j = int64_t(k & 0x1FFFFFFFull);
            m->level[c] = l;
            m->ix[c] = int32_t(i);
            m->iy[c] = int32_t(j);
            m->dx[c] = mb.cdx(l);
            m->dy[c] = mb.cdy(l);
            m->x[c] = spec->xmin + (double(i) + 0.5) * m->dx[c];
            m->y[c] = spec->ymin + (double(j) + 0.5) * m->dy[c];
            for (int s = 0; s < 4; ++s) {
                const int64_t ni = i + DI[s], nj = j + DJ[s];
                int32_t a = -1, b = -1;
                if (ni >= 0 && nj >= 0 && ni < mb.nx(l) && nj < mb.ny(l)) {
                    auto it = index.find(leaf_key(l, ni, nj));
                    if (it != index.end()) {
                        a = b = it->second;
                    } else if (l > 0 && (it = index.find(leaf_key(l - 1, ni >> 1, nj >> 1))) != index.end()) {
                        a = b = it->second;
                    } else {
                        // two finer neighbours across this side
                        int64_t ci0, cj0, ci1, cj1;
                        if (DI[s] != 0) {  // +-x side: children stacked in y
                            ci0 = ci1 = 2 * ni + (DI[s] > 0 ? 0 : 1);
                            cj0 = 2 * nj;
                            cj1 = 2 * nj + 1;
                        } else {  // +-y side: children side by side in x
                            cj0 = cj1 = 2 * nj + (DJ[s] > 0 ? 0 : 1);
                            ci0 = 2 * ni;
                            ci1 = 2 * ni + 1;
                        }
                        auto i0 = index.find(leaf_key(l + 1, ci0, cj0));
                        auto i1 = index.find(leaf_key(l + 1, ci1, cj1));
                        if (i0 == index.end() || i1 == index.end()) throw std::runtime_error("unbalanced mesh");
                        a = i0->second;
                        b = i1->second;
                    }
                }
                m->nbr[size_t(s) * n + c] = a;
                m->nbr[size_t(s + 4) * n + c] = b;
            }
        }

        // ---- terrain
        Terrain t;
        if (dem) {
            t.nrows = dem->nrows;
            t.ncols = dem->ncols;
            t.res = dem->res;
            t.xmin = dem->xmin;
            t.ymax = dem->ymin + (dem->nrows - 1) * dem->res;
            t.elev.assign(dem->elev, dem->elev + size_t(dem->nrows) * dem->ncols);
            t.mat = dem->mat;
            t.prepare();
        }
        for (int32_t c = 0; c < n; ++c) {
            double e = 0, zx = 0, zy = 0, kx = 0, ky = 0;
            int mat = 0;
            if (dem) t.sample(m->x[c], m->y[c], &e, &zx, &zy, &kx, &ky, &mat);
            m->elevation[c] = e / length_scale;
            m->zeta[c] = zx;
            m->zeta[size_t(n) + c] = zy;
            m->curvature[c] = kx * length_scale;
            m->curvature[size_t(n) + c] = ky * length_scale;
            m->material[c] = mat;
            // Element::calc_gravity_vector (element2.C:3545-3564)
            const double max_slope = std::sqrt(zx * zx + zy * zy);
            const double max_angle = std::atan(max_slope);
            const double down = 9.8 * std::sin(max_angle);
            double g0, g1, g2;
            if ((down < 0 ? -down : down) > kTiny) {
                g0 = -down * zx / max_slope;
                g1 = -down * zy / max_slope;
                g2 = 9.8 * std::cos(max_angle);
            } else {
                g0 = 0; g1 = 0; g2 = 9.8;
            }
            m->gravity[c] = g0 / gravity_scale;
            m->gravity[size_t(n) + c] = g1 / gravity_scale;
            m->gravity[size_t(2) * n + c] = g2 / gravity_scale;
        }
        // Element::calc_d_gravity (element2.C:3574-3653): weighted central difference of g_z
        // with the first neighbour on each side, one-sided at the domain edge.
        for (int32_t c = 0; c < n; ++c) {
            const double *gz = m->gravity + size_t(2) * n;
            for (int d = 0; d < 2; ++d) {
                const int32_t ep = m->nbr[size_t(d) * n + c], em = m->nbr[size_t(d + 2) * n + c];
                const double *co = d == 0 ? m->x : m->y;
                double v;
                if (ep >= 0 && em >= 0) {
                    const double dxp = co[ep] - co[c];
                    const double dp = (gz[ep] - gz[c]) / dxp;
                    const double dxm = co[c] - co[em];
                    const double dm = (gz[c] - gz[em]) / dxm;
                    v = (dp * dxm + dm * dxp) / (dxm + dxp);
                } else if (em >= 0) {
                    v = (gz[c] - gz[em]) / (co[c] - co[em]);
                } else if (ep >= 0) {
                    v = (gz[ep] - gz[c]) / (co[ep] - co[c]);
                } else {
                    v = 0;
                }
                m->d_gravity[size_t(d) * n + c] = v;
            }
        }

        // ---- initial piles: elliptical_pile_height (init_piles.C:167-277)
        std::vector<double> cosr(n_piles), sinr(n_piles);
        for (int p = 0; p < n_piles; ++p) {
            cosr[p] = std::cos(piles[p].rot_deg * M_PI / 180.0);
            sinr[p] = std::sin(piles[p].rot_deg * M_PI / 180.0);
        }
        // node order: 4 corners, 4 edge midpoints, centre; weights 1, 2, 4 (over 16)
        static const double NX[9] = {-0.5, 0.5, 0.5, -0.5, 0.0, 0.5, 0.0, -0.5, 0.0};
        static const double NY[9] = {-0.5, -0.5, 0.5, 0.5, -0.5, 0.0, 0.5, 0.0, 0.0};
        static const double W[9] = {1, 1, 1, 1, 2, 2, 2, 2, 4};
        for (int32_t c = 0; c < n; ++c) {
            double hn[9], xm[9], ym[9], dP[DA_MAX_PILES][9];
            for (int q = 0; q < 9; ++q) {
                const double ndx = m->x[c] + NX[q] * m->dx[c], ndy = m->y[c] + NY[q] * m->dy[c];
                double node_h = 0.0, sum_h = 0.0, sx = 0.0, sy = 0.0, height = 0.0;
                int arg = -1;
                for (int p = 0; p < n_piles; ++p) {
                    dP[p][q] = 0.0;
                    double major = ndx - piles[p].xc, minor = ndy - piles[p].yc;
                    const double sw = (major * cosr[p] + minor * sinr[p]) / piles[p].major;
                    minor = (-major * sinr[p] + minor * cosr[p]) / piles[p].minor;
                    major = sw;
                    height = piles[p].height * (1. - major * major - minor * minor);
                    height = (height >= 0.0) ? height : 0.0;
                    sum_h += height;
                    sx += height * piles[p].vx;
                    sy += height * piles[p].vy;
                    if (node_h < height) {
                        node_h = height;
                        arg = p;
                    }
                }
                if (sum_h <= kTiny) {
                    sx = sy = 0.0;
                } else {
                    // the reference scales by the last pile's height here (init_piles.C:243-246)
                    sx *= height / sum_h;
                    sy *= height / sum_h;
                }
                if (arg >= 0) {
                    double major = ndx - piles[arg].xc, minor = ndy - piles[arg].yc;
                    const double sw = (major * cosr[arg] + minor * sinr[arg]) / piles[arg].major;
                    minor = (-major * sinr[arg] + minor * cosr[arg]) / piles[arg].minor;
                    dP[arg][q] = 1. - sw * sw - minor * minor;
                }
                hn[q] = node_h;
                xm[q] = sx;
                ym[q] = sy;
            }
            m->h0[c] = (hn[0] + hn[1] + hn[2] + hn[3] + 2.0 * (hn[4] + hn[5] + hn[6] + hn[7]) + 4.0 * hn[8]) / 16.0;
            m->hu0[c] = (xm[0] + xm[1] + xm[2] + xm[3] + 2.0 * (xm[4] + xm[5] + xm[6] + xm[7]) + 4.0 * xm[8]) / 16.0;
            m->hv0[c] = (ym[0] + ym[1] + ym[2] + ym[3] + 2.0 * (ym[4] + ym[5] + ym[6] + ym[7]) + 4.0 * ym[8]) / 16.0;
            for (int p = 0; p < n_piles; ++p) {
                double acc = 0.0;
                for (int q = 0; q < 9; ++q) acc += W[q] * dP[p][q];
                m->dh0_dpile[size_t(p) * n + c] = acc / 16.0;
            }
        }
        *out = m;
        return DA_OK;
    } catch (const std::bad_alloc &) {
        da_mesh_free(m);
        return DA_ERR_OOM;
    } catch (...) {
        da_mesh_free(m);
        return DA_ERR_INVALID;
    }
}

extern "C" void da_mesh_free(da_mesh_host *m) {
    if (!m) return;
    std::free(m->level); std::free(m->ix); std::free(m->iy); std::free(m->nbr);
    std::free(m->x); std::free(m->y); std::free(m->dx); std::free(m->dy);
    std::free(m->elevation); std::free(m->zeta); std::free(m->curvature);
    std::free(m->gravity); std::free(m->d_gravity); std::free(m->material);
    std::free(m->h0); std::free(m->hu0); std::free(m->hv0); std::free(m->dh0_dpile);
    std::free(m);
}

extern "C" int da_mesh_view(const da_mesh_host *m, da_mesh_soa *v) {
    if (!m || !v) return DA_ERR_INVALID;
    v->n_cells = m->n_cells;
    v->nbr = m->nbr;
    v->x = m->x; v->y = m->y;
    v->dx = m->dx; v->dy = m->dy;
    v->gravity = m->gravity;
    v->d_gravity = m->d_gravity;
    v->curvature = m->curvature;
    v->material = m->material;
    return DA_OK;
}
