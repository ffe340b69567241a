// The reference's restart files, on the host: restart_<rank> written by save_forward and read by
// loadrun (src/main/restart.C:21-239), and the max-depth map outline_<rank> written beside it.
//
// A restart file is one gzip stream of native-endian records:
//   double min_dx[2], double min_gen                          the driver's mesh-size globals
//   int maxh_iter, double maxh_hmax                           MaxH_Functional (restart.C:46-49)
//   int iter, int adjiter, double time, int n, double dt[n]   TimeProps::wrtie_to_file (properties.h:494)
//   table header, int count, count x node                     the node table (HashTable::write_table,
//                                                             hashtab2.C:347; Node::write_node, node.C:356)
//   table header, int count, count x element                  the element table (Element::write_elem,
//                                                             element2.C:4493-4540)
//   table header, int last_solution_time_step                 the SolRec table (dualmesh.C:28-33)
// with the table header = unsigned MinKey[2], MaxKey[2], Range; double doublekeyrange[2],
// hashconstant, Xrange[2], Yrange[2], invdxrange, invdyrange; int NBUCKETS, PRIME, ENTRIES.
//
// Reading keeps the elements whose adapted flag is positive (the active cells of every loop of the
// reference), orders them by key (the space-filling curve) and resolves their neighbour keys
// into the flattened neighbour table: relative side r = (absolute side a - positive_x_side) mod 4,
// a domain edge where neigh_proc[a] is INIT.  An element keeps a side's two finer neighbours in
// the counter-clockwise order of its boundary (adapt/refine2.C:590-805), the table lists the
// lower (sides +-x) or left (sides +-y) one first: the pair is swapped on +y and -x, both ways.
//
// Writing builds the tables of a flattened quadtree mesh the way the reference lays them out:
// nodes on the lattice of half the finest cell -- corners 0-3 counter-clockwise from the lower
// left, edge nodes 4-7 at the middle of side k (between corners k and k+1), the bubble node at the
// centre -- so side 1 faces +x (positive_x_side = 1); node info CORNER, SIDE, BUBBLE, S_C_CON (the
// middle of a side with two finer neighbours) or S_S_CON (the edge node of a side whose neighbour
// is coarser), the stronger of the two where cells share a node; node and element keys are the
// Hilbert keys of the coordinates in the table's range (the keys da_cell_keys gives).
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "da_mesh.h"
#include "discrete_adjoint.h"

namespace {

// node info and element flags of the format (src/header/constant.h:39-48,76-84)
constexpr int kCorner = 2, kSide = 4, kSSCon = 5, kBubble = 6, kSCCon = 7;
constexpr int kInit = -1, kOneSideNeigh = -2;
constexpr int kNotRecAdapted = 1;
constexpr int kPrime = 2017;

struct Gz {
    gzFile f = nullptr;
    bool ok = true;
    ~Gz() {
        if (f) gzclose(f);
    }
    template <class T>
    void put(const T *p, size_t n) {
        if (!ok || n == 0) return;
        const size_t b = sizeof(T) * n;
        ok = gzwrite(f, p, (unsigned)b) == (int)b;
    }
    template <class T>
    void put1(T v) { put(&v, 1); }
    template <class T>
    void get(T *p, size_t n) {
        if (!ok || n == 0) return;
        const size_t b = sizeof(T) * n;
        ok = gzread(f, p, (unsigned)b) == (int)b;
    }
    template <class T>
    T get1() {
        T v{};
        get(&v, 1);
        return v;
    }
};

struct TableHeader {
    uint32_t min_key[2] = {0, 0}, max_key[2] = {0, 0}, range = 0;
    double dkr[2] = {0, 0}, hashconstant = 0, xr[2] = {0, 0}, yr[2] = {0, 0}, invdx = 0, invdy = 0;
    int32_t nbuckets = 0, prime = kPrime, entries = 0;
};

void put_header(Gz &g, const TableHeader &t) {
    g.put(t.min_key, 2);
    g.put(t.max_key, 2);
    g.put1(t.range);
    g.put(t.dkr, 2);
    g.put1(t.hashconstant);
    g.put(t.xr, 2);
    g.put(t.yr, 2);
    g.put1(t.invdx);
    g.put1(t.invdy);
    g.put1(t.nbuckets);
    g.put1(t.prime);
    g.put1(t.entries);
}

void get_header(Gz &g, TableHeader &t) {
    g.get(t.min_key, 2);
    g.get(t.max_key, 2);
    g.get(&t.range, 1);
    g.get(t.dkr, 2);
    g.get(&t.hashconstant, 1);
    g.get(t.xr, 2);
    g.get(t.yr, 2);
    g.get(&t.invdx, 1);
    g.get(&t.invdy, 1);
    g.get(&t.nbuckets, 1);
    g.get(&t.prime, 1);
    g.get(&t.entries, 1);
}

uint64_t key64(const uint32_t *k) { return (uint64_t(k[0]) << 32) | k[1]; }

// A table header over keys spanning the full 32-bit range per word, buckets ~2 per entry; the
// constant is the one HashTable's constructor derives (hashtab2.C:71), so the reference's hash
// of every key stays below 8 x NBUCKETS.
TableHeader make_header(const std::vector<uint64_t> &keys, const double xr[2], const double yr[2]) {
    TableHeader t;
    uint64_t lo = ~uint64_t(0), hi = 0;
    for (uint64_t k : keys) {
        lo = std::min(lo, k);
        hi = std::max(hi, k);
    }
    if (keys.empty()) lo = hi = 0;
    t.min_key[0] = uint32_t(lo >> 32);
    t.min_key[1] = uint32_t(lo);
    t.max_key[0] = uint32_t(hi >> 32);
    t.max_key[1] = uint32_t(hi);
    t.range = t.max_key[0] - t.min_key[0];
    t.dkr[0] = t.dkr[1] = 4294967296.0;
    t.nbuckets = int32_t(std::min<size_t>(std::max<size_t>(1024, 2 * keys.size()), 1u << 26));
    t.hashconstant = 8.0 * t.nbuckets / (t.dkr[0] * t.dkr[1] + t.dkr[1]);
    for (int q = 0; q < 2; ++q) {
        t.xr[q] = xr[q];
        t.yr[q] = yr[q];
    }
    t.invdx = 1.0 / (xr[1] - xr[0]);
    t.invdy = 1.0 / (yr[1] - yr[0]);
    t.entries = int32_t(keys.size());
    return t;
}

int node_priority(int info) {
    switch (info) {
        case kSCCon: return 4;
        case kSSCon: return 3;
        case kSide: return 2;
        case kBubble: return 1;
        default: return 0;
    }
}

}  // namespace

extern "C" {

int da_write_restart(const char *path, const da_restart_header *hd, const double *dt_hist, int32_t n_dt,
                     const da_mesh_soa *m, const int32_t *level, const int32_t *ix, const int32_t *iy,
                     const double *zeta, const double *elevation, const double *bedfrict, const double *h,
                     const double *hu, const double *hv) {
    if (!path || !hd || n_dt < 0 || (n_dt > 0 && !dt_hist) || !m || m->n_cells <= 0 || !m->nbr || !m->x ||
        !m->y || !m->dx || !m->dy || !m->gravity || !m->d_gravity || !m->curvature || !m->material || !level ||
        !ix || !iy || !h || !hu || !hv)
        return DA_ERR_INVALID;
    const int n = m->n_cells;
    int L = 0;
    for (int c = 0; c < n; ++c) {
        if (level[c] < 0 || level[c] > 29 || ix[c] < 0 || iy[c] < 0 || !(h[c] >= 0.0)) return DA_ERR_INVALID;
        L = std::max(L, level[c]);
    }
    for (size_t k = 0; k < 8 * (size_t)n; ++k)
        if (m->nbr[k] < -1 || m->nbr[k] >= n) return DA_ERR_INVALID;
    // lattice of half the finest cell; x0, y0 = the lower-left corner of the mesh
    const double fdx = m->dx[0] / double(1 << (L - level[0])), fdy = m->dy[0] / double(1 << (L - level[0]));
    const double x0 = m->x[0] - (ix[0] + 0.5) * m->dx[0], y0 = m->y[0] - (iy[0] + 0.5) * m->dy[0];
    std::unordered_map<uint64_t, int> info;   // lattice point -> node info
    std::vector<int64_t> px(9 * (size_t)n), py(9 * (size_t)n);
    int64_t maxX = 0, maxY = 0;
    auto put = [&](int64_t X, int64_t Y, int inf) {
        const uint64_t k = (uint64_t(X) << 32) | uint64_t(Y);
        auto it = info.find(k);
        if (it == info.end()) info.emplace(k, inf);
        else if (node_priority(inf) > node_priority(it->second)) it->second = inf;
        maxX = std::max(maxX, X);
        maxY = std::max(maxY, Y);
    };
    for (int c = 0; c < n; ++c) {
        const int64_t s = int64_t(1) << (L - level[c] + 1);
        const int64_t X0 = int64_t(ix[c]) * s, Y0 = int64_t(iy[c]) * s;
        const int64_t P[9][2] = {{X0, Y0}, {X0 + s, Y0}, {X0 + s, Y0 + s}, {X0, Y0 + s}, {X0 + s / 2, Y0},
                                 {X0 + s, Y0 + s / 2}, {X0 + s / 2, Y0 + s}, {X0, Y0 + s / 2}, {X0 + s / 2, Y0 + s / 2}};
        for (int q = 0; q < 9; ++q) {
            px[9 * (size_t)c + q] = P[q][0];
            py[9 * (size_t)c + q] = P[q][1];
        }
        for (int q = 0; q < 4; ++q) put(P[q][0], P[q][1], kCorner);
        put(P[8][0], P[8][1], kBubble);
        for (int a = 0; a < 4; ++a) {
            const int r = (a + 3) % 4;  // relative side of absolute side a (positive_x_side = 1)
            const int e1 = m->nbr[(size_t)r * n + c], e2 = m->nbr[(size_t)(r + 4) * n + c];
            int inf = kSide;
            if (e1 >= 0 && e2 != e1) inf = kSCCon;
            else if (e1 >= 0 && level[e1] < level[c]) inf = kSSCon;
            put(P[a + 4][0], P[a + 4][1], inf);
        }
    }
    // the table's range: a quarter lattice step beyond the outermost nodes, so no key is 0
    const double hx = 0.5 * fdx, hy = 0.5 * fdy;
    const double xr[2] = {x0 - 0.5 * hx, x0 + maxX * hx + 0.5 * hx};
    const double yr[2] = {y0 - 0.5 * hy, y0 + maxY * hy + 0.5 * hy};
    // node keys
    std::vector<uint64_t> lat;
    lat.reserve(info.size());
    for (auto &kv : info) lat.push_back(kv.first);
    std::sort(lat.begin(), lat.end());
    const size_t nn = lat.size();
    std::vector<double> nxs(nn), nys(nn);
    for (size_t k = 0; k < nn; ++k) {
        nxs[k] = x0 + double(int64_t(lat[k] >> 32)) * hx;
        nys[k] = y0 + double(int64_t(lat[k] & 0xffffffffu)) * hy;
    }
    std::vector<uint32_t> nkeys(2 * nn);
    if (da_cell_keys((int32_t)nn, nxs.data(), nys.data(), xr, yr, nkeys.data()) != DA_OK) return DA_ERR_INVALID;
    std::unordered_map<uint64_t, size_t> node_of;   // lattice point -> node index
    node_of.reserve(2 * nn);
    for (size_t k = 0; k < nn; ++k) node_of.emplace(lat[k], k);
    auto nkey = [&](int c, int q) -> const uint32_t * {
        const uint64_t p = (uint64_t(px[9 * (size_t)c + q]) << 32) | uint64_t(py[9 * (size_t)c + q]);
        return &nkeys[2 * node_of.at(p)];
    };
    // the sons of a cell's father (brothers), counter-clockwise from the lower left: their centres
    auto brother_key = [&](int c, int b, uint32_t out[2]) {
        if (level[c] == 0) {
            out[0] = out[1] = 0;
            return;
        }
        const int64_t s = int64_t(1) << (L - level[c] + 1);
        const int64_t fx = (ix[c] >> 1) * 2, fy = (iy[c] >> 1) * 2;
        static const int off[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
        const double cx = x0 + double((fx + off[b][0]) * s + s / 2) * hx;
        const double cy = y0 + double((fy + off[b][1]) * s + s / 2) * hy;
        da_cell_keys(1, &cx, &cy, xr, yr, out);
    };

    Gz g;
    g.f = gzopen(path, "wb");
    if (!g.f) return DA_ERR_IO;
    g.put(hd->min_dx, 2);
    g.put1(hd->min_gen);
    g.put1(hd->maxh_iter);
    g.put1(hd->maxh_hmax);
    g.put1(hd->iter);
    g.put1(hd->adjiter);
    g.put1(hd->time);
    g.put1(n_dt);
    g.put(dt_hist, (size_t)n_dt);
    // node table
    {
        std::vector<uint64_t> k64(nn);
        for (size_t k = 0; k < nn; ++k) k64[k] = key64(&nkeys[2 * k]);
        put_header(g, make_header(k64, xr, yr));
        g.put1(int32_t(nn));
        for (size_t k = 0; k < nn; ++k) {
            g.put1(int32_t(0));                 // id
            g.put1(int32_t(info.at(lat[k])));   // info
            g.put(&nkeys[2 * k], 2);
            const double co[2] = {nxs[k], nys[k]};
            g.put(co, 2);
            g.put1(0.0);                        // elevation (the cells carry theirs)
        }
    }
    // element table
    std::vector<uint64_t> ek(n);
    for (int c = 0; c < n; ++c) ek[c] = key64(nkey(c, 8));
    put_header(g, make_header(ek, xr, yr));
    g.put1(int32_t(n));
    const uint32_t zero2[2] = {0, 0};
    for (int c = 0; c < n; ++c) {
        const uint32_t *key = nkey(c, 8);
        g.put1(int32_t(level[c]));   // generation
        g.put(key, 2);               // lb_key
        g.put(key, 2);               // key
        int32_t nproc[8], ngen[8];
        const uint32_t *nbk[8];
        for (int a = 0; a < 4; ++a) {
            const int r = (a + 3) % 4;
            const int e1 = m->nbr[(size_t)r * n + c], e2 = m->nbr[(size_t)(r + 4) * n + c];
            if (e1 < 0) {
                nproc[a] = kInit;
                nproc[a + 4] = kOneSideNeigh;
                nbk[a] = nbk[a + 4] = zero2;
                ngen[a] = ngen[a + 4] = 0;
            } else {
                // two finer neighbours go counter-clockwise around the element: on +y and -x the
                // table's second one comes first
                const bool swap = r == 1 || r == 2;
                nproc[a] = 0;
                nproc[a + 4] = e2 != e1 ? 0 : kOneSideNeigh;
                nbk[a] = nkey(swap ? e2 : e1, 8);
                nbk[a + 4] = nkey(swap ? e1 : e2, 8);
                ngen[a] = ngen[a + 4] = level[e1];
            }
        }
        for (int q = 0; q < 8; ++q) {
            g.put(nkey(c, q), 2);
            g.put(nbk[q], 2);
        }
        for (int b = 0; b < 4; ++b) {
            uint32_t bk[2];
            brother_key(c, b, bk);
            g.put(zero2, 2);  // son: a leaf has none
            g.put(bk, 2);
        }
        g.put(nproc, 8);
        g.put(ngen, 8);
        g.put1(int32_t(0));              // refined
        g.put1(int32_t(kNotRecAdapted)); // adapted
        g.put1(int32_t(1));              // new_old
        const double co[2] = {m->x[c], m->y[c]};
        g.put(co, 2);
        const int32_t loc[2] = {ix[c], iy[c]};
        g.put(loc, 2);
        const double st[3] = {h[c], hu[c], hv[c]};
        g.put(st, 3);                    // state_vars
        g.put(st, 3);                    // prev_state_vars
        const double zt[2] = {zeta ? zeta[c] : 0.0, zeta ? zeta[(size_t)n + c] : 0.0};
        g.put(zt, 2);
        const double bf = bedfrict ? bedfrict[m->material[c]] : 0.0;
        g.put1(bf);                      // effect_bedfrict
        g.put1(std::tan(bf));            // effect_tanbedfrict
        const int32_t which_son = level[c] == 0 ? 0 : ((ix[c] & 1) ? ((iy[c] & 1) ? 2 : 1) : ((iy[c] & 1) ? 3 : 0));
        g.put1(which_son);
        g.put1(int32_t(1));              // positive_x_side
        const double d[2] = {m->dx[c], m->dy[c]};
        g.put(d, 2);
        const double cv[2] = {m->curvature[c], m->curvature[(size_t)n + c]};
        g.put(cv, 2);
        g.put1(elevation ? elevation[c] : 0.0);
        const double gr[3] = {m->gravity[c], m->gravity[(size_t)n + c], m->gravity[2 * (size_t)n + c]};
        g.put(gr, 3);
        const double dg[2] = {m->d_gravity[c], m->d_gravity[(size_t)n + c]};
        g.put(dg, 2);
        g.put1(int32_t(0));              // opposite_brother_flag
        g.put1(0.0);                     // shortspeed
        g.put1(int32_t(m->material[c] + 1));
        g.put1(int32_t(0));              // stoppedflags
        g.put1(1.0);                     // Awet
        g.put1(1.0);                     // Swet
        g.put1(int32_t(8));              // iwetnode
        g.put1(1.0);                     // lb_weight
        g.put1(int32_t(c));              // ithelem
    }
    // SolRec table: the element keys' range, no records kept in the file
    put_header(g, make_header(ek, xr, yr));
    g.put1(hd->solrec_last_step);
    if (!g.ok) return DA_ERR_IO;
    return gzclose(std::exchange(g.f, nullptr)) == Z_OK ? DA_OK : DA_ERR_IO;
}

int da_read_restart(const char *path, da_restart_header *hd, int32_t *n_cells, int32_t *n_dt, double *dt_hist,
                    const da_restart_cells *out) {
    if (!path || !hd || !n_cells || !n_dt) return DA_ERR_INVALID;
    const int32_t cap_cells = *n_cells, cap_dt = *n_dt;
    Gz g;
    g.f = gzopen(path, "rb");
    if (!g.f) return DA_ERR_IO;
    std::memset(hd, 0, sizeof(*hd));
    g.get(hd->min_dx, 2);
    g.get(&hd->min_gen, 1);
    g.get(&hd->maxh_iter, 1);
    g.get(&hd->maxh_hmax, 1);
    g.get(&hd->iter, 1);
    g.get(&hd->adjiter, 1);
    g.get(&hd->time, 1);
    const int32_t ndt = g.get1<int32_t>();
    if (!g.ok || ndt < 0) return DA_ERR_IO;
    std::vector<double> dts((size_t)ndt);
    g.get(dts.data(), dts.size());
    TableHeader th;
    get_header(g, th);
    const int32_t nnodes = g.get1<int32_t>();
    if (!g.ok || nnodes < 0) return DA_ERR_IO;
    for (int32_t k = 0; k < nnodes && g.ok; ++k) {  // id, info, key[2], coord[2], elevation
        char rec[4 + 4 + 8 + 16 + 8];
        g.get(rec, sizeof(rec));
    }
    get_header(g, th);
    hd->xrange[0] = th.xr[0];
    hd->xrange[1] = th.xr[1];
    hd->yrange[0] = th.yr[0];
    hd->yrange[1] = th.yr[1];
    const int32_t nel = g.get1<int32_t>();
    if (!g.ok || nel < 0) return DA_ERR_IO;
    struct El {
        int32_t gen, mat, xp, adapted, nproc[8], loc[2];
        uint32_t key[2], nbk[8][2];
        double coord[2], st[3], zeta[2], dx[2], curv[2], elev, grav[3], dgrav[2];
    };
    std::vector<El> els;
    els.reserve((size_t)nel);
    for (int32_t k = 0; k < nel && g.ok; ++k) {
        El e{};
        uint32_t skip2[2];
        int32_t i1, ngen[8];
        double d1, prev[3];
        e.gen = g.get1<int32_t>();
        g.get(skip2, 2);                 // lb_key
        g.get(e.key, 2);
        for (int q = 0; q < 8; ++q) {
            g.get(skip2, 2);             // node key
            g.get(e.nbk[q], 2);
        }
        for (int q = 0; q < 8; ++q) g.get(skip2, 2);  // sons and brothers
        g.get(e.nproc, 8);
        g.get(ngen, 8);
        g.get(&i1, 1);                   // refined
        e.adapted = g.get1<int32_t>();
        g.get(&i1, 1);                   // new_old
        g.get(e.coord, 2);
        g.get(e.loc, 2);
        g.get(e.st, 3);
        g.get(prev, 3);
        g.get(e.zeta, 2);
        g.get(&d1, 1);                   // effect_bedfrict
        g.get(&d1, 1);                   // effect_tanbedfrict
        g.get(&i1, 1);                   // which_son
        e.xp = g.get1<int32_t>();
        g.get(e.dx, 2);
        g.get(e.curv, 2);
        g.get(&e.elev, 1);
        g.get(e.grav, 3);
        g.get(e.dgrav, 2);
        g.get(&i1, 1);                   // opposite_brother_flag
        g.get(&d1, 1);                   // shortspeed
        e.mat = g.get1<int32_t>();
        g.get(&i1, 1);                   // stoppedflags
        g.get(&d1, 1);                   // Awet
        g.get(&d1, 1);                   // Swet
        g.get(&i1, 1);                   // iwetnode
        g.get(&d1, 1);                   // lb_weight
        g.get(&i1, 1);                   // ithelem
        if (e.adapted > 0) els.push_back(e);
    }
    get_header(g, th);
    hd->solrec_last_step = g.get1<int32_t>();
    if (!g.ok) return DA_ERR_IO;
    std::sort(els.begin(), els.end(), [](const El &a, const El &b) { return key64(a.key) < key64(b.key); });
    const int32_t n = (int32_t)els.size();
    *n_cells = n;
    *n_dt = ndt;
    hd->n_nodes = nnodes;
    hd->n_elements = nel;
    if (dt_hist && cap_dt >= ndt) std::copy(dts.begin(), dts.end(), dt_hist);
    if (!out) return DA_OK;
    if (cap_cells < n || (dt_hist && cap_dt < ndt)) return DA_ERR_INVALID;
    std::unordered_map<uint64_t, int32_t> index;
    index.reserve(2 * (size_t)n);
    for (int32_t i = 0; i < n; ++i) index.emplace(key64(els[i].key), i);
    int32_t unresolved = 0;
    for (int32_t i = 0; i < n; ++i) {
        const El &e = els[i];
        if (out->keys) {
            out->keys[2 * (size_t)i] = e.key[0];
            out->keys[2 * (size_t)i + 1] = e.key[1];
        }
        if (out->nbr) {
            for (int r = 0; r < 4; ++r) {
                const int a = (e.xp + r) % 4;
                int32_t i1 = -1, i2 = -1;
                if (e.nproc[a] != kInit) {
                    auto it = index.find(key64(e.nbk[a]));
                    if (it != index.end()) i1 = it->second;
                    auto it2 = index.find(key64(e.nbk[a + 4]));
                    i2 = (e.nproc[a + 4] == kOneSideNeigh) ? i1 : (it2 != index.end() ? it2->second : -1);
                    if (i1 < 0 || i2 < 0) {  // a neighbour outside the file (another rank's)
                        ++unresolved;
                        i1 = i2 = -1;
                    }
                }
                const bool swap = r == 1 || r == 2;   // counter-clockwise pair -> lower / left first
                out->nbr[(size_t)r * n + i] = swap ? i2 : i1;
                out->nbr[(size_t)(r + 4) * n + i] = swap ? i1 : i2;
            }
        }
        if (out->level) out->level[i] = e.gen;
        if (out->material) out->material[i] = e.mat - 1;
        if (out->x) out->x[i] = e.coord[0];
        if (out->y) out->y[i] = e.coord[1];
        if (out->dx) out->dx[i] = e.dx[0];
        if (out->dy) out->dy[i] = e.dx[1];
        if (out->elevation) out->elevation[i] = e.elev;
        for (int q = 0; q < 2; ++q) {
            if (out->zeta) out->zeta[(size_t)q * n + i] = e.zeta[q];
            if (out->curvature) out->curvature[(size_t)q * n + i] = e.curv[q];
            if (out->d_gravity) out->d_gravity[(size_t)q * n + i] = e.dgrav[q];
        }
        for (int q = 0; q < 3; ++q)
            if (out->gravity) out->gravity[(size_t)q * n + i] = e.grav[q];
        if (out->h) out->h[i] = e.st[0];
        if (out->hu) out->hu[i] = e.st[1];
        if (out->hv) out->hv[i] = e.st[2];
    }
    hd->n_unresolved = unresolved;
    return DA_OK;
}

int da_write_outline(const char *path, const double dxy[2], const double xrange[2], const double yrange[2],
                     int32_t nx, int32_t ny, const double *map) {
    if (!path || !dxy || !xrange || !yrange || nx <= 0 || ny <= 0 || !map) return DA_ERR_INVALID;
    Gz g;
    g.f = gzopen(path, "wb");
    if (!g.f) return DA_ERR_IO;
    g.put(dxy, 2);
    g.put(xrange, 2);
    g.put(yrange, 2);
    g.put(map, (size_t)nx * ny);
    if (!g.ok) return DA_ERR_IO;
    return gzclose(std::exchange(g.f, nullptr)) == Z_OK ? DA_OK : DA_ERR_IO;
}

}  // extern "C"
