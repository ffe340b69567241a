// Rebuilding the reference's tables from a flattened mesh (see harness_tables.h).
// TEST INFRASTRUCTURE ONLY.
#include <sys/sysinfo.h>
#include <sys/types.h>
#include <unistd.h>
#include <zlib.h>

// every standard header the reference's headers pull in comes before the access override below
#include <algorithm>
#include <array>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include <hdf5.h>
#include <mpi.h>

// the harness sets Element/Node fields directly instead of replaying the preprocessor
#define private public
#define protected public
#include "hpfem.h"
#undef private
#undef protected

#include "harness_tables.h"

namespace harness {
namespace {

struct NodeRec {
    double x, y;
    int info;
};

int priority(int info) {
    switch (info) {
        case S_C_CON: return 4;
        case S_S_CON: return 3;
        case SIDE: return 2;
        case BUBBLE: return 1;
        default: return 0;  // CORNER
    }
}

}  // namespace

// ---- the flattened mesh every table-building mode reads (see the file comment)

void read_mesh(FILE *f, const int32_t hdr[6], MeshIn &m) {
    m.n = hdr[1];
    m.L = hdr[2];
    m.nmat = hdr[3];
    m.nsteps = hdr[4];
    m.flag = hdr[5];
    const size_t n = (size_t)m.n;
    rd(f, m.sc, 5);
    rd(f, m.bed, 16);
    m.nbr.resize(8 * n);
    m.level.resize(n);
    m.ix.resize(n);
    m.iy.resize(n);
    m.mat.resize(n);
    rd(f, m.nbr.data(), m.nbr.size());
    rd(f, m.level.data(), n);
    rd(f, m.ix.data(), n);
    rd(f, m.iy.data(), n);
    rd(f, m.mat.data(), n);
    m.x.resize(n); m.y.resize(n); m.dx.resize(n); m.dy.resize(n);
    m.zeta.resize(2 * n); m.grav.resize(3 * n); m.dgrav.resize(2 * n); m.curv.resize(2 * n);
    rd(f, m.x.data(), n); rd(f, m.y.data(), n); rd(f, m.dx.data(), n); rd(f, m.dy.data(), n);
    rd(f, m.zeta.data(), m.zeta.size()); rd(f, m.grav.data(), m.grav.size()); rd(f, m.dgrav.data(), m.dgrav.size());
    rd(f, m.curv.data(), m.curv.size());
}


void make_props(const MeshIn &m, Props &pr) {
    static char nm[] = "m";
    pr.bedin.assign(m.nmat + 1, 0.0);
    pr.names.assign(m.nmat + 1, nullptr);
    for (int k = 1; k <= m.nmat; ++k) {
        pr.bedin[k] = m.bed[k - 1];
        pr.names[k] = nm;
    }
    const double *sc = m.sc;
    pr.matprops = new MatProps(m.nmat, pr.names.data(), sc[0], pr.bedin.data(), 0.0, 0.0, sc[1], sc[3], 0.1, 1.0,
                               sc[1], sc[2]);
    MatProps &mp = *pr.matprops;
    mp.epsilon = sc[1];
    mp.GRAVITY_SCALE = sc[2];
    mp.LENGTH_SCALE = 1.0;
    mp.HEIGHT_SCALE = sc[1];
    mp.gamma = sc[3];
    mp.MAX_NEGLIGIBLE_HEIGHT = mp.HEIGHT_SCALE / 10000.0;  // datread.C:210
}

// Nodes at integer positions (units of half the finest cell), node info as constant.h:39-43
// defines it, elements with positive_x_side = 1.

// The hash table's bucket index spreads the element keys as the element table's does.
SolRec *solrec_for(const Tables &t, int n) {
    double dkr[2] = {t.dkr[0], t.dkr[1]}, XR[2] = {t.XR[0], t.XR[1]}, YR[2] = {t.YR[0], t.YR[1]};
    return new SolRec(dkr, std::max(1024, 2 * n), 2017, XR, YR, 0);
}

Tables build_tables(const MeshIn &m, const double *h, const double *hu, const double *hv, MatProps &matprops,
                    bool ref_static) {
    const int n = m.n, L = m.L;
    const int32_t *nbr = m.nbr.data();
    const auto &level = m.level;
    const auto &x = m.x, &y = m.y, &dx = m.dx, &dy = m.dy;
    double fine_dx = 0, fine_dy = 0, x0 = 0, y0 = 0;
    {
        const int sh = L - level[0];
        fine_dx = dx[0] / double(1 << sh);
        fine_dy = dy[0] / double(1 << sh);
        x0 = x[0] - (m.ix[0] + 0.5) * dx[0];
        y0 = y[0] - (m.iy[0] + 0.5) * dy[0];
    }
    std::map<std::pair<int64_t, int64_t>, NodeRec> nodes;
    std::vector<std::array<std::pair<int64_t, int64_t>, 9>> cell_nodes(n);
    auto put = [&](int64_t X, int64_t Y, int info) {
        auto key = std::make_pair(X, Y);
        auto it = nodes.find(key);
        if (it == nodes.end())
            nodes[key] = NodeRec{x0 + X * 0.5 * fine_dx, y0 + Y * 0.5 * fine_dy, info};
        else if (priority(info) > priority(it->second.info))
            it->second.info = info;
    };
    for (int c = 0; c < n; ++c) {
        const int64_t s = int64_t(1) << (L - level[c] + 1);
        const int64_t X0 = m.ix[c] * s, Y0 = m.iy[c] * s;
        const int64_t P[9][2] = {{X0, Y0}, {X0 + s, Y0}, {X0 + s, Y0 + s}, {X0, Y0 + s},
                                 {X0 + s / 2, Y0}, {X0 + s, Y0 + s / 2}, {X0 + s / 2, Y0 + s}, {X0, Y0 + s / 2},
                                 {X0 + s / 2, Y0 + s / 2}};
        for (int q = 0; q < 9; ++q) cell_nodes[c][q] = std::make_pair(P[q][0], P[q][1]);
        for (int q = 0; q < 4; ++q) put(P[q][0], P[q][1], CORNER);
        put(P[8][0], P[8][1], BUBBLE);
        for (int a = 0; a < 4; ++a) {  // absolute side a has edge node a + 4
            const int r = (a + 3) % 4;  // relative side (0=+x,1=+y,2=-x,3=-y) with positive_x_side = 1
            const int e1 = nbr[(size_t)r * n + c], e2 = nbr[(size_t)(r + 4) * n + c];
            int info = SIDE;
            if (e1 >= 0 && e2 != e1) info = S_C_CON;
            else if (e1 >= 0 && level[e1] < level[c]) info = S_S_CON;
            put(P[a + 4][0], P[a + 4][1], info);
        }
    }
    int64_t maxX = 0, maxY = 0;
    for (auto &kv : nodes) {
        maxX = std::max(maxX, kv.first.first);
        maxY = std::max(maxY, kv.first.second);
    }
    double dkr[2] = {double(maxX + 2), double(maxY + 2)};
    double XR[2] = {x0, x0 + (maxX + 1) * 0.5 * fine_dx}, YR[2] = {y0, y0 + (maxY + 1) * 0.5 * fine_dy};
    const int nb = std::max(1024, 2 * (int)nodes.size());
    Tables t;
    for (int q = 0; q < 2; ++q) {
        t.dkr[q] = dkr[q];
        t.XR[q] = XR[q];
        t.YR[q] = YR[q];
    }
    t.NodeTable = new HashTable(dkr, nb, 2017, XR, YR, 0);
    t.El_Table = new HashTable(dkr, std::max(1024, 2 * n), 2017, XR, YR, 0);
    auto keyof = [](const std::pair<int64_t, int64_t> &p, unsigned k[2]) {
        k[0] = unsigned(p.first + 1);  // +1 keeps {0,0} free: it is the boundary's "NULL" neighbour key
        k[1] = unsigned(p.second + 1);
    };
    for (auto &kv : nodes) {
        unsigned k[2];
        keyof(kv.first, k);
        double co[2] = {kv.second.x, kv.second.y};
        Node *nd = new Node(k, co, kv.second.info, 0.0, 0);
        t.NodeTable->add(k, nd);
    }
    t.els.resize(n);
    const double eps = m.sc[1];
    for (int c = 0; c < n; ++c) {
        Element *e = new Element();
        keyof(cell_nodes[c][8], e->key);
        for (int q = 0; q < 8; ++q) keyof(cell_nodes[c][q], e->node_key[q]);
        e->positive_x_side = 1;
        for (int a = 0; a < 4; ++a) {
            const int r = (a + 3) % 4;
            // the reference stores a side's two finer neighbours in the counter-clockwise order of
            // the element's boundary (+x: lower, upper; +y: right, left; -x: upper, lower; -y: left,
            // right -- adapt/refine2.C:590-805); the flattened table lists them lower/left first
            const bool ccw_swap = r == 1 || r == 2;
            const int f1 = nbr[(size_t)r * n + c], f2 = nbr[(size_t)(r + 4) * n + c];
            const int e1 = ccw_swap ? f2 : f1, e2 = ccw_swap ? f1 : f2;
            if (e1 < 0) {
                e->neigh_proc[a] = -1;
                e->neigh_proc[a + 4] = -2;
                e->neighbor[a][0] = e->neighbor[a][1] = 0;
                e->neighbor[a + 4][0] = e->neighbor[a + 4][1] = 0;
            } else {
                e->neigh_proc[a] = 0;
                e->neigh_proc[a + 4] = (e2 != e1) ? 0 : -2;
                keyof(cell_nodes[e1][8], e->neighbor[a]);
                keyof(cell_nodes[e2][8], e->neighbor[a + 4]);
            }
            e->neigh_gen[a] = e->neigh_gen[a + 4] = e1 >= 0 ? level[e1] : 0;
        }
        e->generation = level[c];
        e->material = m.mat[c] + 1;
        e->adapted = NOTRECADAPTED;
        e->refined = 0;
        e->myprocess = 0;
        e->coord[0] = x[c];
        e->coord[1] = y[c];
        e->dx[0] = dx[c];
        e->dx[1] = dy[c];
        e->state_vars[0] = h[c];
        e->state_vars[1] = hu[c];
        e->state_vars[2] = hv[c];
        for (int v = 0; v < 3; ++v) e->prev_state_vars[v] = e->state_vars[v];
        for (int v = 0; v < 6; ++v) e->d_state_vars[v] = 0.0;
        e->kactxy[0] = e->kactxy[1] = eps;
        e->effect_kactxy[0] = e->effect_kactxy[1] = eps;
        e->zeta[0] = m.zeta[c];
        e->zeta[1] = m.zeta[(size_t)n + c];
        e->curvature[0] = m.curv[c];
        e->curvature[1] = m.curv[(size_t)n + c];
        for (int k = 0; k < 3; ++k) e->gravity[k] = m.grav[(size_t)k * n + c];
        for (int k = 0; k < 2; ++k) e->d_gravity[k] = m.dgrav[(size_t)k * n + c];
        e->elevation = 0.0;
        for (int v = 0; v < 3; ++v) e->Influx[v] = 0.0;
        e->stoppedflags = 0;
        e->Awet = 1.0;
        e->Swet = 1.0;
        e->iwetnode = 8;
        t.El_Table->add(e->key, e);
        t.els[c] = e;
    }
    if (ref_static) {
        for (int c = 0; c < n; ++c) t.els[c]->calc_gravity_vector(&matprops);
        for (int c = 0; c < n; ++c) t.els[c]->calc_d_gravity(t.El_Table);
    }
    return t;
}


}  // namespace harness
