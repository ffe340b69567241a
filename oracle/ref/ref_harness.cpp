// Oracle harness: runs the reference's own compiled step() on a flattened mesh.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/ref_build.py into oracle/_ref/ref_harness from
// the reference's sources where they lie (plus the single-rank MPI/HDF5 stand-ins and the C
// restatements of the three Fortran kernels in this directory).  It never ships in the
// product library.
//
// It reads a flattened mesh + state (format below), rebuilds the reference's Node and
// Element hash tables from it (node keys from integer node positions, info SIDE / S_C_CON /
// S_S_CON / CORNER / BUBBLE as src/header/constant.h:39-43 defines them), then calls
//     step(El_Table, NodeTable, 0, 1, &matprops, &timeprops, &pileprops, &fluxprops,
//          &statprops, &order_flag, &outline, &discharge, 0)            src/geoflow/step.C:29
// nsteps times with matprops.frict_tiny set as the driver does (src/main/hpfem.C:232-235),
// and writes the state, the dt history and the per-element fields of the last step.
//
// Input (little endian):  int32 magic 'DAH1', n, max_level, n_materials, nsteps, ref_static
//   double intfrict, epsilon, gravity_scale, gamma, maxtime, bedfrict[16]
//   int32 nbr[8n] level[n] ix[n] iy[n] material[n]
//   double x[n] y[n] dx[n] dy[n] zeta[2n] gravity[3n] d_gravity[2n] curvature[2n] h[n] hu[n] hv[n]
// Output: int32 magic 'DAO1', n, nsteps; double dt[nsteps], time;
//   double h[n] hu[n] hv[n] slopes[6n] kact[n] flux[4][3][n] gravity[3n] d_gravity[2n]
// ref_static = 1 recomputes gravity with Element::calc_gravity_vector and d_gravity with
// Element::calc_d_gravity instead of taking the input's.
//
// Other modes, chosen by the first word of the input:
//   'DAK1' n, double u[n], v[n]  ->  'DAK2' n, uint32 key[2n]: fhsfc2d_ (src/main/hilbert.C) of
//       each normalised point, the element key of Element::gen_my_sons_key.
//   'DAW1' rank, step, n, uint32 key[2n], double h[n], hu[n], hv[n]  ->  'DAW2': the reference's
//       SolRec writes the file solution_<rank>_<step> in the working directory
//       (record_solution's zero / non-zero split, wrtie_sol_to_disk).
//   'DAR1' rank, step, n, uint32 key[2n]  ->  'DAR2' n, int32 found[n] (0 none, 1 zero record,
//       2 state record), double state[3n]: the reference's SolRec reads solution_<rank>_<step>
//       (read_sol_from_disk) and each key is looked up.
#include <sys/sysinfo.h>
#include <sys/types.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cassert>
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

int REFINE_LEVEL = 0;  // global of the reference's driver (hpfem.C)

void step(HashTable *El_Table, HashTable *NodeTable, int myid, int nump, MatProps *matprops_ptr,
          TimeProps *timeprops_ptr, PileProps *pileprops_ptr, FluxProps *fluxprops, StatProps *statprops_ptr,
          int *order_flag, OutLine *outline_ptr, DISCHARGE *discharge, int adaptflag);

namespace {

template <class T>
void rd(FILE *f, T *p, size_t n) {
    if (std::fread(p, sizeof(T), n, f) != n) {
        std::fprintf(stderr, "ref_harness: short read\n");
        std::exit(2);
    }
}
template <class T>
void wr(FILE *f, const T *p, size_t n) {
    std::fwrite(p, sizeof(T), n, f);
}

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

namespace {

SolRec *make_solrec() {
    double dkr[2] = {4294967296.0, 4294967296.0}, XR[2] = {0.0, 1.0}, YR[2] = {0.0, 1.0};
    return new SolRec(dkr, 4099, 2017, XR, YR, 0);
}

int keys_mode(FILE *f, const char *out) {
    int32_t n;
    rd(f, &n, 1);
    std::vector<double> u(n), v(n);
    rd(f, u.data(), n);
    rd(f, v.data(), n);
    std::vector<unsigned> k(2 * (size_t)n);
    for (int32_t i = 0; i < n; ++i) {
        double c[2] = {u[i], v[i]};
        unsigned nkey = 2;
        fhsfc2d_(c, &nkey, &k[2 * (size_t)i]);
    }
    FILE *o = std::fopen(out, "wb");
    const int32_t m = 0x324B4144;
    wr(o, &m, 1);
    wr(o, &n, 1);
    wr(o, k.data(), k.size());
    std::fclose(o);
    return 0;
}

int write_mode(FILE *f, const char *out) {
    int32_t h3[3];
    rd(f, h3, 3);
    const int rank = h3[0], stp = h3[1], n = h3[2];
    std::vector<unsigned> k(2 * (size_t)n);
    std::vector<double> h(n), hu(n), hv(n);
    rd(f, k.data(), k.size());
    rd(f, h.data(), n);
    rd(f, hu.data(), n);
    rd(f, hv.data(), n);
    SolRec *sr = make_solrec();
    for (int32_t i = 0; i < n; ++i) {
        Jacobian *j = new Jacobian(&k[2 * (size_t)i]);
        sr->add(j->get_key(), j);
        if (h[i] > 0.) {
            double s[3] = {h[i], hu[i], hv[i]};
            j->put_solution(new Solution(s), stp);
        } else {
            j->put_solution(&(Solution::solution_zero), stp);
        }
    }
    sr->update_first_sol_time(stp);
    sr->update_last_sol_time(stp + 1);
    sr->wrtie_sol_to_disk(rank);
    FILE *o = std::fopen(out, "wb");
    const int32_t m = 0x32574144;
    wr(o, &m, 1);
    std::fclose(o);
    return 0;
}

int read_mode(FILE *f, const char *out) {
    int32_t h3[3];
    rd(f, h3, 3);
    const int rank = h3[0], stp = h3[1], n = h3[2];
    std::vector<unsigned> k(2 * (size_t)n);
    rd(f, k.data(), k.size());
    SolRec *sr = make_solrec();
    sr->read_sol_from_disk(rank, stp);
    std::vector<int32_t> found(n, 0);
    std::vector<double> st(3 * (size_t)n, 0.0);
    for (int32_t i = 0; i < n; ++i) {
        Jacobian *j = (Jacobian *)sr->lookup(&k[2 * (size_t)i]);
        Solution *s = j ? j->get_solution(stp) : nullptr;
        if (!s) continue;
        found[i] = s == &(Solution::solution_zero) ? 1 : 2;
        for (int v = 0; v < 3; ++v) st[3 * (size_t)i + v] = s->get_solution()[v];
    }
    FILE *o = std::fopen(out, "wb");
    const int32_t m = 0x32524144;
    wr(o, &m, 1);
    wr(o, &n, 1);
    wr(o, found.data(), n);
    wr(o, st.data(), st.size());
    std::fclose(o);
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: ref_harness in.bin out.bin\n");
        return 2;
    }
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t magic;
    rd(f, &magic, 1);
    if (magic == 0x314B4144) return keys_mode(f, argv[2]);
    if (magic == 0x31574144) return write_mode(f, argv[2]);
    if (magic == 0x31524144) return read_mode(f, argv[2]);
    int32_t hdr[6];
    hdr[0] = magic;
    rd(f, hdr + 1, 5);
    if (hdr[0] != 0x31484144) return 3;
    const int n = hdr[1], L = hdr[2], nmat = hdr[3], nsteps = hdr[4], ref_static = hdr[5];
    double sc[5], bed[16];
    rd(f, sc, 5);
    rd(f, bed, 16);
    std::vector<int32_t> nbr(8 * (size_t)n), level(n), ix(n), iy(n), mat(n);
    rd(f, nbr.data(), nbr.size());
    rd(f, level.data(), n);
    rd(f, ix.data(), n);
    rd(f, iy.data(), n);
    rd(f, mat.data(), n);
    std::vector<double> x(n), y(n), dx(n), dy(n), zeta(2 * (size_t)n), grav(3 * (size_t)n), dgrav(2 * (size_t)n),
        curv(2 * (size_t)n), h(n), hu(n), hv(n);
    rd(f, x.data(), n); rd(f, y.data(), n); rd(f, dx.data(), n); rd(f, dy.data(), n);
    rd(f, zeta.data(), zeta.size()); rd(f, grav.data(), grav.size()); rd(f, dgrav.data(), dgrav.size());
    rd(f, curv.data(), curv.size());
    rd(f, h.data(), n); rd(f, hu.data(), n); rd(f, hv.data(), n);
    // statistics inputs (StatProps, properties.h:180-200; DISCHARGE planes): test point height and
    // position, Vslump, then the discharge planes (xa, xb, ya, yb each)
    double stat_in[4];
    rd(f, stat_in, 4);
    int32_t n_planes = 0;
    rd(f, &n_planes, 1);
    std::vector<double> plane_in(4 * (size_t)n_planes);
    if (n_planes > 0) rd(f, plane_in.data(), plane_in.size());
    std::fclose(f);

    // ---- MatProps (properties.h:527-640): material ids are 1-based in the reference
    std::vector<double> bedin(nmat + 1, 0.0);
    std::vector<char *> names(nmat + 1, nullptr);
    static char nm[] = "m";
    for (int m = 1; m <= nmat; ++m) {
        bedin[m] = bed[m - 1];
        names[m] = nm;
    }
    MatProps matprops(nmat, names.data(), sc[0], bedin.data(), 0.0, 0.0, sc[1], sc[3], 0.1, 1.0, sc[1], sc[2]);
    matprops.epsilon = sc[1];
    matprops.GRAVITY_SCALE = sc[2];
    matprops.LENGTH_SCALE = 1.0;
    matprops.HEIGHT_SCALE = sc[1];
    matprops.gamma = sc[3];
    matprops.MAX_NEGLIGIBLE_HEIGHT = matprops.HEIGHT_SCALE / 10000.0;  // datread.C:210
    matprops.Vslump = stat_in[3];
    TimeProps timeprops;
    timeprops.inittime(1 << 30, sc[4], HUGE_VAL, HUGE_VAL, 1.0);
    PileProps pileprops;
    FluxProps fluxprops;
    StatProps statprops;
    statprops.hxyminmax = matprops.MAX_NEGLIGIBLE_HEIGHT * 10.0;  // datread.C:315-316
    statprops.heightifreach = stat_in[0];
    statprops.xyifreach[0] = stat_in[1];
    statprops.xyifreach[1] = stat_in[2];
    statprops.timereached = -1.0;
    DISCHARGE discharge;
    std::vector<double *> plane_rows(n_planes);
    for (int k = 0; k < n_planes; ++k) plane_rows[k] = &plane_in[4 * (size_t)k];
    if (n_planes > 0) discharge.init(n_planes, plane_rows.data());
    OutLine outline;

    // ---- nodes at integer positions (units of half the finest cell)
    double fine_dx = 0, fine_dy = 0, x0 = 0, y0 = 0;
    {
        const int sh = L - level[0];
        fine_dx = dx[0] / double(1 << sh);
        fine_dy = dy[0] / double(1 << sh);
        x0 = x[0] - (ix[0] + 0.5) * dx[0];
        y0 = y[0] - (iy[0] + 0.5) * dy[0];
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
        const int64_t X0 = ix[c] * s, Y0 = iy[c] * s;
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
    HashTable *NodeTable = new HashTable(dkr, nb, 2017, XR, YR, 0);
    HashTable *El_Table = new HashTable(dkr, std::max(1024, 2 * n), 2017, XR, YR, 0);
    auto keyof = [](const std::pair<int64_t, int64_t> &p, unsigned k[2]) {
        k[0] = unsigned(p.first + 1);  // +1 keeps {0,0} free: it is the boundary's "NULL" neighbour key
        k[1] = unsigned(p.second + 1);
    };
    for (auto &kv : nodes) {
        unsigned k[2];
        keyof(kv.first, k);
        double co[2] = {kv.second.x, kv.second.y};
        Node *nd = new Node(k, co, kv.second.info, 0.0, 0);
        NodeTable->add(k, nd);
    }
    std::vector<Element *> els(n);
    for (int c = 0; c < n; ++c) {
        Element *e = new Element();
        keyof(cell_nodes[c][8], e->key);
        for (int q = 0; q < 8; ++q) keyof(cell_nodes[c][q], e->node_key[q]);
        e->positive_x_side = 1;
        for (int a = 0; a < 4; ++a) {
            const int r = (a + 3) % 4;
            const int e1 = nbr[(size_t)r * n + c], e2 = nbr[(size_t)(r + 4) * n + c];
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
        e->material = mat[c] + 1;
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
        e->kactxy[0] = e->kactxy[1] = sc[1];
        e->effect_kactxy[0] = e->effect_kactxy[1] = sc[1];
        e->zeta[0] = zeta[c];
        e->zeta[1] = zeta[(size_t)n + c];
        e->curvature[0] = curv[c];
        e->curvature[1] = curv[(size_t)n + c];
        for (int k = 0; k < 3; ++k) e->gravity[k] = grav[(size_t)k * n + c];
        for (int k = 0; k < 2; ++k) e->d_gravity[k] = dgrav[(size_t)k * n + c];
        e->elevation = 0.0;
        for (int v = 0; v < 3; ++v) e->Influx[v] = 0.0;
        e->stoppedflags = 0;
        e->Awet = 1.0;
        e->Swet = 1.0;
        e->iwetnode = 8;
        El_Table->add(e->key, e);
        els[c] = e;
    }
    if (ref_static) {
        for (int c = 0; c < n; ++c) els[c]->calc_gravity_vector(&matprops);
        for (int c = 0; c < n; ++c) els[c]->calc_d_gravity(El_Table);
    }

    // ---- time loop of the driver (hpfem.C:222-357) with adaptation off
    std::vector<double> dts(nsteps);
    int order_flag = 1;
    const auto t_start = std::chrono::steady_clock::now();
    for (int it = 0; it < nsteps; ++it) {
        if (timeprops.iter < 50)
            matprops.frict_tiny = 0.1;
        else
            matprops.frict_tiny = 0.000000001;
        step(El_Table, NodeTable, 0, 1, &matprops, &timeprops, &pileprops, &fluxprops, &statprops, &order_flag,
             &outline, &discharge, 0);
        dts[it] = timeprops.dtime;
    }
    const double step_seconds =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    std::fprintf(stderr, "ref_harness_step_seconds=%.9f\n", step_seconds);

    // ---- output in the flattened cell order
    FILE *o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    int32_t oh[3] = {0x314F4144, n, nsteps};
    wr(o, oh, 3);
    wr(o, dts.data(), dts.size());
    wr(o, &timeprops.time, 1);
    std::vector<double> buf((size_t)12 * n);
    for (int v = 0; v < 3; ++v) {
        for (int c = 0; c < n; ++c) buf[c] = els[c]->state_vars[v];
        wr(o, buf.data(), n);
    }
    for (int j = 0; j < 6; ++j) {
        for (int c = 0; c < n; ++c) buf[c] = els[c]->d_state_vars[j];
        wr(o, buf.data(), n);
    }
    for (int c = 0; c < n; ++c) buf[c] = els[c]->kactxy[0];
    wr(o, buf.data(), n);
    for (int r = 0; r < 4; ++r) {
        const int a = (r + 1) % 4;
        for (int v = 0; v < 3; ++v) {
            for (int c = 0; c < n; ++c) {
                Node *nd = (Node *)NodeTable->lookup(els[c]->node_key[a + 4]);
                buf[c] = nd ? nd->flux[v] : NAN;
            }
            wr(o, buf.data(), n);
        }
    }
    for (int k = 0; k < 3; ++k) {
        for (int c = 0; c < n; ++c) buf[c] = els[c]->gravity[k];
        wr(o, buf.data(), n);
    }
    for (int k = 0; k < 2; ++k) {
        for (int c = 0; c < n; ++c) buf[c] = els[c]->d_gravity[k];
        wr(o, buf.data(), n);
    }
    // calc_stats of the last step (StatProps) and the discharge through each plane
    const double st_out[22] = {statprops.xcen,     statprops.ycen,    statprops.xvar,       statprops.yvar,
                               statprops.rmean,    statprops.area,    statprops.vmean,      statprops.umean,
                               statprops.vxmean,   statprops.vymean,  statprops.slopemean,  statprops.statvolume,
                               statprops.piler,    statprops.hmax,    statprops.vmax,       statprops.umax,
                               statprops.vstar,    statprops.xyminmax[0], statprops.xyminmax[1],
                               statprops.xyminmax[2], statprops.xyminmax[3], statprops.timereached};
    wr(o, st_out, 22);
    for (int k = 0; k < n_planes; ++k) wr(o, &discharge.planes[k][9], 1);
    std::fclose(o);
    return 0;
}
