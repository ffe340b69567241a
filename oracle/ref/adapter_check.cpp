// The drop-in adapter (the element-table flattening and the step() replacement) compiled against the
// reference's own headers and linked with its objects and with libda_b200.so, then checked against
// the reference.
// TEST INFRASTRUCTURE ONLY: built by oracle/ref_build.py into oracle/_ref/adapter_check.
//
// The adapter is what a maintainer adds to the reference: da_flatten walks the reference's element
// table (Element::get_positive_x_side, neighbour keys and neigh_proc, element2.C:694-716) into the
// flattened SoA of include/discrete_adjoint.h and uploads it; adapter_step replaces the body of
// step() (src/geoflow/step.C:29, called at src/main/hpfem.C:271) by da_forward_step.
//
// usage: adapter_check in.bin out.bin
// Input: int32 'DAI1', n, max_level, n_materials, nsteps, mode (0: flatten only, 1: flatten and
// step), the mesh as harness_tables.h describes, then double h[n], hu[n], hv[n].
// The reference's tables are rebuilt from the input mesh (oracle/ref/harness_tables.cpp), the
// adapter flattens them, and the flattening is compared with the input: neighbour table (mapped
// through the elements back to the input's cell order) and every per-cell field, bit for bit.
// Mode 1 then steps a second copy of the tables with the reference's own step() and the first copy
// with the adapter (the device path), nsteps times, and compares state, dt and time bit for bit.
// Output: int32 'DIO1', n, nbr_mismatch, field_mismatch, state_mismatch, dt_mismatch, steps;
//         double max |state difference|.
#include <algorithm>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include <hdf5.h>
#include <mpi.h>

#include "hpfem.h"

#include "discrete_adjoint.h"
#include "harness_tables.h"

int REFINE_LEVEL = 0;        // globals of the reference's driver (hpfem.C)
MaxH_Functional maxh_func;

void step(HashTable *El_Table, HashTable *NodeTable, int myid, int nump, MatProps *matprops_ptr,
          TimeProps *timeprops_ptr, PileProps *pileprops_ptr, FluxProps *fluxprops, StatProps *statprops_ptr,
          int *order_flag, OutLine *outline_ptr, DISCHARGE *discharge, int adaptflag);

// ============================================================================ the adapter
namespace adapter {

da_ctx *g_da = nullptr;
std::vector<Element *> g_cells;  // flattened order
std::vector<int32_t> nbr, mat;
std::vector<double> x, y, dx, dy, g, dg, kv;

uint64_t key64(const unsigned *k) { return (uint64_t(k[0]) << 32) | uint64_t(k[1]); }

// Once per adapt (hpfem.C:243-267): the element table as the C ABI's flattened mesh.
int da_flatten(HashTable *El_Table, int epoch, bool upload) {
    g_cells.clear();
    for (int b = 0; b < El_Table->get_no_of_buckets(); ++b)
        for (HashEntryPtr e = *(El_Table->getbucketptr() + b); e; e = e->next) {
            Element *el = (Element *)e->value;
            if (el->get_adapted_flag() > 0) g_cells.push_back(el);
        }
    // the order of the element keys (the reference's space-filling curve) keeps neighbours close
    std::sort(g_cells.begin(), g_cells.end(),
              [](Element *a, Element *b) { return key64(a->pass_key()) < key64(b->pass_key()); });
    const int n = (int)g_cells.size();
    std::unordered_map<uint64_t, int32_t> index;
    index.reserve(2 * (size_t)n);
    for (int i = 0; i < n; ++i) index[key64(g_cells[i]->pass_key())] = i;
    nbr.assign(8 * (size_t)n, -1);
    mat.assign(n, 0);
    x.assign(n, 0.0); y.assign(n, 0.0); dx.assign(n, 0.0); dy.assign(n, 0.0);
    g.assign(3 * (size_t)n, 0.0); dg.assign(2 * (size_t)n, 0.0); kv.assign(2 * (size_t)n, 0.0);
    for (int i = 0; i < n; ++i) {
        Element *el = g_cells[i];
        const int xp = el->get_positive_x_side();
        for (int r = 0; r < 4; ++r) {  // relative side: +x, +y, -x, -y
            const int a = (xp + r) % 4;
            if (el->get_neigh_proc()[a] == INIT) continue;  // domain edge stays -1
            // the table lists a side's two finer neighbours lower / left first; the element keeps
            // them counter-clockwise, which on +y and -x is the other way round
            const int s1 = (r == 1 || r == 2) ? 4 : 0;
            nbr[(size_t)r * n + i] = index.at(key64(el->get_neighbors() + 2 * (a + s1)));
            nbr[(size_t)(r + 4) * n + i] = index.at(key64(el->get_neighbors() + 2 * (a + 4 - s1)));
        }
        x[i] = el->get_coord()[0];
        y[i] = el->get_coord()[1];
        dx[i] = el->get_dx()[0];
        dy[i] = el->get_dx()[1];
        for (int k = 0; k < 3; ++k) g[(size_t)k * n + i] = el->get_gravity()[k];
        for (int k = 0; k < 2; ++k) {
            dg[(size_t)k * n + i] = el->get_d_gravity()[k];
            kv[(size_t)k * n + i] = el->get_curvature()[k];
        }
        mat[i] = el->get_material() - 1;  // the reference counts materials from 1
    }
    if (!upload) return DA_OK;
    da_mesh_soa m = {n, nbr.data(), x.data(), y.data(), dx.data(), dy.data(), g.data(), dg.data(), kv.data(),
                     mat.data()};
    return da_upload_mesh(g_da, &m, epoch);
}

// State between the elements and the device, in the flattened order.
int push_state() {
    const size_t n = g_cells.size();
    std::vector<double> h(n), hu(n), hv(n);
    for (size_t i = 0; i < n; ++i) {
        h[i] = g_cells[i]->get_state_vars()[0];
        hu[i] = g_cells[i]->get_state_vars()[1];
        hv[i] = g_cells[i]->get_state_vars()[2];
    }
    return da_set_state(g_da, h.data(), hu.data(), hv.data());
}
int pull_state() {
    const size_t n = g_cells.size();
    std::vector<double> h(n), hu(n), hv(n);
    const int rc = da_get_state(g_da, h.data(), hu.data(), hv.data());
    if (rc != DA_OK) return rc;
    for (size_t i = 0; i < n; ++i) {
        g_cells[i]->get_state_vars()[0] = h[i];
        g_cells[i]->get_state_vars()[1] = hu[i];
        g_cells[i]->get_state_vars()[2] = hv[i];
    }
    return DA_OK;
}

// The MatProps / TimeProps fields the path reads (angles already in radians).
da_params params_of(const MatProps *mp, const TimeProps *tp) {
    da_params p;
    da_params_default(&p);
    p.epsilon = mp->epsilon;
    p.gravity_scale = mp->GRAVITY_SCALE;
    p.gamma = mp->gamma;
    p.intfrict = mp->intfrict;
    p.n_materials = mp->material_count;
    for (int k = 0; k < p.n_materials; ++k) p.bedfrict[k] = mp->bedfrict[k + 1];
    p.max_time = tp->ndmaxtime;
    p.next_output = tp->ndnextoutput;
    p.next_save = tp->ndnextsave;
    return p;
}

// The body of step(): the parameters, one device step, the TimeProps bookkeeping incrtime does.
int adapter_step(MatProps *mp, TimeProps *tp, StatProps *sp) {
    const da_params p = params_of(mp, tp);
    int rc = da_set_params(g_da, &p);
    if (rc == DA_OK) rc = da_set_time(g_da, tp->time, tp->iter);
    da_step_stats s;
    if (rc == DA_OK) rc = da_forward_step(g_da, &s);
    if (rc != DA_OK) {
        std::fprintf(stderr, "adapter: %s\n", da_last_error(g_da));
        return rc;
    }
    tp->dtime = s.dt;
    tp->time = s.time;
    tp->iter = (int)s.iter;
    tp->dt.push_back(s.dt);
    sp->realvolume = s.volume;
    return DA_OK;
}

}  // namespace adapter

// ============================================================================ the check
int main(int argc, char **argv) {
    using namespace harness;
    if (argc != 3) {
        std::fprintf(stderr, "usage: adapter_check in.bin out.bin\n");
        return 2;
    }
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t hdr[6];
    rd(f, hdr, 6);
    if (hdr[0] != 0x31494144) return 3;
    MeshIn m;
    read_mesh(f, hdr, m);
    const int n = m.n, nsteps = m.nsteps, mode = m.flag;
    std::vector<double> h(n), hu(n), hv(n);
    rd(f, h.data(), n);
    rd(f, hu.data(), n);
    rd(f, hv.data(), n);
    std::fclose(f);

    Props pa;
    make_props(m, pa);
    Tables A = build_tables(m, h.data(), hu.data(), hv.data(), *pa.matprops, false);
    std::unordered_map<Element *, int> input_index;
    for (int c = 0; c < n; ++c) input_index[A.els[c]] = c;

    int32_t nbr_mismatch = 0, field_mismatch = 0, state_mismatch = 0, dt_mismatch = 0;
    double max_diff = 0.0;
    if (adapter::da_flatten(A.El_Table, 0, false) != DA_OK) return 4;
    if ((int)adapter::g_cells.size() != n) return 5;
    for (int i = 0; i < n; ++i) {
        const int c = input_index.at(adapter::g_cells[i]);
        for (int s = 0; s < 8; ++s) {
            const int e = adapter::nbr[(size_t)s * n + i];
            const int mapped = e < 0 ? -1 : input_index.at(adapter::g_cells[e]);
            if (mapped != m.nbr[(size_t)s * n + c]) ++nbr_mismatch;
        }
        bool same = adapter::x[i] == m.x[c] && adapter::y[i] == m.y[c] && adapter::dx[i] == m.dx[c] &&
                    adapter::dy[i] == m.dy[c] && adapter::mat[i] == m.mat[c];
        for (int k = 0; k < 3; ++k) same = same && adapter::g[(size_t)k * n + i] == m.grav[(size_t)k * n + c];
        for (int k = 0; k < 2; ++k)
            same = same && adapter::dg[(size_t)k * n + i] == m.dgrav[(size_t)k * n + c] &&
                   adapter::kv[(size_t)k * n + i] == m.curv[(size_t)k * n + c];
        if (!same) ++field_mismatch;
    }

    int steps_done = 0;
    if (mode == 1) {
        // the reference's own step() on a second copy of the tables (the driver's loop, hpfem.C:222-271)
        Props pb;
        make_props(m, pb);
        Tables B = build_tables(m, h.data(), hu.data(), hv.data(), *pb.matprops, false);
        TimeProps ta, tb;
        ta.inittime(1 << 30, m.sc[4], HUGE_VAL, HUGE_VAL, 1.0);
        tb.inittime(1 << 30, m.sc[4], HUGE_VAL, HUGE_VAL, 1.0);
        PileProps pile;
        FluxProps flux;
        StatProps sa, sb;
        sb.hxyminmax = pb.matprops->MAX_NEGLIGIBLE_HEIGHT * 10.0;
        sb.timereached = -1.0;
        DISCHARGE discharge;
        OutLine outline;
        int order_flag = 1;
        // the device context (created with the run's materials) and the adapter's tables
        const da_params p = adapter::params_of(pa.matprops, &ta);
        int err = 0;
        adapter::g_da = da_create(&p, &err);
        if (!adapter::g_da) return 6;
        if (adapter::da_flatten(A.El_Table, 0, true) != DA_OK || adapter::push_state() != DA_OK) {
            std::fprintf(stderr, "adapter: %s\n", da_last_error(adapter::g_da));
            return 7;
        }
        for (int it = 0; it < nsteps; ++it) {
            pb.matprops->frict_tiny = tb.iter < 50 ? 0.1 : 0.000000001;
            step(B.El_Table, B.NodeTable, 0, 1, pb.matprops, &tb, &pile, &flux, &sb, &order_flag, &outline,
                 &discharge, 0);
            if (adapter::adapter_step(pa.matprops, &ta, &sa) != DA_OK) return 8;
            ++steps_done;
        }
        if (adapter::pull_state() != DA_OK) return 9;
        for (int c = 0; c < n; ++c)
            for (int v = 0; v < 3; ++v) {
                const double a = A.els[c]->get_state_vars()[v], b = B.els[c]->get_state_vars()[v];
                if (!(a == b)) ++state_mismatch;
                max_diff = std::max(max_diff, std::fabs(a - b));
            }
        if (ta.dt.size() != tb.dt.size()) dt_mismatch = 1 << 20;
        for (size_t k = 0; k < ta.dt.size() && k < tb.dt.size(); ++k)
            if (!(ta.dt[k] == tb.dt[k])) ++dt_mismatch;
        if (!(ta.time == tb.time) || ta.iter != tb.iter) ++dt_mismatch;
        da_destroy(adapter::g_da);
    }
    FILE *o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    const int32_t out[7] = {0x314F4944, n, nbr_mismatch, field_mismatch, state_mismatch, dt_mismatch, steps_done};
    wr(o, out, 7);
    wr(o, &max_diff, 1);
    std::fclose(o);
    return 0;
}
