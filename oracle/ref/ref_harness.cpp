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
//   'DAJ1' (mesh as 'DAH1', then reverse-step records; see adjoint_mode) -> 'DJO1': the
//       reference's own dual solver steps -- update_dual_grid, calc_jacobian, calc_adjoint --
//       taken backward from a given adjoint.
//   'DAF1' (mesh as 'DAH1', initial state, functional box; see fwdadj_mode) -> 'DFO1': the
//       reference's forward steps with solution recording, then its dual-solver reverse steps,
//       each timed (the CPU baseline of the forward + adjoint path).
//   'DAS1' (mesh as 'DAH1', state, outline grid; see save_mode) -> 'DSO1': nsteps reference
//       steps, then save_forward writes restart_0000 and outline_0000 in the working directory.
//   'DAL1' (materials, nsteps, outline grid; see load_mode) -> 'DLO1': loadrun reads restart_0000
//       and outline_0000 from the working directory, then nsteps reference steps.
//   'DAE1' (the refined error grid, its parents, a coarse step's states and adjoint; see
//       dwr_mode) -> 'DEO1': the reference's DWR estimate of that step -- bilinear_interp,
//       update_bilinear_error_grid, error_compute -- on the error grid.
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

#include "harness_tables.h"

int REFINE_LEVEL = 0;  // global of the reference's driver (hpfem.C)
// the driver's max-h functional (adjoint.h:299); default-constructed, its iteration (0) never
// matches a reverse step, so calc_adjoint's functional sensitivity is zero
MaxH_Functional maxh_func;

void step(HashTable *El_Table, HashTable *NodeTable, int myid, int nump, MatProps *matprops_ptr,
          TimeProps *timeprops_ptr, PileProps *pileprops_ptr, FluxProps *fluxprops, StatProps *statprops_ptr,
          int *order_flag, OutLine *outline_ptr, DISCHARGE *discharge, int adaptflag);

using harness::rd;
using harness::wr;
using harness::MeshIn;
using harness::Props;
using harness::Tables;
using harness::build_tables;
using harness::make_props;
using harness::read_mesh;
using harness::solrec_for;


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

namespace {

// ---- 'DAJ1': the reference's own adjoint, reverse steps from a given lambda
//
// Input after the mesh (header: 'DAJ1', n, max_level, n_materials, K reverse steps, 0):
//   int32 iter[K]           the adjoint iteration of each reverse step, descending (iter = the
//                           forward step U^{iter-1} -> U^iter that is taken back)
//   double dt[K]            TimeProps::dt.at(iter - 1) of each
//   double state[K][3][n]   U^{iter-1}: h, hu, hv
//   double lambda[3][n]     the adjoint of the first reverse step's U^{iter}
// Output: 'DJO1', n, K; double lambda[K][3][n] after each reverse step; double seconds.
//
// The forward states go through the reference's SolRec (record_solution's rule: a zero record
// for h <= 0), the dual elements are the reference's DualElem copies of the elements
// (dual_solver.C:101-106), and each reverse step runs update_dual_grid (prev state and
// prev adjoint, get_slopes_prev + hslope_sens, gmfggetcoef, calc_flux with the flux Jacobians,
// dual_grid_routines.C:15-93), calc_jacobian (calc_jacobain.C:40-153) and calc_adjoint
// (calc_adjoint.C:35-167) as dual_solver does at dual_solver.C:197-206, with the functional
// sensitivity zero (the MaxH functional's iteration never matches).
int adjoint_mode(FILE *f, const int32_t hdr[6], const char *out) {
    MeshIn m;
    read_mesh(f, hdr, m);
    const int n = m.n, K = m.nsteps;
    std::vector<int32_t> iters(K);
    std::vector<double> dts(K), states((size_t)K * 3 * n), lam((size_t)3 * n);
    rd(f, iters.data(), K);
    rd(f, dts.data(), K);
    rd(f, states.data(), states.size());
    rd(f, lam.data(), lam.size());
    std::fclose(f);
    Props pr;
    make_props(m, pr);
    MatProps &matprops = *pr.matprops;
    Tables t = build_tables(m, states.data(), states.data() + n, states.data() + 2 * (size_t)n, matprops, false);

    TimeProps timeprops;
    timeprops.inittime(1 << 30, HUGE_VAL, HUGE_VAL, HUGE_VAL, 1.0);
    int maxit = 0;
    for (int k = 0; k < K; ++k) maxit = std::max(maxit, (int)iters[k]);
    timeprops.dt.assign(maxit + 1, 0.0);
    for (int k = 0; k < K; ++k) timeprops.dt[iters[k] - 1] = dts[k];
    timeprops.adjiter = 1;  // not the seeding pass of calc_adjoint_elem

    // dual grid: one DualElem per element, in the element table's own bucket structure
    HashTable *Dual_El_Tab = new HashTable(t.El_Table);
    std::vector<DualElem *> duals(n);
    for (int c = 0; c < n; ++c) {
        DualElem *d = new DualElem(t.els[c]);
        Dual_El_Tab->add(d->pass_key(), d);
        duals[c] = d;
        for (int v = 0; v < 3; ++v) d->get_adjoint()[v] = lam[(size_t)v * n + c];
    }
    // forward records of every state the sweep takes back
    SolRec *solrec = solrec_for(t, n);
    for (int c = 0; c < n; ++c) {
        Jacobian *j = new Jacobian(t.els[c]->key);
        solrec->add(j->get_key(), j);
        for (int k = 0; k < K; ++k) {
            const double *U = states.data() + (size_t)k * 3 * n;
            if (U[c] > 0.) {
                double s[3] = {U[c], U[(size_t)n + c], U[(size_t)2 * n + c]};
                j->put_solution(new Solution(s), iters[k] - 1);
            } else {
                j->put_solution(&(Solution::solution_zero), iters[k] - 1);
            }
        }
    }
    MeshCTX mctx;
    mctx.el_table = Dual_El_Tab;
    mctx.nd_table = t.NodeTable;
    PropCTX pctx;
    pctx.matprops = &matprops;
    pctx.timeprops = &timeprops;
    pctx.mapnames = nullptr;
    pctx.outline = nullptr;
    pctx.numproc = 1;
    pctx.myid = 0;
    pctx.adapt_flag = 0;

    std::vector<double> outv((size_t)K * 3 * n);
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < K; ++k) {
        timeprops.iter = iters[k];
        update_dual_grid(solrec, &mctx, &pctx);
        calc_jacobian(&mctx, &pctx);
        calc_adjoint(&mctx, &pctx);
        for (int c = 0; c < n; ++c)
            for (int v = 0; v < 3; ++v) outv[((size_t)k * 3 + v) * n + c] = duals[c]->get_adjoint()[v];
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    FILE *o = std::fopen(out, "wb");
    if (!o) return 2;
    const int32_t oh[3] = {0x314F4A44, n, K};
    wr(o, oh, 3);
    wr(o, outv.data(), outv.size());
    wr(o, &secs, 1);
    std::fclose(o);
    return 0;
}

// ---- 'DAF1': the reference's own forward + adjoint, timed step by step
//
// Header: 'DAF1', n, max_level, n_materials, K forward steps, W (the first W steps are not timed
// and not taken back).  After the mesh: double h[n], hu[n], hv[n] (the initial state), box[4].
// K forward steps as the driver takes them (hpfem.C:232-285: frict_tiny, step(), then
// SolRec::record_solution of the step's starting state; the gz flushes every 50 steps are
// skipped), then the dual grid (DualElem copies, dual_solver.C:101-106) seeded with
// lambda^K = dJ/dU^K of J = sum over the cells whose centre lies in the box of h^2 dx dy, then
// K - W reverse steps as dual_solver takes them (setup_dual_flow's update_dual_grid and
// clear_empty_jacobians, calc_jacobian, calc_adjoint; dual_solver.C:183-207 without its one-step
// gating and without the DWR estimate and the output writers).
// Output: 'DFO1', n, K, W; double fwd_seconds[K], rev_seconds[K - W], lambda[3][n] (lambda^W).
int fwdadj_mode(FILE *f, const int32_t hdr[6], const char *out) {
    MeshIn m;
    read_mesh(f, hdr, m);
    const int n = m.n, K = m.nsteps, W = m.flag;
    std::vector<double> h(n), hu(n), hv(n);
    double box[4];
    rd(f, h.data(), n); rd(f, hu.data(), n); rd(f, hv.data(), n);
    rd(f, box, 4);
    std::fclose(f);
    if (W < 0 || W >= K) return 3;
    Props pr;
    make_props(m, pr);
    MatProps &matprops = *pr.matprops;
    TimeProps timeprops;
    timeprops.inittime(1 << 30, HUGE_VAL, HUGE_VAL, HUGE_VAL, 1.0);
    PileProps pileprops;
    FluxProps fluxprops;
    StatProps statprops;
    statprops.hxyminmax = matprops.MAX_NEGLIGIBLE_HEIGHT * 10.0;
    statprops.timereached = -1.0;
    DISCHARGE discharge;
    OutLine outline;
    Tables t = build_tables(m, h.data(), hu.data(), hv.data(), matprops, false);
    SolRec *solrec = solrec_for(t, n);
    MeshCTX fctx;
    fctx.el_table = t.El_Table;
    fctx.nd_table = t.NodeTable;
    PropCTX pctx;
    pctx.matprops = &matprops;
    pctx.timeprops = &timeprops;
    pctx.mapnames = nullptr;
    pctx.outline = nullptr;
    pctx.numproc = 1;
    pctx.myid = 0;
    pctx.adapt_flag = 0;
    int order_flag = 1;
    std::vector<double> fwd_s(K), rev_s(K - W);
    for (int it = 0; it < K; ++it) {
        const auto t0 = std::chrono::steady_clock::now();
        matprops.frict_tiny = timeprops.iter < 50 ? 0.1 : 0.000000001;
        step(t.El_Table, t.NodeTable, 0, 1, &matprops, &timeprops, &pileprops, &fluxprops, &statprops, &order_flag,
             &outline, &discharge, 0);
        solrec->record_solution(&fctx, &pctx);
        fwd_s[it] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    // dual grid seeded with dJ/dU^K
    HashTable *Dual_El_Tab = new HashTable(t.El_Table);
    std::vector<DualElem *> duals(n);
    for (int c = 0; c < n; ++c) {
        DualElem *d = new DualElem(t.els[c]);
        Dual_El_Tab->add(d->pass_key(), d);
        duals[c] = d;
        const double *cc = t.els[c]->coord;
        const bool in = cc[0] >= box[0] && cc[0] <= box[1] && cc[1] >= box[2] && cc[1] <= box[3];
        d->get_adjoint()[0] = in ? 2.0 * t.els[c]->state_vars[0] * (t.els[c]->dx[0] * t.els[c]->dx[1]) : 0.0;
        d->get_adjoint()[1] = d->get_adjoint()[2] = 0.0;
    }
    MeshCTX dctx;
    dctx.el_table = Dual_El_Tab;
    dctx.nd_table = t.NodeTable;
    for (int k = 0; k < K - W; ++k) {
        const int iter = K - k;
        const auto t0 = std::chrono::steady_clock::now();
        timeprops.iter = iter;
        timeprops.adjiter++;
        update_dual_grid(solrec, &dctx, &pctx);
        clear_empty_jacobians(solrec, iter);
        calc_jacobian(&dctx, &pctx);
        calc_adjoint(&dctx, &pctx);
        rev_s[k] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    FILE *o = std::fopen(out, "wb");
    if (!o) return 2;
    const int32_t oh[4] = {0x314F4644, n, K, W};
    wr(o, oh, 4);
    wr(o, fwd_s.data(), K);
    wr(o, rev_s.data(), K - W);
    std::vector<double> lam((size_t)3 * n);
    for (int c = 0; c < n; ++c)
        for (int v = 0; v < 3; ++v) lam[(size_t)v * n + c] = duals[c]->get_adjoint()[v];
    wr(o, lam.data(), lam.size());
    std::fclose(o);
    return 0;
}

// The driver's time loop with adaptation off (hpfem.C:222-357): frict_tiny by iteration, step().
void drive(HashTable *El_Table, HashTable *NodeTable, MatProps &matprops, TimeProps &timeprops, int nsteps) {
    PileProps pileprops;
    FluxProps fluxprops;
    StatProps statprops;
    statprops.hxyminmax = matprops.MAX_NEGLIGIBLE_HEIGHT * 10.0;
    statprops.timereached = -1.0;
    DISCHARGE discharge;
    OutLine outline;
    int order_flag = 1;
    for (int it = 0; it < nsteps; ++it) {
        matprops.frict_tiny = timeprops.iter < 50 ? 0.1 : 0.000000001;
        step(El_Table, NodeTable, 0, 1, &matprops, &timeprops, &pileprops, &fluxprops, &statprops, &order_flag,
             &outline, &discharge, 0);
    }
}

// Every active element (adapted > 0): coordinates and state, then the TimeProps history.
int write_elements(const char *out, int32_t magic, HashTable *El_Table, const TimeProps &tp) {
    std::vector<Element *> act;
    HashEntryPtr *buck = El_Table->getbucketptr();
    for (int b = 0; b < El_Table->get_no_of_buckets(); ++b)
        for (HashEntryPtr e = buck[b]; e; e = e->next) {
            Element *el = (Element *)e->value;
            if (el->adapted > 0) act.push_back(el);
        }
    FILE *o = std::fopen(out, "wb");
    if (!o) return 2;
    const int32_t oh[4] = {magic, (int32_t)act.size(), tp.iter, (int32_t)tp.dt.size()};
    wr(o, oh, 4);
    wr(o, &tp.time, 1);
    if (!tp.dt.empty()) wr(o, tp.dt.data(), tp.dt.size());
    for (Element *el : act) {
        wr(o, el->key, 2);
        wr(o, el->coord, 2);
        wr(o, el->state_vars, 3);
    }
    std::fclose(o);
    return 0;
}

// 'DAS1': the mesh and state as 'DAH1' (nsteps in the header), then double dxy[2], xr[2], yr[2]
// of the outline grid.  nsteps reference steps, then save_forward (restart.C:21-125) writes
// restart_0000 and outline_0000 into the working directory.  Output: 'DSO1' as write_elements.
int save_mode(FILE *f, const int32_t hdr[6], const char *out) {
    MeshIn m;
    read_mesh(f, hdr, m);
    const int n = m.n;
    std::vector<double> h(n), hu(n), hv(n);
    rd(f, h.data(), n); rd(f, hu.data(), n); rd(f, hv.data(), n);
    double dxy[2], xr[2], yr[2];
    rd(f, dxy, 2); rd(f, xr, 2); rd(f, yr, 2);
    std::fclose(f);
    Props pr;
    make_props(m, pr);
    MatProps &matprops = *pr.matprops;
    TimeProps timeprops;
    timeprops.inittime(1 << 30, HUGE_VAL, HUGE_VAL, HUGE_VAL, 1.0);
    Tables t = build_tables(m, h.data(), hu.data(), hv.data(), matprops, false);
    drive(t.El_Table, t.NodeTable, matprops, timeprops, m.nsteps);
    OutLine outline;
    outline.init2(dxy, xr, yr);
    SolRec *solrec = solrec_for(t, n);
    MeshCTX mctx;
    mctx.el_table = t.El_Table;
    mctx.nd_table = t.NodeTable;
    PropCTX pctx;
    pctx.matprops = &matprops;
    pctx.timeprops = &timeprops;
    pctx.mapnames = nullptr;
    pctx.outline = &outline;
    pctx.numproc = 1;
    pctx.myid = 0;
    pctx.adapt_flag = 0;
    save_forward(mctx, pctx, solrec);
    return write_elements(out, 0x314F5344, t.El_Table, timeprops);
}

// 'DAL1': int32 magic, n_materials, nsteps; double intfrict, epsilon, gravity_scale, gamma,
// maxtime, bedfrict[16]; double dxy[2], xr[2], yr[2] of the outline grid in the file.  loadrun
// (restart.C:127-239) rebuilds the tables from restart_0000 / outline_0000 in the working
// directory, then nsteps reference steps.  Output: 'DLO1' as write_elements.
int load_mode(FILE *f, const char *out) {
    MeshIn m;
    int32_t a[2];
    rd(f, a, 2);
    m.nmat = a[0];
    m.nsteps = a[1];
    rd(f, m.sc, 5);
    rd(f, m.bed, 16);
    double dxy[2], xr[2], yr[2];
    rd(f, dxy, 2); rd(f, xr, 2); rd(f, yr, 2);
    std::fclose(f);
    Props pr;
    make_props(m, pr);
    MatProps &matprops = *pr.matprops;
    matprops.number_of_cells_across_axis = 1;
    matprops.smallest_axis = 1.0;
    TimeProps timeprops;
    timeprops.inittime(1 << 30, HUGE_VAL, HUGE_VAL, HUGE_VAL, 1.0);
    OutLine outline;
    outline.init2(dxy, xr, yr);   // loadrun reads the grid with the caller's dimensions
    HashTable *NodeTable = nullptr, *El_Table = nullptr;
    SolRec *solrec = nullptr;
    if (!loadrun(0, 1, &NodeTable, &El_Table, &solrec, &matprops, &timeprops, &outline)) return 4;
    drive(El_Table, NodeTable, matprops, timeprops, m.nsteps);
    return write_elements(out, 0x314F4C44, El_Table, timeprops);
}

// 'DAE1': header (magic, nf, L, n_materials, iter, n); scalars and bed friction as 'DAH1'; the
// error grid as a flattened mesh of nf cells ('DAH1' arrays); int32 parent[nf] (the coarse cell
// each fine cell was split from); double prev[3][n] = U^{iter-1}, state[3][n] = U^{iter},
// adjoint[3][n] of the coarse cells, dt of the step.  As dual_solver does after an adjoint step
// (dual_solver.C:213-230): every fine cell takes its father's prev/state/adjoint
// (send_from_dual_to_error, error_grid_routines.C:129-183), then bilinear_interp,
// update_bilinear_error_grid and error_compute with TimeProps::iter = iter and dt[iter - 1] = dt.
// Output 'DEO1' nf; per fine cell (input order) bilin_state[3] bilin_prev_state[3] bilin_adj[3]
// residual[3] el_error[2] correction.
int dwr_mode(FILE *f, const int32_t hdr[6], const char *out) {
    const int32_t fh[6] = {hdr[0], hdr[1], hdr[2], hdr[3], 0, 0};
    MeshIn m;
    read_mesh(f, fh, m);
    const int nf = m.n, iter = hdr[4], n = hdr[5];
    std::vector<int32_t> parent(nf);
    rd(f, parent.data(), nf);
    std::vector<double> prev((size_t)3 * n), st((size_t)3 * n), adj((size_t)3 * n);
    double dt = 0;
    rd(f, prev.data(), prev.size());
    rd(f, st.data(), st.size());
    rd(f, adj.data(), adj.size());
    rd(f, &dt, 1);
    std::fclose(f);
    if (iter < 1) return 3;
    for (int c = 0; c < nf; ++c)
        if (parent[c] < 0 || parent[c] >= n || m.level[c] < 1) return 3;
    Props pr;
    make_props(m, pr);
    MatProps &matprops = *pr.matprops;
    std::vector<double> zero(nf, 0.0);
    Tables t = build_tables(m, zero.data(), zero.data(), zero.data(), matprops, false);
    // lattice keys of the build (harness_tables.cpp): bubble of a cell at (level, ix, iy), +1 per word
    auto bubble_key = [&](int lev, int64_t ix, int64_t iy, unsigned k[2]) {
        const int64_t s = int64_t(1) << (m.L - lev + 1);
        k[0] = unsigned(ix * s + s / 2 + 1);
        k[1] = unsigned(iy * s + s / 2 + 1);
    };
    static const int off[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};   // sons counter-clockwise
    std::vector<ErrorElem *> errs(nf);
    for (int c = 0; c < nf; ++c) {
        Element *e = t.els[c];
        const int lev = m.level[c];
        const int64_t fx = m.ix[c] >> 1, fy = m.iy[c] >> 1;
        bubble_key(lev - 1, fx, fy, e->father);
        for (int j = 0; j < 4; ++j) {
            bubble_key(lev, 2 * fx + off[j][0], 2 * fy + off[j][1], e->brothers[j]);
            if (2 * fx + off[j][0] == m.ix[c] && 2 * fy + off[j][1] == m.iy[c]) e->which_son = j;
        }
        ErrorElem *ee = new ErrorElem(e);
        const int p = parent[c];
        for (int v = 0; v < 3; ++v) {
            ee->prev_state_vars[v] = prev[(size_t)v * n + p];
            ee->state_vars[v] = st[(size_t)v * n + p];
            ee->adjoint[v] = adj[(size_t)v * n + p];
        }
        t.El_Table->remove(e->key);
        t.El_Table->add(ee->key, ee);
        errs[c] = ee;
    }
    TimeProps timeprops;
    timeprops.inittime(1 << 30, HUGE_VAL, HUGE_VAL, HUGE_VAL, 1.0);
    timeprops.iter = iter;
    timeprops.dt.assign(iter, 0.0);
    timeprops.dt[iter - 1] = dt;
    MeshCTX ectx;
    ectx.el_table = t.El_Table;
    ectx.nd_table = t.NodeTable;
    PropCTX pctx;
    pctx.matprops = &matprops;
    pctx.timeprops = &timeprops;
    pctx.mapnames = nullptr;
    pctx.outline = nullptr;
    pctx.numproc = 1;
    pctx.myid = 0;
    pctx.adapt_flag = 0;
    bilinear_interp(t.El_Table);
    update_bilinear_error_grid(&ectx, &pctx);
    error_compute(&ectx, &pctx);
    FILE *o = std::fopen(out, "wb");
    if (!o) return 2;
    const int32_t oh[2] = {0x314F4544, nf};
    wr(o, oh, 2);
    for (int c = 0; c < nf; ++c) {
        ErrorElem *e = errs[c];
        wr(o, e->bilin_state, 3);
        wr(o, e->bilin_prev_state, 3);
        wr(o, e->bilin_adj, 3);
        wr(o, e->residual, 3);
        wr(o, e->el_error, 2);
        wr(o, &e->correction, 1);
    }
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
    if (magic == 0x314C4144) return load_mode(f, argv[2]);
    int32_t hdr[6];
    hdr[0] = magic;
    rd(f, hdr + 1, 5);
    if (hdr[0] == 0x314A4144) return adjoint_mode(f, hdr, argv[2]);
    if (hdr[0] == 0x31464144) return fwdadj_mode(f, hdr, argv[2]);
    if (hdr[0] == 0x31534144) return save_mode(f, hdr, argv[2]);
    if (hdr[0] == 0x31454144) return dwr_mode(f, hdr, argv[2]);
    if (hdr[0] != 0x31484144) return 3;
    MeshIn m;
    read_mesh(f, hdr, m);
    const int n = m.n, nsteps = m.nsteps, ref_static = m.flag;
    std::vector<double> h(n), hu(n), hv(n);
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

    Props pr;
    make_props(m, pr);
    MatProps &matprops = *pr.matprops;
    matprops.Vslump = stat_in[3];
    TimeProps timeprops;
    timeprops.inittime(1 << 30, m.sc[4], HUGE_VAL, HUGE_VAL, 1.0);
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

    Tables t = build_tables(m, h.data(), hu.data(), hv.data(), matprops, ref_static != 0);
    HashTable *El_Table = t.El_Table, *NodeTable = t.NodeTable;
    std::vector<Element *> &els = t.els;

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
