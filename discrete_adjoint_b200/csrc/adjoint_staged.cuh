// Gather phase of the cooperative reverse step with each listed tile staged in shared memory
// (included by adjoint_kernels.cuh).
//
// The gather of cell j reads, at j and at every face neighbour k, U^n, lambda^{n+1}, the recorded
// branch byte, boundary flags, material, g_z, the cell sizes and the slope coefficients B that the
// source phase wrote.  Read from global memory, each face is a chain of dependent loads (the
// neighbour index, then its values, then its branch byte through the tile epoch), taken one face
// after another.  Here all of it is copied first, for the tile's 256 cells and its halo (the same
// host-built halo lists as the forward phases), by asynchronous copies (cp.async) and plain byte
// loads all in flight together; the faces then read shared memory.  The tile's own A, running
// parameter sensitivities and neighbour slots come along.  The arithmetic and its order are
// adj_gather_phase's, so results are identical.
#pragma once

namespace da {
namespace adj {
namespace {

using fwd::kSlots;

template <class R>
struct GatherBuf {
    uint4 nl[kTileCells];                     // the tile's cells' neighbour slots (8 x int16)
    double b[4][kSlots];                      // slope coefficients B per side
    double a[3][kTileCells];                  // A of the tile's cells
    double gb[kTileCells], gi[kTileCells];    // running d J / d phi_bed, phi_int of the tile's cells
    R h[kSlots], hu[kSlots], hv[kSlots];      // U^n
    R lh[kSlots], lhu[kSlots], lhv[kSlots];   // lambda^{n+1}
    R gz[kSlots];                             // g_z
    R sx[kSlots], sy[kSlots];                 // cell sizes (FP64: dx, dy; FP32: the float sizes)
    uint8_t mask[kSlots];                     // recorded branch byte, 0 outside this recording
    uint8_t bf[kSlots];                       // boundary / two-neighbour flags
    uint8_t mat[kSlots];                      // material
};

template <class R>
struct GatherSmem {
    GatherBuf<R> g;
    double term[4][2][5][64];  // quarter mode: the face terms of side s, neighbour q, per cell
    int hoff[kTileCells];      // halo range of each listed tile of the round
    int hcnt[kTileCells];
};

template <class R>
constexpr size_t gather_smem_bytes() {
    return sizeof(GatherSmem<R>);
}

// The copies of one slot's values (slot s, cell e).
template <class R>
__device__ __forceinline__ void gather_slot(GatherBuf<R> &g, int s, int e, const MeshArgs &m, const StateRef<R> &U,
                                            const StateRef<R> &L, const AdjArgs &aa) {
    constexpr int B = sizeof(R);
    using fwd::cp_async;
    cp_async<B>(&g.h[s], U.h + e);
    cp_async<B>(&g.hu[s], U.hu + e);
    cp_async<B>(&g.hv[s], U.hv + e);
    cp_async<B>(&g.lh[s], L.h + e);
    cp_async<B>(&g.lhu[s], L.hu + e);
    cp_async<B>(&g.lhv[s], L.hv + e);
    if constexpr (sizeof(R) == 8) {
        cp_async<B>(&g.gz[s], m.g + (size_t)2 * m.n + e);
        cp_async<B>(&g.sx[s], m.dx + e);
        cp_async<B>(&g.sy[s], m.dy + e);
    } else {
        cp_async<B>(&g.gz[s], m.fg + (size_t)2 * m.n + e);
        cp_async<B>(&g.sx[s], m.fdx + e);
        cp_async<B>(&g.sy[s], m.fdy + e);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) cp_async<8>(&g.b[q][s], aa.B + (size_t)q * m.n + e);
}

// The byte fields of one slot (plain loads; the branch byte of a cell whose tile the recording
// step did not list is 0).
__device__ __forceinline__ void gather_bytes(uint8_t &mk, uint8_t &bf, uint8_t &mat, int e, const MeshArgs &m,
                                             const AdjArgs &aa) {
    const int ep = aa.tile_epoch[e >> 8];
    const uint8_t mv = aa.mask[e];
    bf = m.bflag[e];
    mat = m.mat[e];
    mk = ep == aa.rec_id ? mv : uint8_t(0);
}

// Tile t and its halo (hc cells of the halo list from hoff) into g; returns with every value in
// shared memory and every thread past the copy.  Thread c copies cell c of the tile and halo cell
// c (a halo holds at most kHaloMax <= kTileCells cells).
template <class R>
__device__ __forceinline__ void gather_stage(GatherBuf<R> &g, int t, int hoff, int hc, const fwd::HaloArgs &ha,
                                             const MeshArgs &m, const StateRef<R> &U, const StateRef<R> &L,
                                             const AdjArgs &aa) {
    static_assert(kHaloMax <= kTileCells, "one halo cell per thread");
    const int c = threadIdx.x;
    const int i = t * kTileCells + c;
    const bool own = i < m.n;
    const int e = c < hc ? ha.idx[hoff + c] : -1;
    uint8_t mk = 0, bf = 0, mat = 0, hmk = 0, hbf = 0, hmat = 0;
    if (own) gather_bytes(mk, bf, mat, i, m, aa);
    if (own) {
        gather_slot<R>(g, c, i, m, U, L, aa);
        fwd::cp_async<16>(&g.nl[c], ha.nloc + (size_t)i * 8);
#pragma unroll
        for (int q = 0; q < 3; ++q) fwd::cp_async<8>(&g.a[q][c], aa.A + (size_t)q * m.n + i);
        fwd::cp_async<8>(&g.gb[c], aa.gbed + i);
        fwd::cp_async<8>(&g.gi[c], aa.gint + i);
    }
    if (e >= 0) {
        gather_bytes(hmk, hbf, hmat, e, m, aa);
        gather_slot<R>(g, kTileCells + c, e, m, U, L, aa);
    }
    fwd::cp_async_commit();
    // the byte fields, their loads in flight with the copies
    g.mask[c] = mk;
    g.bf[c] = bf;
    g.mat[c] = mat;
    if (e >= 0) {
        g.mask[kTileCells + c] = hmk;
        g.bf[kTileCells + c] = hbf;
        g.mat[kTileCells + c] = hmat;
    }
    fwd::cp_async_wait_all();
    __syncthreads();
}

// The terms face (s, q) of cell c adds to lambda_j (staged tile): tb the neighbour's slope
// coefficient (to the depth row), tg the flux adjoint, tk the k act/pass sensitivity.  A term the
// face does not have is -0.0, which adds exactly nothing, so summing all of them in face order
// gives the same bits as adding only the present ones.
template <class R>
__device__ __forceinline__ void gather_face(const GatherBuf<R> &g, const MatConsts &mc, int c, int s, int qq,
                                            uint8_t bf, uint8_t mj, R h_j, const R lj[3], R dt, double &tb,
                                            double tg[3], double &tk) {
    tb = tg[0] = tg[1] = tg[2] = tk = -0.0;
    if (bf & (1 << s)) return;
    if (qq && !(bf & (0x10 << s))) return;
    const int d = s & 1;
    const bool plus = s < 2;
    const int sl = reinterpret_cast<const int16_t *>(&g.nl[c])[s + 4 * qq];
    const uint8_t bk = g.bf[sl];
    const R h_k = g.h[sl];
    if (h_k > R(DA_TINY)) {
        // slope coefficient of neighbour k for j (k's side s^2 faces j)
        double bk_s = g.b[s ^ 2][sl];
        if (bk & (0x10 << (s ^ 2))) bk_s *= 0.5;
        tb = bk_s;
    }
    if (!(h_k >= R(DA_TINY) || h_j >= R(DA_TINY))) return;
    const R wj = side_outflow<R>(bf, s) ? R(0) : side_weight_of<R>(d == 0 ? g.sx[c] : g.sy[c], bf, s, dt);
    const R wk = side_outflow<R>(bk, s ^ 2) ? R(0) : side_weight_of<R>(d == 0 ? g.sx[sl] : g.sy[sl], bk, s ^ 2, dt);
    if (wj == R(0) && wk == R(0)) return;
    const uint8_t mk = g.mask[sl];
    const R lk[3] = {(mk & 4) ? R(0) : g.lh[sl], g.lhu[sl], g.lhv[sl]};
    const R mu[3] = {wj * lj[0] + wk * lk[0], wj * lj[1] + wk * lk[1], wj * lj[2] + wk * lk[2]};
    if (mu[0] == R(0) && mu[1] == R(0) && mu[2] == R(0)) return;
    // the edge's left and right sides: j then k on a plus side, k then j on a minus side
    const int eL = plus ? c : sl, eR = plus ? sl : c;
    const uint8_t mL = plus ? mj : mk, mR = plus ? mk : mj;
    Side<R> sL, sR;
    side_of<R>(mc, d, g.h[eL], g.hu[eL], g.hv[eL], g.gz[eL], g.mat[eL], mL, sL);
    side_of<R>(mc, d, g.h[eR], g.hu[eR], g.hv[eR], g.gz[eR], g.mat[eR], mR, sR);
    R gL[3], gR[3], gkL, gkR;
    riemann_adj<R>(d, sL, sR, mu, gL, gR, gkL, gkR);
    tg[0] = double(plus ? gL[0] : gR[0]);
    tg[1] = double(plus ? gL[1] : gR[1]);
    tg[2] = double(plus ? gL[2] : gR[2]);
    tk = double(plus ? gkL : gkR);
}

// lambda^n of an active cell c of the staged tile from its face terms (face(s, q, tb, tg, tk)
// gives them in face order), and its parameter sensitivities.
template <class R, bool BATCH, class Faces>
__device__ __forceinline__ void gather_cell(const GatherBuf<R> &g, const AdjArgs &aa, const InstArgs &ia, int inst,
                                            int c, int j, const R lj[3], uint8_t mj, const StateOut<R> &Lout,
                                            const Faces &face) {
    double out[3] = {double(lj[0]), double(lj[1]), double(lj[2])};
    if (g.h[c] > R(DA_TINY)) {
        out[0] += g.a[0][c];
        out[1] += g.a[1][c];
        out[2] += g.a[2][c];
    }
    // the branch's parameter derivatives, loaded ahead of the faces
    const uint8_t code = mj & 3;
    const int mat = g.mat[c];
    const InstTables it = inst_tables<BATCH>(aa, ia, inst);
    const double dkb = dk_of(it.dk_dbed, mat, code), dki = dk_of(it.dk_dint, mat, code);
    double dJ_dkj = 0.0;
    // faces f = 2 s + q in the order side s = 0..3, neighbour q = 0 (1 on a hanging side); in
    // FP64 one loop body for all of them keeps the code small
#pragma unroll(sizeof(R) == 8 ? 1 : 8)
    for (int f = 0; f < 8; ++f) {
        double tb, tg[3], tk;
        face(f >> 1, f & 1, tb, tg, tk);
        out[0] += tb;
        out[0] += tg[0];
        out[1] += tg[1];
        out[2] += tg[2];
        dJ_dkj += tk;
    }
    Lout.h[j] = R(out[0]);
    Lout.hu[j] = R(out[1]);
    Lout.hv[j] = R(out[2]);
    if (dJ_dkj != 0.0) {
        aa.gbed[j] = g.gb[c] + dJ_dkj * dkb;
        aa.gint[j] = g.gi[c] + dJ_dkj * dki;
    }
}

// adj_gather_phase with every listed tile staged.  The tile listing is the same (tiles the
// recording step listed with an active segment, and tiles whose two adjoint buffers differ); a
// segment's "both buffers agree" flag is set exactly where none of its cells is active, as
// there (a recorded tile's segment activity is the OR of its cells' active bits).
// Two ways to share the work out, with the same results:
// * tiles (a block per listed tile, a thread per cell), when the listed tiles keep the grid busy;
// * quarters (quarter = true: a block per listed quarter tile of 64 cells, a thread per cell and
//   side): a flow over few tiles is spread over four times as many blocks, and each thread takes
//   one face instead of a cell's four, which shortens the dependent FP64 chain of a cell about
//   fourfold.  The face terms meet in shared memory and the cell's thread adds them in face order.
template <class R, bool BATCH>
__device__ __forceinline__ void adj_gather_phase_staged(const MeshArgs &m, const fwd::HaloArgs &ha,
                                                        const StateRef<R> &U, const StateRef<R> &Lnext,
                                                        const StateOut<R> &Lout, const MatConsts &mc0,
                                                        const AdjArgs &aa, R dt0, int *list, const InstArgs &ia,
                                                        GatherSmem<R> &S, bool quarter) {
    GatherBuf<R> &g = S.g;
    const int lane = threadIdx.x & 31;
    const int nunits = quarter ? 4 * aa.ntiles : aa.ntiles;
    for (int round = 0; sched_more(round, nunits); ++round) {
        const int uq = sched_tile(round);
        const int tq = quarter ? uq >> 2 : uq;
        bool need = false;
        if (uq < nunits) {
            const int ep = aa.tile_epoch[tq];
            if (quarter) {
                // the quarter's two segments
                const size_t o = (size_t)tq * 8 + 2 * (uq & 3);
                const unsigned sa = *reinterpret_cast<const uint16_t *>(aa.seg_act + o);
                const unsigned lc = *reinterpret_cast<const uint16_t *>(aa.lam_clean + o);
                need = (ep == aa.rec_id && sa != 0u) || lc != 0x0101u;
            } else {
                const unsigned long long sa = seg_flags8(aa.seg_act, tq), lc = seg_flags8(aa.lam_clean, tq);
                need = (ep == aa.rec_id && sa != 0ull) || lc != 0x0101010101010101ull;
            }
        }
        int ho, hc;
        fwd::halo_range(ha, uq < nunits ? tq : aa.ntiles, aa.ntiles, ho, hc);
        const int cnt = compact_tiles(need, uq, list, ho, hc, S.hoff, S.hcnt);
        for (int q = 0; q < cnt; ++q) {
            const int u = list[q];
            const int t = quarter ? u >> 2 : u;
            gather_stage<R>(g, t, S.hoff[q], S.hcnt[q], ha, m, U, Lnext, aa);
            const int inst = BATCH ? ia.tile_inst[t] : 0;
            const MatConsts &mc = BATCH ? ia.mcs[inst] : mc0;
            const R dt = BATCH ? R(ia.dt[inst]) : dt0;
            if (!quarter) {
                const int c = threadIdx.x;
                const int j = t * kTileCells + c;
                const uint8_t mj = g.mask[c];  // 0 for cells past n
                const bool act = (mj & 8) != 0;
                const unsigned act_bits = __ballot_sync(0xffffffffu, act);
                if (lane == 0) aa.lam_clean[j >> 5] = act_bits ? 0 : 1;
                if (j < m.n) {
                    const R lj[3] = {(mj & 4) ? R(0) : g.lh[c], g.lhu[c], g.lhv[c]};
                    if (!act) {
                        // not active in the forward step: its update was the identity, and no neighbour is wet
                        Lout.h[j] = g.lh[c];
                        Lout.hu[j] = g.lhu[c];
                        Lout.hv[j] = g.lhv[c];
                    } else {
                        const uint8_t bf = g.bf[c];
                        const R h_j = g.h[c];
                        gather_cell<R, BATCH>(g, aa, ia, inst, c, j, lj, mj, Lout,
                                              [&](int s, int qq, double &tb, double tg[3], double &tk) {
                                                  gather_face<R>(g, mc, c, s, qq, bf, mj, h_j, lj, dt, tb, tg, tk);
                                              });
                    }
                }
            } else {
                // thread = side s (0..3) x cell cl (0..63) of the quarter
                const int s = threadIdx.x >> 6, cl = threadIdx.x & 63;
                const int c = (u & 3) * 64 + cl;
                const int j = t * kTileCells + c;
                const uint8_t mj = g.mask[c];  // 0 for cells past n
                const bool act = (mj & 8) != 0;
                const R lj[3] = {(mj & 4) ? R(0) : g.lh[c], g.lhu[c], g.lhv[c]};
                if (act) {
                    const uint8_t bf = g.bf[c];
                    const R h_j = g.h[c];
#pragma unroll
                    for (int qq = 0; qq < 2; ++qq) {
                        double tb, tg[3], tk;
                        gather_face<R>(g, mc, c, s, qq, bf, mj, h_j, lj, dt, tb, tg, tk);
                        S.term[s][qq][0][cl] = tb;
                        S.term[s][qq][1][cl] = tg[0];
                        S.term[s][qq][2][cl] = tg[1];
                        S.term[s][qq][3][cl] = tg[2];
                        S.term[s][qq][4][cl] = tk;
                    }
                }
                __syncthreads();
                if (s == 0) {
                    const unsigned act_bits = __ballot_sync(0xffffffffu, act);
                    if (lane == 0) aa.lam_clean[j >> 5] = act_bits ? 0 : 1;
                    if (j < m.n) {
                        if (!act) {
                            Lout.h[j] = g.lh[c];
                            Lout.hu[j] = g.lhu[c];
                            Lout.hv[j] = g.lhv[c];
                        } else {
                            gather_cell<R, BATCH>(g, aa, ia, inst, c, j, lj, mj, Lout,
                                                  [&](int sd, int qq, double &tb, double tg[3], double &tk) {
                                                      tb = S.term[sd][qq][0][cl];
                                                      tg[0] = S.term[sd][qq][1][cl];
                                                      tg[1] = S.term[sd][qq][2][cl];
                                                      tg[2] = S.term[sd][qq][3][cl];
                                                      tk = S.term[sd][qq][4][cl];
                                                  });
                        }
                    }
                }
            }
            __syncthreads();  // every thread is done with the tile before the next one is copied
        }
    }
}

// The reverse step's source adjoint inside its staged update phase: lambda^{n+1} of a wet cell is
// loaded before its update, the slopes, velocities and friction signs are the update's own, the
// rest comes from the update's staged tile.
template <class R, bool BATCH>
struct SrcEpilogue {
    const MeshArgs &m;
    const StateRef<R> &Ln;
    const MatConsts &mc;
    const AdjArgs &aa;
    const InstArgs &ia;
    R dt, ft;
    struct Pre {
        R l[3];
    };
    __device__ __forceinline__ Pre pre(int i, bool wet) const {
        Pre p{};
        if (wet) {
            p.l[0] = Ln.h[i];
            p.l[1] = Ln.hu[i];
            p.l[2] = Ln.hv[i];
        }
        return p;
    }
    // inside the update of wet cell i (h > GEOFLOW_TINY), with the forward's source quantities f
    __device__ __forceinline__ void operator()(int t, int i, const fwd::StagedView<R> &v, int c, const R *prev,
                                               uint8_t bf, uint8_t code, R gz, const CellSrc<R> &cs, const Pre &p,
                                               const SrcFwd<R> &f) const {
        const int inst = BATCH ? ia.tile_inst[t] : 0;
        const MatConsts &mci = BATCH ? ia.mcs[inst] : mc;
        const R dti = BATCH ? R(ia.dt[inst]) : dt;
        adj_src_wet<R>(v, c, m, prev, gz, code, bf, p.l, cs, mci, aa, inst_tables<BATCH>(aa, ia, inst), dti, ft, i,
                       [&]() -> const SrcFwd<R> & { return f; });
    }
};

}  // namespace
}  // namespace adj
}  // namespace da
