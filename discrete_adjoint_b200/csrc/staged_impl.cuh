// Staged coefficient and update phases of the cooperative step kernels (included by
// forward_impl.cuh).
//
// A block works through its listed tiles one after another.  The values a tile's cells read at
// their neighbours (depth, momenta, k act/pass, g_z and the centres or sizes) are copied, for the
// tile's 256 cells and its halo (the outside cells they name as neighbours, at most kHaloMax),
// into a shared-memory buffer by asynchronous copies (cp.async) one tile ahead: while the block
// computes tile q, the copies of tile q + 1 and the halo list of tile q + 2 are in flight.  The
// per-cell arithmetic is the global path's (the same helpers through StagedView), so results are
// identical; only where the operands come from changes.  Each cell's neighbour entries come from
// the host-built table of tile-local slots (one 16-byte load per cell).
//
// Activity: a cell is updated when it or a face neighbour is wet.  The global path marks every
// neighbour of a wet cell in the active bitmask with atomics; here the update phase recomputes
// that set from the staged depths of the tile and its halo, and the coefficient phase only marks
// neighbours in other tiles (and each warp's own wet cells), which the tile listing needs.
#pragma once

namespace da {
namespace fwd {
namespace {

constexpr int kSlots = kTileCells + kHaloMax;  // slot s < 256: cell 256 t + s; 256 + k: halo cell k

template <class R>
struct StageBuf {
    // the tile's own cells
    uint4 nl[kTileCells];                      // neighbour slots (8 x int16)
    uint8_t bf[kTileCells], mat[kTileCells];   // boundary flags, material
    R sz[2][sizeof(R) == 8 ? kTileCells : 1];  // FP64: dx, dy (FP32: c0, c1 below)
    R src[6][kTileCells];                      // update phase: g_x, g_y, the gravity derivatives, curvatures
    // every slot
    R h[kSlots], hu[kSlots], hv[kSlots];
    R k[kSlots];   // k act/pass (update phase)
    R gz[kSlots];  // g_z
    R c0[kSlots];  // FP64: x centre; FP32: dx
    R c1[kSlots];  // FP64: y centre; FP32: dy
};

template <class R>
struct StageSmem {
    StageBuf<R> buf[2];
    int hidx[3][kHaloMax];  // halo cells of three tiles in flight
    int hoff[kTileCells];   // halo range of each listed tile of the round
    int hcnt[kTileCells];
};

template <class R>
constexpr size_t stage_smem_bytes() {
    return sizeof(StageSmem<R>);
}

struct HaloArgs {
    const int32_t *off;   // [ntiles + 1]
    const int32_t *idx;   // halo cells, tile after tile
    const int16_t *nloc;  // [n][8] tile-local neighbour slots
    void *slopes;         // [6][n] reals: the limited slopes of each wet cell (h > GEOFLOW_TINY), written
                          // by the coefficient phase and read by the same step's update phase
};

inline HaloArgs halo_args(const da_ctx *ctx) {
    return HaloArgs{ctx->mesh.halo_off, ctx->mesh.halo_idx, ctx->mesh.nloc, ctx->slopes};
}

// The staged phases run when the parameters ask for them, the mesh's halo tables exist and the
// slopes are kept (the staged update of the forward step reads them instead of staging the centres).
inline bool staged_ok(const da_ctx *ctx) {
    return ctx->p.tile_staging >= 1 && ctx->mesh.nloc != nullptr && ctx->slopes != nullptr;
}

// cp.async of BYTES (4 or 8) from global to shared memory; completes at the group's wait.
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <class R>
struct StagedView {
    const StageBuf<R> &b;
    int nl[8];  // the cell's neighbour slots
    __device__ __forceinline__ int nb(int s, int) const { return nl[s]; }
    __device__ __forceinline__ R h(int e) const { return b.h[e]; }
    __device__ __forceinline__ R hu(int e) const { return b.hu[e]; }
    __device__ __forceinline__ R hv(int e) const { return b.hv[e]; }
    __device__ __forceinline__ R k(int e) const { return b.k[e]; }
    __device__ __forceinline__ R gz(int e) const { return b.gz[e]; }
    __device__ __forceinline__ double coord(int dir, int e) const { return double(dir == 0 ? b.c0[e] : b.c1[e]); }
    __device__ __forceinline__ float size(int dir, int e) const { return float(dir == 0 ? b.c0[e] : b.c1[e]); }
};

// The eight neighbour slots of cell i (one 16-byte load).
__device__ __forceinline__ void load_slots(const int16_t *nloc, int i, int nl[8]) {
    const uint4 w = *reinterpret_cast<const uint4 *>(nloc + (size_t)i * 8);
    const unsigned u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        nl[2 * q] = int(int16_t(u[q] & 0xffffu));
        nl[2 * q + 1] = int(int16_t(u[q] >> 16));
    }
}

// Copies of one slot's values.  UPD: also k act/pass and g_z (the update phase reads them at
// neighbours; the coefficient phase reads g_z at the cell itself only).  XY (FP64): the centres,
// which only the limited slopes read (the coefficient phase, and the reverse step's source
// adjoint inside its update phase).
template <class R, bool UPD, bool XY = true>
__device__ __forceinline__ void stage_slot(StageBuf<R> &b, int s, int e, bool own, const MeshArgs &m,
                                           const StateRef<R> &U, const R *kact) {
    constexpr int B = sizeof(R);
    cp_async<B>(&b.h[s], U.h + e);
    cp_async<B>(&b.hu[s], U.hu + e);
    cp_async<B>(&b.hv[s], U.hv + e);
    if (UPD) cp_async<B>(&b.k[s], kact + e);
    if constexpr (sizeof(R) == 8) {
        if (UPD || own) cp_async<B>(&b.gz[s], m.g + (size_t)2 * m.n + e);
        if (XY) {
            cp_async<B>(&b.c0[s], m.x + e);
            cp_async<B>(&b.c1[s], m.y + e);
        }
    } else {
        if (UPD || own) cp_async<B>(&b.gz[s], m.fg + (size_t)2 * m.n + e);
        cp_async<B>(&b.c0[s], m.fdx + e);
        cp_async<B>(&b.c1[s], m.fdy + e);
    }
}

// What only the tile's own cells need: neighbour slots, sizes (FP64), source coefficients (UPD),
// and the tile's flag and material bytes in 16-byte pieces (the byte arrays are padded to tiles).
template <class R, bool UPD>
__device__ __forceinline__ void stage_own(StageBuf<R> &b, int t, const MeshArgs &m, const int16_t *nloc) {
    constexpr int B = sizeof(R);
    const int c = threadIdx.x;
    const int i = t * kTileCells + c;
    if (i < m.n) {
        cp_async<16>(&b.nl[c], nloc + (size_t)i * 8);
        if constexpr (sizeof(R) == 8) {
            cp_async<8>(&b.sz[0][c], m.dx + i);
            cp_async<8>(&b.sz[1][c], m.dy + i);
        }
        if (UPD) {
            const R *g = sizeof(R) == 8 ? (const R *)m.g : (const R *)m.fg;
            const R *dg = sizeof(R) == 8 ? (const R *)m.dg : (const R *)m.fdg;
            const R *cv = sizeof(R) == 8 ? (const R *)m.curv : (const R *)m.fcurv;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                cp_async<B>(&b.src[q][c], g + (size_t)q * m.n + i);
                cp_async<B>(&b.src[2 + q][c], dg + (size_t)q * m.n + i);
                cp_async<B>(&b.src[4 + q][c], cv + (size_t)q * m.n + i);
            }
        }
    }
    if (c < kTileCells / 16)
        cp_async<16>(&b.bf[16 * c], m.bflag + (size_t)t * kTileCells + 16 * c);
    else if (c < kTileCells / 8)
        cp_async<16>(&b.mat[16 * (c - kTileCells / 16)], m.mat + (size_t)t * kTileCells + 16 * (c - kTileCells / 16));
}

// The staged source coefficients of own cell c.
template <class R>
__device__ __forceinline__ CellSrc<R> staged_src(const StageBuf<R> &b, int c) {
    CellSrc<R> s;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        s.g[q] = b.src[q][c];
        s.dg[q] = b.src[2 + q][c];
        s.cv[q] = b.src[4 + q][c];
    }
    s.mat = b.mat[c];
    return s;
}

// The eight neighbour slots of own cell c from the staged table.
template <class R>
__device__ __forceinline__ void staged_slots(const StageBuf<R> &b, int c, int nl[8]) {
    const uint4 w = b.nl[c];
    const unsigned u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        nl[2 * q] = int(int16_t(u[q] & 0xffffu));
        nl[2 * q + 1] = int(int16_t(u[q] >> 16));
    }
}

// Tile t's own cells and its halo (halo list already in shared memory) into buffer b.
template <class R, bool UPD, bool XY = true>
__device__ __forceinline__ void stage_tile(StageBuf<R> &b, int t, const int *hidx, int hcnt, const MeshArgs &m,
                                           const StateRef<R> &U, const R *kact, const int16_t *nloc) {
    const int i = t * kTileCells + (int)threadIdx.x;
    if (i < m.n) stage_slot<R, UPD, XY>(b, threadIdx.x, i, true, m, U, kact);
    stage_own<R, UPD>(b, t, m, nloc);
    for (int k = threadIdx.x; k < hcnt; k += kTileCells)
        stage_slot<R, UPD, XY>(b, kTileCells + k, hidx[k], false, m, U, kact);
}

__device__ __forceinline__ void stage_halo_list(int *dst, const int32_t *src, int cnt) {
    for (int k = threadIdx.x; k < cnt; k += kTileCells) cp_async<4>(dst + k, src + k);
}

// The halo range of tile tq (or nothing past the last tile), loaded beside its flags by the scan
// and kept with the tile by compact_tiles.
__device__ __forceinline__ void halo_range(const HaloArgs &ha, int tq, int ntiles, int &off, int &cnt) {
    off = 0;
    cnt = 0;
    if (tq < ntiles) {
        off = ha.off[tq];
        cnt = ha.off[tq + 1] - off;
    }
}

// The listed tiles of a round, pipelined: fn(t, buffer, halo list) computes tile t from shared
// memory.  Needs blockDim.x == kTileCells; every thread of the block calls it with the same cnt;
// S.hoff / S.hcnt hold the listed tiles' halo ranges (compact_tiles).  The first tile's halo
// cells are read by the threads that copy them; later tiles' lists arrive two tiles ahead.
template <class R, bool UPD, bool XY = true, class F>
__device__ __forceinline__ void staged_tiles(const MeshArgs &m, const HaloArgs &ha, const StateRef<R> &U,
                                             const R *kact, int cnt, const int *list, StageSmem<R> &S, F &&fn) {
    {
        const int t0 = list[0], hc = S.hcnt[0];
        const int32_t *src = ha.idx + S.hoff[0];
        const int i = t0 * kTileCells + (int)threadIdx.x;
        if (i < m.n) stage_slot<R, UPD, XY>(S.buf[0], threadIdx.x, i, true, m, U, kact);
        stage_own<R, UPD>(S.buf[0], t0, m, ha.nloc);
        for (int k = threadIdx.x; k < hc; k += kTileCells) {
            const int e = src[k];
            S.hidx[0][k] = e;
            stage_slot<R, UPD, XY>(S.buf[0], kTileCells + k, e, false, m, U, kact);
        }
    }
    if (cnt > 1) stage_halo_list(S.hidx[1], ha.idx + S.hoff[1], S.hcnt[1]);
    cp_async_commit();
    for (int q = 0; q < cnt; ++q) {
        // tile q's values and tile q + 1's halo list have landed; every thread is past tile q - 1
        cp_async_wait_all();
        __syncthreads();
        if (q + 1 < cnt) {
            stage_tile<R, UPD, XY>(S.buf[(q + 1) & 1], list[q + 1], S.hidx[(q + 1) % 3], S.hcnt[q + 1], m, U,
                                   kact, ha.nloc);
            if (q + 2 < cnt) stage_halo_list(S.hidx[(q + 2) % 3], ha.idx + S.hoff[q + 2], S.hcnt[q + 2]);
        }
        cp_async_commit();
        fn(list[q], S.buf[q & 1], S.hidx[q % 3]);
    }
    __syncthreads();
}

// Coefficient phase (see coef_phase) with the tile and its halo staged.
template <class R, bool RECORD, bool BATCH = false>
__device__ __forceinline__ void coef_phase_staged(const MeshArgs &m, const HaloArgs &ha, const StateRef<R> &U,
                                                  R *kact, unsigned *active, const uint8_t *seg_wet, int ntiles,
                                                  int cull, const MatConsts &mc0, DevScalars *sc, uint8_t *mask,
                                                  int *list, unsigned long long &my_min, unsigned long long &my_max,
                                                  const InstArgs &ia, StageSmem<R> &S) {
    for (int round = 0; sched_more(round, ntiles); ++round) {
        const int tq = sched_tile(round);
        const bool need = tq < ntiles && (!cull || seg_flags(seg_wet, tq) != 0ull);
        int ho, hc;
        halo_range(ha, tq, ntiles, ho, hc);
        const int cnt = compact_tiles(need, tq, list, ho, hc, S.hoff, S.hcnt);
        if (cnt == 0) continue;
        staged_tiles<R, false>(m, ha, U, kact, cnt, list, S, [&](int t, const StageBuf<R> &b, const int *hidx) {
            const int inst = BATCH ? ia.tile_inst[t] : 0;
            const MatConsts &mc = BATCH ? ia.mcs[inst] : mc0;
            const int c = threadIdx.x;
            const int i = t * kTileCells + c;
            bool wet = false;
            if (i < m.n) {
                const R h = b.h[c];
                if (!(h == h)) raise_err(sc, DA_ERR_NAN);
                wet = h >= R(DA_TINY);
                uint8_t code = 0;
                if (wet) {
                    const uint8_t bf = b.bf[c];
                    const int mat = b.mat[c];
                    R dxm, dym;
                    if constexpr (sizeof(R) == 8) {
                        dxm = b.sz[0][c];
                        dym = b.sz[1][c];
                    } else {
                        dxm = b.c0[c];
                        dym = b.c1[c];
                    }
                    StagedView<R> v{b};
                    staged_slots(b, c, v.nl);
                    // neighbours in other tiles: mark them for the tile listing of the update
#pragma unroll
                    for (int s = 0; s < 4; ++s) {
                        if (bf & (1 << s)) continue;
                        const int ne = (bf & (0x10 << s)) ? 2 : 1;
                        for (int q = 0; q < ne; ++q) {
                            const int sl = v.nl[s + 4 * q];
                            if (sl >= kTileCells) {
                                const int e = hidx[sl - kTileCells];
                                atomicOr(&active[e >> 5], 1u << (e & 31));
                            }
                        }
                    }
                    if (!(h > R(DA_TINY))) {  // h == GEOFLOW_TINY: dry for get_coef_and_eigen, wet for the fluxes
                        kact[i] = R(mc.kact_rest);
                    } else {
                        const R ui[3] = {h, b.hu[c], b.hv[c]};
                        R s[6];
                        cell_slopes<R>(v, c, bf, R(mc.gamma), ui, s);
                        if (ha.slopes) {  // kept for the update phase's source terms
                            R *sl = (R *)ha.slopes;
#pragma unroll
                            for (int j = 0; j < 6; ++j) sl[(size_t)j * m.n + i] = s[j];
                        }
                        const R k = cell_kact<R>(mc, mat, h, ui[1], ui[2], s, &code);
                        kact[i] = k;
                        const R gz = b.gz[c];
                        const R vx = ui[1] / h, vy = ui[2] / h;
                        const R cc = sqrt(k * gz * h);
                        const R evx = dabs(vx) + cc, evy = dabs(vy) + cc;
                        const R ev = evx > evy ? evx : evy;
                        if (ev > R(1000000000.)) raise_err(sc, DA_ERR_EIGEN);
                        const unsigned long long rb = __double_as_longlong(double((dxm > dym ? dym : dxm) / ev));
                        const unsigned long long hb = __double_as_longlong(double(h));
                        my_min = rb < my_min ? rb : my_min;
                        my_max = hb > my_max ? hb : my_max;
                    }
                }
                if (RECORD) mask[i] = code;
            }
            const unsigned self = __ballot_sync(0xffffffffu, wet);
            if (self && (threadIdx.x & 31) == 0) atomicOr(&active[i >> 5], self);
            if (BATCH) {
                push_minmax(my_min, my_max, ia.acc_min + inst, ia.acc_max + inst);
                my_min = 0x7FF0000000000000ull;
                my_max = 0ull;
            }
        });
    }
}

// No per-cell epilogue.
struct NoEpilogue {
    struct Pre {};
    __device__ __forceinline__ Pre pre(int, bool) const { return Pre{}; }
    template <class... A>
    __device__ __forceinline__ void operator()(A &&...) const {}
};

// Update phase (see update_phase) with the tile and its halo staged.  A listed tile's cells
// recompute their activity from the staged depths; the segment flags follow it.
// epi(t, i, v, c, prev, bf, code, gz, cs, pre, f) runs for every wet cell i of a listed tile t inside
// its update, where the corrector has formed the source terms' slopes, velocities and friction
// signs f (the reverse step's source adjoint, which needs exactly these), with the staged view v
// of the cell (slot c), its U^n, boundary flags, recorded branch byte, g_z and source coefficients,
// and what epi.pre(i, wet) loaded before the update (so that those loads overlap it).
template <class R, bool RECORD, bool BATCH = false, class Epi = NoEpilogue>
__device__ __forceinline__ void update_phase_staged(const MeshArgs &m, const HaloArgs &ha, const StateRef<R> &U,
                                                    const StateOut<R> &O, const R *kact, unsigned *active,
                                                    uint8_t *seg_clean, uint8_t *seg_wet, double *seg_vol,
                                                    uint8_t *seg_dirty, int ntiles, int cull, const MatConsts &mc0,
                                                    DevScalars *sc, R dt0, R ft, uint8_t *mask, int *tile_epoch,
                                                    uint8_t *seg_act, int rec_id, int *list, const InstArgs &ia,
                                                    StageSmem<R> &S, const Epi &epi = Epi{}) {
    const int lane = threadIdx.x & 31;
    for (int round = 0; sched_more(round, ntiles); ++round) {
        const int tq = sched_tile(round);
        bool need = false;
        if (tq < ntiles) {
            // the clean flags and the bitmask words of the tile, loaded together
            const unsigned long long cf = seg_flags(seg_clean, tq);
            const uint4 *w4 = reinterpret_cast<const uint4 *>(active + (size_t)tq * (kTileCells / 32));
            const uint4 a = w4[0], b = w4[1];
            need = !cull || cf != kAllSegs || (a.x | a.y | a.z | a.w | b.x | b.y | b.z | b.w) != 0u;
        }
        int ho, hc;
        halo_range(ha, tq, ntiles, ho, hc);
        const int cnt = compact_tiles(need, tq, list, ho, hc, S.hoff, S.hcnt);
        if (cnt == 0) continue;
        if (RECORD && threadIdx.x == 0) atomicAdd(&sc->listed, (unsigned)cnt);
        // the centres only for an epilogue (the source adjoint's slope derivatives read them); the
        // update itself takes the kept slopes
        constexpr bool XY = !std::is_same<Epi, NoEpilogue>::value;
        staged_tiles<R, true, XY>(m, ha, U, kact, cnt, list, S, [&](int t, const StageBuf<R> &b, const int *) {
            const int inst = BATCH ? ia.tile_inst[t] : 0;
            const MatConsts &mc = BATCH ? ia.mcs[inst] : mc0;
            const R dt = BATCH ? R(ia.dt[inst]) : dt0;
            const int c = threadIdx.x;
            const int i = t * kTileCells + c;
            const int seg = i >> 5;
            const unsigned word = active[seg];  // marks to clear (padded: bits of cells >= n never set)
            double vol = 0.0;
            bool wet_after = false, act = false;
            if (i < m.n) {
                const R prev[3] = {b.h[c], b.hu[c], b.hv[c]};
                // the slopes this step's coefficient phase left for a wet cell, loaded ahead of the fluxes
                const bool own_s = ha.slopes != nullptr && prev[0] > R(DA_TINY);
                R pre_s[6];
                if (own_s) {
                    const R *sl = (const R *)ha.slopes;
#pragma unroll
                    for (int j = 0; j < 6; ++j) pre_s[j] = sl[(size_t)j * m.n + i];
                }
                const auto pre = epi.pre(i, prev[0] > R(DA_TINY));
                const uint8_t bf = b.bf[c];
                StagedView<R> v{b};
                staged_slots(b, c, v.nl);
                act = prev[0] >= R(DA_TINY);
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    if (bf & (1 << s)) continue;
                    act |= b.h[v.nl[s]] >= R(DA_TINY);
                    if (bf & (0x10 << s)) act |= b.h[v.nl[s + 4]] >= R(DA_TINY);
                }
                R dxc, dyc;
                if constexpr (sizeof(R) == 8) {
                    dxc = b.sz[0][c];
                    dyc = b.sz[1][c];
                } else {
                    dxc = b.c0[c];
                    dyc = b.c1[c];
                }
                R st[3] = {prev[0], prev[1], prev[2]};
                bool clamped = false;
                const CellSrc<R> cs = staged_src(b, c);
                // the k act/pass code the coefficient phase recorded
                const uint8_t kcode = RECORD && prev[0] >= R(DA_TINY) ? uint8_t(mask[i] & 3) : uint8_t(0);
                if (act)
                    clamped = update_cell<R>(v, c, bf, cs, mc, dt, ft, prev, dxc, dyc, st, own_s ? pre_s : nullptr,
                                             [&](const SrcFwd<R> &f, bool cl) {
                                                 // a wet cell is active: its branch byte as recorded below
                                                 epi(t, i, v, c, prev, bf, uint8_t(kcode | 8 | (cl ? 4 : 0)), b.gz[c],
                                                     cs, pre, f);
                                             });
                const uint8_t code = RECORD ? uint8_t(kcode | (act ? 8 : 0) | (clamped ? 4 : 0)) : 0;
                if (RECORD) mask[i] = code;
                if (!isfinite(st[0]) || !isfinite(st[1]) || !isfinite(st[2])) raise_err(sc, DA_ERR_NAN);
                O.h[i] = st[0];
                O.hu[i] = st[1];
                O.hv[i] = st[2];
                vol = double(dxc) * double(dyc) * double(st[0]);
                wet_after = st[0] >= R(DA_TINY);
            }
            const unsigned wet_bits = __ballot_sync(0xffffffffu, wet_after);
            const unsigned act_bits = __ballot_sync(0xffffffffu, act);
            vol = warp_sum(vol);
            if (lane == 0) {
                if (word) active[seg] = 0u;
                if (act_bits) seg_dirty[seg] = 1;  // changed since the base checkpoint
                seg_vol[seg] = vol;
                seg_clean[seg] = act_bits ? 0 : 1;
                seg_wet[seg] = wet_bits ? 1 : 0;
                if (RECORD) seg_act[seg] = act_bits ? 1 : 0;
            }
            if (RECORD && threadIdx.x == 0) tile_epoch[t] = rec_id;
        });
    }
}

}  // namespace
}  // namespace fwd
}  // namespace da
