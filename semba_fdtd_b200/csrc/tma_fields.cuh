// TMA-pipelined curl + CPML kernels (the fused fast path of the E and H half
// steps) and their persistent batched form.  Included by kernels.cu and
// batch.cu; the per-cell helpers come from stencil.cuh.
//
// Each CTA owns a 32 x 8 tile of (i, j) columns and marches a z chunk.  One
// producer warp streams every plane the tile needs -- the H (or E) tiles with
// their one-cell halos, the tile's own E (or H) values and the three media
// tiles (one byte a cell, a copy of the int16 matrices kept while the media
// number under 256) -- into a 3-stage shared-memory ring with cp.async.bulk.tensor
// loads that complete on mbarriers; eight consumer warps update one cell per
// thread from shared memory and store the result with plain coalesced stores.
// The x origin of a haloed tile is rounded down to a 16-byte boundary (4
// floats), so a TMA box never starts on an unaligned x coordinate.  Every
// mbarrier wait is bounded by a clock budget: on expiry the kernel records
// an error code in dev_err and leaves the loop; the producer then waits, again
// bounded, for the loads it has in flight before the CTA exits.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "stencil.cuh"

namespace sgpu {
using namespace sgpu::dev;

constexpr int kTX = 32, kTY = 8;          // tile (threads per row, rows)
#ifndef SGPU_TMA_STAGES
#define SGPU_TMA_STAGES 3
#endif
#ifndef SGPU_PSI_SLOTS
#define SGPU_PSI_SLOTS 6
#endif
constexpr int kStages = SGPU_TMA_STAGES;  // shared-memory ring depth
constexpr int kConsumerWarps = kTY;       // one warp per tile row
constexpr int kTmaThreads = (kConsumerWarps + 1) * 32;
constexpr int kHaloW = kTX + 4;           // haloed row width (x rounded to 16 B)
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at the B200 clock

// byte sizes of the boxes and their 128-byte aligned slots in a stage
constexpr int kBoxA = kTX * (kTY + 1) * 4;      // 32 x 9 floats
constexpr int kBoxB = kHaloW * kTY * 4;         // 36 x 8 floats
constexpr int kBoxC = kHaloW * (kTY + 1) * 4;   // 36 x 9 floats
constexpr int kBoxF = kTX * kTY * 4;            // 32 x 8 floats
constexpr int kBoxM = kTX * kTY;                // 32 x 8 one-byte media indices
constexpr int kBoxP = kTX * kTY * 4;            // 32 x 8 floats of one psi slab
constexpr int kPsiSlots = SGPU_PSI_SLOTS;       // psi tiles staged per plane
__host__ __device__ constexpr int align128(int b) { return (b + 127) / 128 * 128; }
constexpr int kOffA = 0;
constexpr int kOffB = kOffA + align128(kBoxA);
constexpr int kOffC = kOffB + align128(kBoxB);
constexpr int kOffF = kOffC + align128(kBoxC);
constexpr int kOffM = kOffF + 3 * align128(kBoxF);
constexpr int kOffP = kOffM + 3 * align128(kBoxM);
constexpr int kOffW = kOffP + kPsiSlots * align128(kBoxP);
constexpr int kStageBytes = kOffW + 128;
constexpr int kPsiSlotFloats = align128(kBoxP) / 4;
constexpr int kPsiMap0 = 9;  // first psi map in TMaps
constexpr int kTmaSmem = kStages * kStageBytes + 2 * kStages * 8;
constexpr unsigned kTxFull = kBoxA + kBoxB + kBoxC + 3 * kBoxF + 3 * kBoxM;
constexpr unsigned kTxEdge = kBoxA + kBoxB;  // the extra plane: two arrays only

// TMaps holds the tensor maps in the order the kernels use them:
//   E kernel: Hx(32x9) Hy(36x8) Hz(36x9) Ex Ey Ez (32x8) Mx My Mz (32x8 one-byte media)
//   H kernel: Ex(32x9) Ey(36x8) Ez(36x9) Hx Hy Hz (32x8) Mx My Mz (32x8 one-byte media)
// then the psi slabs of the side (32x8), map 9+n for slab bit n of the
// CPML masks (cp.s[c0 + n/4][(n/2)%2][n%2]).
//
// Each full plane also carries four words the producer lane writes before
// it arrives on the stage's barrier: the slabs of the tile that hold the
// plane, the plane's inverse z step and its z-indexed P_b / P_c pair, so the
// consumers make no global load in the plane loop.
//
// CPML tiles whose slabs (cpml_tile_mask) number at most kPsiSlots also get
// their psi tiles through the ring: a stage carries, after the media, one
// 32x8 psi tile per slab that holds the plane, in the slot given by the
// slab's rank in the tile mask.  The consumers read the old psi from there
// and store the new value with a plain store.  Tiles with more slabs (narrow
// grids where both sides of an axis fall in one tile) read psi from global
// memory.

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned a, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned a, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned a) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned a, unsigned parity) {
    unsigned done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait; false (and an error code in *err) when `budget` clock
// cycles run out.
__device__ __forceinline__ bool mbar_wait(unsigned a, unsigned parity, int* err, int code, long long budget) {
    const long long t0 = clock64();
    while (!mbar_try(a, parity)) {
        if (clock64() - t0 > budget) {
            atomicExch(err, code);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void tma_load3(unsigned dst, const CUtensorMap* map, int x, int y, int z, unsigned mbar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(mbar)
        : "memory");
}

struct PlaneWords {
    unsigned live;  // bits of the tile mask whose slab holds the plane
    float idz;      // Idzh(k) (E side) or Idze(k) (H side)
    float bz, cz;   // P_be/P_ce (E) or P_bm/P_cm (H) at k, when a z slab holds it
};

// Shared set-up of the two kernels: barriers, coefficient tables, geometry.
struct TmaCta {
    unsigned char* ring;
    unsigned full0, empty0;  // shared addresses of the barrier arrays
    int ib, jb, kb, ke;
    int warp, lane;
    long long wait;  // budget of a pipeline wait (consumers and the producer's
                     // wait for a free stage); the final drain keeps kWaitCycles
};

__device__ __forceinline__ TmaCta tma_cta_setup(unsigned char* smem, int y0, int z0, int z1, int zchunk,
                                                long long wait) {
    TmaCta t;
    t.ring = smem;
    t.wait = wait;
    unsigned long long* bars = (unsigned long long*)(smem + kStages * kStageBytes);
    t.full0 = smem_u32(bars);
    t.empty0 = smem_u32(bars + kStages);
    t.ib = blockIdx.x * kTX;
    t.jb = y0 + blockIdx.y * kTY;
    t.kb = z0 + blockIdx.z * zchunk;
    t.ke = min(t.kb + zchunk - 1, z1);
    t.warp = threadIdx.x >> 5;
    t.lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(t.full0 + 8 * s, 1);
            mbar_init(t.empty0 + 8 * s, kConsumerWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    return t;
}

// The producer's per-item table: the four plane words of every plane of the
// item and the psi TMA coordinates of every slab of the tile, prepared by the
// whole producer warp before lane 0 issues the item, so lane 0's plane loop
// makes no global (or parameter) load between two barrier operations.
constexpr int kMaxItemPlanes = 72;  // z chunk + 1; chunks are at most 64 planes
struct ProdTable {
    PlaneWords w[kMaxItemPlanes];
    int4 psi[12];  // per slab bit: x origin (ib - xb), y origin (jb - ylo), zlo
};

// Producer warp, all lanes: planes p0 .. p1 (edge excluded) of one item.
// `tmask` is the CPML tile's slab mask (0 for a bulk tile).
__device__ __forceinline__ void prod_prepare(ProdTable* tb, const TmaCta& t, int p0, int p1, int edge, bool hside,
                                             const KGrid& g, const KCpml& cp, unsigned tmask) {
    const int c0 = hside ? 3 : 0;
    const float* idz = hside ? g.idze : g.idzh;
    const float* pb = hside ? cp.pbm[2] : cp.pbe[2];
    const float* pc = hside ? cp.pcm[2] : cp.pce[2];
    for (int p = p0 + t.lane; p <= p1; p += 32) {
        PlaneWords w{0u, 0.0f, 0.0f, 0.0f};
        if (p != edge) {
            w.live = tmask ? cpml_plane_mask(cp, c0, tmask, p) : 0u;
            w.idz = idz[p];
            if (w.live & kCpmlZ) {
                w.bz = pb[p];
                w.cz = pc[p];
            }
        }
        tb->w[p - p0] = w;
    }
    if (t.lane < 12 && ((tmask >> t.lane) & 1u)) {
        const Slab& sl = cp.s[c0 + (t.lane >> 2)][(t.lane >> 1) & 1][t.lane & 1];
        tb->psi[t.lane] = make_int4(t.ib - sl.xb, t.jb - sl.ylo, sl.zlo, 0);
    }
    __syncwarp();
}

// The persistent producer's table holds the plane words of a window of 32
// planes of the item (refilled by the warp as the issue loop reaches it), so
// an item may have any number of planes, and the psi coordinates.
struct ProdWindow {
    PlaneWords w[32];
    int4 psi[12];
    int2 zr[12];  // z range of each slab of the tile mask (empty for the others)
};
struct PlaneSource {  // what the window refill reads
    const KGrid* g;
    const KCpml* cp;
    unsigned tmask;
};
// Producer warp, all lanes: the words of the planes m0 .. m0+31 of the
// item's issue order (p = p0 + m upwards, p1 - m downwards on the H side).
// The slabs' z ranges come from the table prod_psi filled, so a refill reads
// only the plane's own metric and CPML values from global memory.
__device__ __forceinline__ void prod_window(ProdWindow* tb, const TmaCta& t, int m0, int p0, int p1, int edge, bool hside,
                                            const PlaneSource& src) {
    const KGrid& g = *src.g;
    const KCpml& cp = *src.cp;
    const int m = m0 + t.lane;
    __syncwarp();  // every lane has read the previous window
    if (m <= p1 - p0) {
        const int p = hside ? p1 - m : p0 + m;
        PlaneWords w{0u, 0.0f, 0.0f, 0.0f};
        if (p != edge) {
            unsigned live = 0;
            if (src.tmask) {
#pragma unroll
                for (int n = 0; n < 12; ++n) {
                    const int2 z = tb->zr[n];
                    if (p >= z.x && p <= z.y) live |= 1u << n;
                }
            }
            w.live = live;
            w.idz = (hside ? g.idze : g.idzh)[p];
            if (live & kCpmlZ) {
                w.bz = (hside ? cp.pbm[2] : cp.pbe[2])[p];
                w.cz = (hside ? cp.pcm[2] : cp.pce[2])[p];
            }
        }
        tb->w[t.lane] = w;
    }
    __syncwarp();
}
// Producer warp, all lanes, once per item: the psi TMA coordinates and the z
// range of every slab of the tile mask.
__device__ __forceinline__ void prod_psi(ProdWindow* tb, const TmaCta& t, bool hside, const KCpml& cp, unsigned tmask) {
    const int c0 = hside ? 3 : 0;
    if (t.lane < 12) {
        int2 z = make_int2(1, 0);
        if ((tmask >> t.lane) & 1u) {
            const Slab& sl = cp.s[c0 + (t.lane >> 2)][(t.lane >> 1) & 1][t.lane & 1];
            tb->psi[t.lane] = make_int4(t.ib - sl.xb, t.jb - sl.ylo, sl.zlo, 0);
            z = make_int2(sl.zlo, sl.zhi);
        }
        tb->zr[t.lane] = z;
    }
    __syncwarp();
}

// Producer (lane 0 of the producer warp): planes p0 .. p1 of one work item
// into the ring, upwards on the E side and downwards on the H side, so that
// either side's edge plane comes first; the item's first plane has the
// running plane number G0 (a plane lands in stage G % kStages; its n-th use
// of that stage is phase n).
// `edge` is the plane that carries only the first two arrays (the E side's
// k-1 plane, the H side's k+1 plane).  Tile origins: E side Hx (ib, jb-1),
// Hy (ib-4, jb), Hz (ib-4, jb-1), own fields and media (ib, jb); H side all
// at (ib, jb).  Returns the number of planes issued: fewer than p1-p0+1 when
// a bounded wait ran out.
//
// `smask` is the staged slab mask (the tile mask or 0): every full plane
// brings the psi tile of each slab of smask that holds it.  The plane words
// and psi coordinates come from the table prod_prepare filled.
__device__ __forceinline__ int tma_issue(const TmaCta& t, const CUtensorMap* maps, unsigned G0, int p0, int p1, int edge,
                                         bool hside, int* err, const ProdTable* tb, unsigned smask) {
    for (int n = 0; n <= p1 - p0; ++n) {
        const int p = hside ? p1 - n : p0 + n;  // the H side marches down
        const unsigned G = G0 + (unsigned)n, s = G % kStages, u = G / kStages;
        const PlaneWords w = tb->w[p - p0];
        if (u >= 1 && !mbar_wait(t.empty0 + 8 * s, (u - 1) & 1, err, hside ? 13 : 11, t.wait)) return n;
        const unsigned bar = t.full0 + 8 * s;
        unsigned char* st = t.ring + s * kStageBytes;
        const bool part = p == edge;
        unsigned live = w.live & smask;
        if (!part) *(PlaneWords*)(st + kOffW) = w;
        mbar_expect_tx(bar, (part ? kTxEdge : kTxFull) + (unsigned)__popc(live) * (unsigned)kBoxP);
        const int xh = hside ? t.ib : t.ib - 4, ya = hside ? t.jb : t.jb - 1;
        tma_load3(smem_u32(st + kOffA), &maps[0], t.ib, ya, p, bar);  // first array (halo in y)
        tma_load3(smem_u32(st + kOffB), &maps[1], xh, t.jb, p, bar);  // second (halo in x)
        if (!part) {
            tma_load3(smem_u32(st + kOffC), &maps[2], xh, ya, p, bar);
            for (int q = 0; q < 3; ++q) tma_load3(smem_u32(st + kOffF + q * align128(kBoxF)), &maps[3 + q], t.ib, t.jb, p, bar);
            for (int q = 0; q < 3; ++q) tma_load3(smem_u32(st + kOffM + q * align128(kBoxM)), &maps[6 + q], t.ib, t.jb, p, bar);
        }
        while (live) {
            const int b = __ffs(live) - 1;
            live &= live - 1u;
            const int4 c = tb->psi[b];
            const int slot = psi_slot(smask, b);
            tma_load3(smem_u32(st + kOffP + slot * align128(kBoxP)), &maps[kPsiMap0 + b], c.x, c.y, p - c.z, bar);
        }
    }
    return p1 - p0 + 1;
}

// The same planes issued by the whole producer warp: lane 0 waits for the
// stage and arms its barrier, then lane q < 9 loads the box of map q (the
// three field arrays of the other side, the three own fields, the three
// media) and lane 9 + n the psi box of slab bit n when the plane holds that
// staged slab.  A lane is the only issuer of its map, so a tensor map that
// lane acquired through the tensormap proxy needs no other thread's fence.
// All lanes return the number of planes issued.
// The first plane of a work item also carries, after its PlaneWords, the item
// (`item`: its index, -1 marking the end of a CTA's items, then six words of
// the item itself), which is how the consumers of a dynamically scheduled
// persistent kernel learn their item without a global load.
constexpr int kOffItem = kOffW + (int)sizeof(PlaneWords);
struct ItemWords {
    int v[7];
};
static_assert(sizeof(PlaneWords) + sizeof(ItemWords) <= 128, "the plane words fit their stage slot");
__device__ __forceinline__ int tma_issue_warp(const TmaCta& t, const CUtensorMap* maps, unsigned G0, int p0, int p1,
                                              int edge, bool hside, int* err, ProdWindow* tb, const PlaneSource& src,
                                              unsigned smask, const ItemWords& item) {
    const int q = t.lane;
    const int xh = hside ? t.ib : t.ib - 4, ya = hside ? t.jb : t.jb - 1;
    // this lane's box: shared-memory offset, x and y origin, and z offset
    // (psi boxes count planes from their slab's zlo)
    int off = 0, bx = t.ib, by = t.jb, bz0 = 0;
    if (q == 0) { off = kOffA; by = ya; }
    else if (q == 1) { off = kOffB; bx = xh; }
    else if (q == 2) { off = kOffC; bx = xh; by = ya; }
    else if (q < 6) off = kOffF + (q - 3) * align128(kBoxF);
    else if (q < 9) off = kOffM + (q - 6) * align128(kBoxM);
    const int n = q - kPsiMap0;
    const bool psi_lane = n >= 0 && n < 12 && ((smask >> n) & 1u);
    if (psi_lane) {
        const int4 pc = tb->psi[n];
        off = kOffP + psi_slot(smask, n) * align128(kBoxP);
        bx = pc.x;
        by = pc.y;
        bz0 = pc.z;
    }
    const CUtensorMap* map = &maps[q < kPsiMap0 + 12 ? q : 0];
    for (int m = 0; m <= p1 - p0; ++m) {
        const int p = hside ? p1 - m : p0 + m;  // the H side marches down
        const unsigned G = G0 + (unsigned)m, s = G % kStages, u = G / kStages;
        const unsigned bar = t.full0 + 8 * s;
        unsigned char* st = t.ring + s * kStageBytes;
        const bool part = p == edge;
        if ((m & 31) == 0) prod_window(tb, t, m, p0, p1, edge, hside, src);
        const PlaneWords w = tb->w[m & 31];
        int ok = 1;
        if (q == 0) {
            if (u >= 1 && !mbar_wait(t.empty0 + 8 * s, (u - 1) & 1, err, hside ? 13 : 11, t.wait)) {
                ok = 0;
            } else {
                if (!part) *(PlaneWords*)(st + kOffW) = w;
                if (m == 0) *(ItemWords*)(st + kOffItem) = item;  // the consumers read it at the item's first plane
                mbar_expect_tx(bar, (part ? kTxEdge : kTxFull) + (unsigned)__popc(w.live & smask) * (unsigned)kBoxP);
            }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) return m;
        __syncwarp();  // the stage is free and armed before any lane writes into it
        const bool issue = q < kPsiMap0 ? (q < 2 || !part) : (psi_lane && ((w.live >> n) & 1u));
        if (issue) tma_load3(smem_u32(st + off), map, bx, by, p - bz0, bar);
    }
    return p1 - p0 + 1;
}

// The end of a CTA's items (producer lane 0): plane G carries item -1 and no
// loads; its full barrier completes on the plain arrive.  False when the wait
// for the free stage ran out.
__device__ __forceinline__ bool tma_publish_end(const TmaCta& t, unsigned G, int* err) {
    const unsigned s = G % kStages, u = G / kStages;
    if (u >= 1 && !mbar_wait(t.empty0 + 8 * s, (u - 1) & 1, err, 16, t.wait)) return false;
    *(int*)(t.ring + s * kStageBytes + kOffItem) = -1;
    mbar_arrive(t.full0 + 8 * s);
    return true;
}

// The slab mask whose psi tiles a CPML tile stages (0: psi from global
// memory): the tile's slabs when they need at most kPsiSlots slots and the
// two sides of each z pair they hold are apart in z (so they can share).
__device__ __forceinline__ unsigned staged_mask(const KCpml& cp, int c0, int ib, int jb) {
    const unsigned m = cpml_tile_mask(cp, c0, ib, ib + kTX - 1, jb, jb + kTY - 1);
    const bool apart = ((m & 0x0Cu) != 0x0Cu || cp.s[c0][1][0].zhi < cp.s[c0][1][1].zlo) &&
                       ((m & 0x30u) != 0x30u || cp.s[c0 + 1][0][0].zhi < cp.s[c0 + 1][0][1].zlo);
    return apart && __popc(psi_slot_groups(m)) <= kPsiSlots ? m : 0u;
}

// One CPML correction of a consumer: CP 2 takes the old psi from the staged
// tile, CP 1 from global memory.
template <int CP, bool ADD>
__device__ __forceinline__ float cpml_corr(const Slab (&s)[2], unsigned live2, int nbase, const float* slots,
                                           int o, const PsiRow* rows, int i, int j, int k, float pb, float pc, float diff,
                                           float g, float v, bool& st) {
    if (CP == 2) return cpml_pair_staged<ADD>(live2, nbase, slots, o, rows, o & 31, k, pb, pc, diff, g, v);
    return cpml_pair<ADD>(s, live2, i, j, k, pb, pc, diff, g, v, st);
}

// Nothing may be in flight into the CTA's shared memory when it exits: wait
// (bounded) for the last loads of the `issued` planes numbered 0..issued-1.
__device__ __forceinline__ void tma_drain(const TmaCta& t, unsigned issued, int* err, int code) {
    const unsigned first = issued > (unsigned)kStages ? issued - kStages : 0;
    for (unsigned G = first; G < issued; ++G)
        mbar_wait(t.full0 + 8 * (G % kStages), (G / kStages) & 1, err, code, kWaitCycles);
}

// Every lane waits on the barrier (each needs the acquire); the warp then
// agrees on the outcome so all lanes leave together on a timeout.  The usual
// case, a plane that has already landed, takes one test and one vote.
__device__ __forceinline__ bool warp_wait(unsigned bar, unsigned parity, int* err, int code, long long budget) {
    if (__all_sync(0xffffffffu, mbar_try(bar, parity))) return true;
    const bool ok = mbar_wait(bar, parity, err, code, budget);
    return __all_sync(0xffffffffu, ok);
}

__device__ __forceinline__ void warp_release(const TmaCta& t, unsigned G) {
    __syncwarp();
    if (t.lane == 0) mbar_arrive(t.empty0 + 8 * (G % kStages));
}

// The coefficient pair (G1, G2) -- or (GM1, GM2) -- of a medium: from a
// shared-memory table of pairs, or from the two global tables.
struct TabPairs {
    const float2* t;
    __device__ __forceinline__ float2 operator()(int m) const { return t[m]; }
};
struct TabSplit {
    const float* a;
    const float* b;
    __device__ __forceinline__ float2 operator()(int m) const { return make_float2(a[m], b[m]); }
};

// Consumers of the E side: Advance_Ex/Ey/Ez + AdvanceelectricCPML from the
// ring, the same per-cell arithmetic as efield_column.  The item's planes are
// G0 (k = kb-1, edge) and G0+1+(k-kb).  Hx and Hy of plane k-1 are carried
// in registers (the edge plane's, then the previous iteration's), so a plane
// is released as soon as it is done and the edge plane right after its two
// values are read; with `release_last` the item's last plane is released too
// (a persistent CTA goes on to another item).  False on a timeout.
template <int CP, class TAB>
__device__ __forceinline__ bool e_consume(const TmaCta& t, unsigned G0, const KGrid& g, const KCpml& cp, const TAB tab,
                                          int* err, bool release_last, PsiRow* rows) {
    const int w = t.warp, l = t.lane;
    const int i = t.ib + l, j = t.jb + w;
    const int nya = (int)(g.plane / g.pitch);
    const bool vx = col_in(g.sw[0], i, j), vy = col_in(g.sw[1], i, j), vz = col_in(g.sw[2], i, j);
    const float idyh = g.idyh[min(j, nya - 1)], idxh = g.idxh[i];
    const long long pitch = g.pitch, plane = g.plane;
    // the grid view may sit in shared memory (the batched kernel): what the
    // plane loop needs is read into registers once
    float* const F0 = g.F[0];
    float* const F1 = g.F[1];
    float* const F2 = g.F[2];
    const int kx0 = g.sw[0][4], kx1 = g.sw[0][5], ky0 = g.sw[1][4], ky1 = g.sw[1][5], kz0 = g.sw[2][4], kz1 = g.sw[2][5];
    const unsigned tmask = CP ? cpml_tile_mask(cp, 0, t.ib, t.ib + kTX - 1, t.jb, t.jb + kTY - 1) : 0u;
    const CpmlCol cc = CP ? cpml_col(cp, 0, tmask, i, j, t.kb, t.ke) : CpmlCol{};
    if (CP == 2) psi_rows_fill(rows, cp, 0, tmask, kPsiSlotFloats, t.ib, j, l);
    float hx_km, hy_km;
    {
        const unsigned sp = G0 % kStages;
        if (!warp_wait(t.full0 + 8 * sp, (G0 / kStages) & 1, err, 2, t.wait)) return false;
        const unsigned char* pv = t.ring + sp * kStageBytes;
        hx_km = ((const float*)(pv + kOffA))[(w + 1) * kTX + l];
        hy_km = ((const float*)(pv + kOffB))[w * kHaloW + l + 4];
        warp_release(t, G0);
    }
    long long c = i + pitch * j + plane * t.kb;
    for (int k = t.kb; k <= t.ke; ++k, c += plane) {
        const unsigned Gk = G0 + 1 + (unsigned)(k - t.kb);
        const unsigned s = Gk % kStages;
        if (!warp_wait(t.full0 + 8 * s, (Gk / kStages) & 1, err, 1, t.wait)) return false;
        const unsigned char* st = t.ring + s * kStageBytes;
        // slabs holding cell (i, j, k): the column's slabs that hold plane k;
        // the plane's Idzh and z-indexed P_b / P_c come with the plane
        const PlaneWords pw = *(const PlaneWords*)(st + kOffW);
        const unsigned pm = CP ? (cc.col & pw.live) : 0u;
        const float bz = pw.bz, cz = pw.cz;
        const float* HX = (const float*)(st + kOffA);
        const float* HY = (const float*)(st + kOffB);
        const float* HZ = (const float*)(st + kOffC);
        const float* EF = (const float*)(st + kOffF);
        const uint8_t* MF = (const uint8_t*)(st + kOffM);
        const float* PS = (const float*)(st + kOffP);
        constexpr int fs = align128(kBoxF) / 4, ms = align128(kBoxM);
        const float hx = HX[(w + 1) * kTX + l], hx_jm = HX[w * kTX + l];
        const float hy = HY[w * kHaloW + l + 4], hy_im = HY[w * kHaloW + l + 3];
        const float hz = HZ[(w + 1) * kHaloW + l + 4], hz_jm = HZ[w * kHaloW + l + 4], hz_im = HZ[(w + 1) * kHaloW + l + 3];
        const float idzh = pw.idz;
        const int o = w * kTX + l;
        bool st_ = true;
        if (vx && k >= kx0 && k <= kx1) {
            float e = EF[o];
            const float2 tt = tab(MF[o]);
            const float dy = hz - hz_jm, dz = hy - hy_km;
            e = tt.x * e + tt.y * (dy * idyh - dz * idzh);
            if (CP && pm) {
                e = cpml_corr<CP, true>(cp.s[0][0], pm & 3, 0, PS, o, rows, i, j, k, cc.by, cc.cy, dy, tt.y, e, st_);
                e = cpml_corr<CP, false>(cp.s[0][1], (pm >> 2) & 3, 2, PS, o, rows, i, j, k, bz, cz, dz, tt.y, e, st_);
            }
            F0[c] = e;
        }
        if (vy && k >= ky0 && k <= ky1) {
            float e = EF[fs + o];
            const float2 tt = tab(MF[ms + o]);
            const float dz = hx - hx_km, dx = hz - hz_im;
            e = tt.x * e + tt.y * (dz * idzh - dx * idxh);
            if (CP && pm) {
                e = cpml_corr<CP, true>(cp.s[1][0], (pm >> 4) & 3, 4, PS, o, rows, i, j, k, bz, cz, dz, tt.y, e, st_);
                e = cpml_corr<CP, false>(cp.s[1][1], (pm >> 6) & 3, 6, PS, o, rows, i, j, k, cc.bx, cc.cx, dx, tt.y, e, st_);
            }
            F1[c] = e;
        }
        if (vz && k >= kz0 && k <= kz1) {
            float e = EF[2 * fs + o];
            const float2 tt = tab(MF[2 * ms + o]);
            const float dx = hy - hy_im, dy = hx - hx_jm;
            e = tt.x * e + tt.y * (dx * idxh - dy * idyh);
            if (CP && pm) {
                e = cpml_corr<CP, false>(cp.s[2][0], (pm >> 8) & 3, 8, PS, o, rows, i, j, k, cc.by, cc.cy, dy, tt.y, e, st_);
                e = cpml_corr<CP, true>(cp.s[2][1], (pm >> 10) & 3, 10, PS, o, rows, i, j, k, cc.bx, cc.cx, dx, tt.y, e, st_);
            }
            F2[c] = e;
        }
        hx_km = hx;
        hy_km = hy;
        if (k < t.ke || release_last) warp_release(t, Gk);  // plane k is no longer needed
    }
    return true;
}

// Consumers of the H side: Advance_Hx/Hy/Hz + AdvanceMagneticCPML from the
// ring (hfield_column's arithmetic), marching down: the item's planes are G0
// (k = ke+1, edge) and G0+1+(ke-k).  Ex and Ey of plane k+1 are carried in
// registers (the edge plane's, then the previous iteration's), so a plane is
// released as soon as it is done and the edge plane right after its two
// values are read; with `release_last` the item's last plane is released too.
template <int CP, class TAB>
__device__ __forceinline__ bool h_consume(const TmaCta& t, unsigned G0, const KGrid& g, const KCpml& cp, const TAB tab,
                                          int* err, bool release_last, PsiRow* rows) {
    const int w = t.warp, l = t.lane;
    const int i = t.ib + l, j = t.jb + w;
    const int nya = (int)(g.plane / g.pitch);
    const bool vx = col_in(g.sw[3], i, j), vy = col_in(g.sw[4], i, j), vz = col_in(g.sw[5], i, j);
    const float idye = g.idye[min(j, nya - 1)], idxe = g.idxe[i];
    const long long pitch = g.pitch, plane = g.plane;
    float* const F3 = g.F[3];
    float* const F4 = g.F[4];
    float* const F5 = g.F[5];
    const int kx0 = g.sw[3][4], kx1 = g.sw[3][5], ky0 = g.sw[4][4], ky1 = g.sw[4][5], kz0 = g.sw[5][4], kz1 = g.sw[5][5];
    const unsigned tmask = CP ? cpml_tile_mask(cp, 3, t.ib, t.ib + kTX - 1, t.jb, t.jb + kTY - 1) : 0u;
    const CpmlCol cc = CP ? cpml_col(cp, 3, tmask, i, j, t.kb, t.ke) : CpmlCol{};
    if (CP == 2) psi_rows_fill(rows, cp, 3, tmask, kPsiSlotFloats, t.ib, j, l);
    float ex_kp, ey_kp;
    {
        const unsigned s0 = G0 % kStages;
        if (!warp_wait(t.full0 + 8 * s0, (G0 / kStages) & 1, err, 4, t.wait)) return false;
        const unsigned char* nx = t.ring + s0 * kStageBytes;
        ex_kp = ((const float*)(nx + kOffA))[w * kTX + l];
        ey_kp = ((const float*)(nx + kOffB))[w * kHaloW + l];
        warp_release(t, G0);
    }
    long long c = i + pitch * j + plane * t.ke;
    for (int k = t.ke; k >= t.kb; --k, c -= plane) {
        const unsigned Gk = G0 + 1 + (unsigned)(t.ke - k);
        const unsigned s = Gk % kStages;
        if (!warp_wait(t.full0 + 8 * s, (Gk / kStages) & 1, err, 3, t.wait)) return false;
        const unsigned char* st = t.ring + s * kStageBytes;
        // slabs holding cell (i, j, k), the plane's Idze and P_b / P_c pair
        const PlaneWords pw = *(const PlaneWords*)(st + kOffW);
        const unsigned pm = CP ? (cc.col & pw.live) : 0u;
        const float bz = pw.bz, cz = pw.cz;
        const float* EX = (const float*)(st + kOffA);
        const float* EY = (const float*)(st + kOffB);
        const float* EZ = (const float*)(st + kOffC);
        const float* HF = (const float*)(st + kOffF);
        const uint8_t* MF = (const uint8_t*)(st + kOffM);
        const float* PS = (const float*)(st + kOffP);
        constexpr int fs = align128(kBoxF) / 4, ms = align128(kBoxM);
        const float ex = EX[w * kTX + l], ex_jp = EX[(w + 1) * kTX + l];
        const float ey = EY[w * kHaloW + l], ey_ip = EY[w * kHaloW + l + 1];
        const float ez = EZ[w * kHaloW + l], ez_ip = EZ[w * kHaloW + l + 1], ez_jp = EZ[(w + 1) * kHaloW + l];
        const float idze = pw.idz;
        const int o = w * kTX + l;
        bool st_ = true;
        if (vx && k >= kx0 && k <= kx1) {
            float h = HF[o];
            const float2 tt = tab(MF[o]);
            const float dz = ey_kp - ey, dy = ez_jp - ez;
            h = tt.x * h + tt.y * (dz * idze - dy * idye);
            if (CP && pm) {
                h = cpml_corr<CP, false>(cp.s[3][0], pm & 3, 0, PS, o, rows, i, j, k, cc.by, cc.cy, dy, tt.y, h, st_);
                h = cpml_corr<CP, true>(cp.s[3][1], (pm >> 2) & 3, 2, PS, o, rows, i, j, k, bz, cz, dz, tt.y, h, st_);
            }
            F3[c] = h;
        }
        if (vy && k >= ky0 && k <= ky1) {
            float h = HF[fs + o];
            const float2 tt = tab(MF[ms + o]);
            const float dx = ez_ip - ez, dz = ex_kp - ex;
            h = tt.x * h + tt.y * (dx * idxe - dz * idze);
            if (CP && pm) {
                h = cpml_corr<CP, false>(cp.s[4][0], (pm >> 4) & 3, 4, PS, o, rows, i, j, k, bz, cz, dz, tt.y, h, st_);
                h = cpml_corr<CP, true>(cp.s[4][1], (pm >> 6) & 3, 6, PS, o, rows, i, j, k, cc.bx, cc.cx, dx, tt.y, h, st_);
            }
            F4[c] = h;
        }
        if (vz && k >= kz0 && k <= kz1) {
            float h = HF[2 * fs + o];
            const float2 tt = tab(MF[2 * ms + o]);
            const float dy = ex_jp - ex, dx = ey_ip - ey;
            h = tt.x * h + tt.y * (dy * idye - dx * idxe);
            if (CP && pm) {
                h = cpml_corr<CP, true>(cp.s[5][0], (pm >> 8) & 3, 8, PS, o, rows, i, j, k, cc.by, cc.cy, dy, tt.y, h, st_);
                h = cpml_corr<CP, false>(cp.s[5][1], (pm >> 10) & 3, 10, PS, o, rows, i, j, k, cc.bx, cc.cx, dx, tt.y, h, st_);
            }
            F5[c] = h;
        }
        ex_kp = ex;
        ey_kp = ey;
        if (k > t.kb || release_last) warp_release(t, Gk);  // plane k is no longer needed
    }
    return true;
}

}  // namespace sgpu
