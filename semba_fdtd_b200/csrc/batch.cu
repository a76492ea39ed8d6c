// Batched form: many independent FDTD problems of uneven sizes advanced
// together on one GPU.
//
// * Every instance is an ordinary context (the same device layout and
//   set-up as a single problem) whose buffers are carved out of one device
//   arena (first fit, 256-byte aligned, coalescing free list).
// * A descriptor table on the device holds each instance's grid, CPML, ADE,
//   source and probe views plus its step offset; flattened work lists hold
//   (instance, tile, z chunk) items for the field kernels and node / row /
//   probe ranges for the other phases.
// * One persistent kernel per phase walks its work list; an instance's step
//   index is the batch's device step counter plus the instance's offset, and
//   an instance outside 0..last step does nothing.  So instances can join at
//   any chunk boundary and finish at any step while the graph of 32 captured
//   steps stays valid: changing the batch only rewrites the tables.
// * The per-cell arithmetic is the single-problem code (stencil.cuh,
//   tma_fields.cuh), so an instance gives the same bits alone, in any mix
//   and on the plain path.
// * The z-chunk length of the field work items is chosen per size class and
//   the persistent grid size per batch by an online autotuner that times real
//   steps (results do not depend on either choice).
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "sgpu_internal.h"
#include "stencil.cuh"
// The persistent batched field kernels keep a 4-stage ring (3 CTAs an SM,
// bound by their registers); the plain ones run 3 stages at 4 CTAs an SM.
#define SGPU_TMA_STAGES 4
#include "tma_fields.cuh"

using namespace sgpu;
using namespace sgpu::dev;

// ---------------------------------------------------------------------------
// Arena

struct sgpu::Arena {
    char* base = nullptr;
    size_t cap = 0;
    size_t in_use = 0;
    std::map<size_t, size_t> free_;            // offset -> size, address ordered
    std::unordered_map<size_t, size_t> used_;  // offset -> size
    std::mutex mu;
};

namespace sgpu {
namespace {
constexpr size_t kArenaAlign = 256;
}
}  // namespace sgpu

void* sgpu::arena_alloc(Arena* a, size_t bytes) {
    if (!a || bytes == 0) return nullptr;
    const size_t need = (bytes + kArenaAlign - 1) / kArenaAlign * kArenaAlign;
    std::lock_guard<std::mutex> lock(a->mu);
    for (auto it = a->free_.begin(); it != a->free_.end(); ++it) {
        if (it->second < need) continue;
        const size_t off = it->first, rest = it->second - need;
        a->free_.erase(it);
        if (rest) a->free_[off + need] = rest;
        a->used_[off] = need;
        a->in_use += need;
        return a->base + off;
    }
    return nullptr;
}

void sgpu::arena_free(Arena* a, void* p) {
    if (!a || !p) return;
    std::lock_guard<std::mutex> lock(a->mu);
    const size_t off = (size_t)((char*)p - a->base);
    auto u = a->used_.find(off);
    if (u == a->used_.end()) return;
    size_t start = off, size = u->second;
    a->in_use -= size;
    a->used_.erase(u);
    auto next = a->free_.lower_bound(start);
    if (next != a->free_.end() && next->first == start + size) {
        size += next->second;
        next = a->free_.erase(next);
    }
    if (next != a->free_.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == start) {
            start = prev->first;
            size += prev->second;
            a->free_.erase(prev);
        }
    }
    a->free_[start] = size;
}

namespace sgpu {
namespace {

size_t arena_largest(Arena* a) {
    std::lock_guard<std::mutex> lock(a->mu);
    size_t m = 0;
    for (auto& f : a->free_) m = std::max(m, f.second);
    return m;
}

// ---------------------------------------------------------------------------
// Device tables

struct InstDesc {
    KGrid g;
    KCpml cp;
    KDisp d, md;  // electric and magnetic pole-residue media
    KSrc src[2];
    KProbes pr;
    KBorder bd;
    const double* tiempo;
    double dt;
    int step_off;  // instance step n = batch counter + step_off
    int last_n;    // steps 0..last_n are advanced; -1: inactive slot
};

struct FieldItem {
    int slot, ib, jb, kb, ke, cp;
};
struct RangeItem {
    int slot, sub;     // sub: E component (ADE) or side (sources)
    long long q0, q1;  // node / row / probe range
};

enum : int { kCntE = 0, kCntH, kCntNode, kCntSrcE, kCntSrcH, kCntProbe, kCntClone, kCntMur, kCntMNode, kNumCounts };

constexpr int kNodeChunk = 2048;  // ADE nodes per work item
constexpr int kPhaseThreads = 256;
constexpr int kRowChunk = kPhaseThreads;  // source rows / probes per work item (one per thread)
constexpr int kBorderChunk = 1024;  // clone / Mur cells per work item

__device__ __forceinline__ int inst_step(const InstDesc& D, const int* G, bool* on) {
    const int n = *G + D.step_off;
    *on = n >= 0 && n <= D.last_n;
    return n;
}

// Per-warp copy of an instance's grid (and CPML) view into shared memory:
// the field kernels then read slab bounds, pointers and sweep limits with
// shared loads instead of global ones, and no warp waits for another.
constexpr int kWarpTab = 32;  // media per coefficient table held in a warp's view
struct WarpView {
    KGrid g;
    KCpml cp;
    float2 tab[kWarpTab];  // the side's coefficient pairs, when nmed1 <= kWarpTab
};
template <class T> __device__ __forceinline__ void warp_copy(T* dst, const T* src, int lane) {
    static_assert(sizeof(T) % 4 == 0, "word copy");
    const int* s = (const int*)src;
    int* d = (int*)dst;
    for (int q = lane; q < (int)(sizeof(T) / 4); q += 32) d[q] = s[q];
}
// side < 0: no tables; 0: G1 / G2; 1: GM1 / GM2 (when the instance has at
// most kWarpTab media, else the consumers read the tables from global memory).
__device__ __forceinline__ const WarpView& stage_view(WarpView* slot, const InstDesc& D, bool cpml, int lane,
                                                      int side = -1) {
    __syncwarp();  // the warp is done with the previous item's view
    warp_copy(&slot->g, &D.g, lane);
    if (cpml) warp_copy(&slot->cp, &D.cp, lane);
    if (side >= 0 && lane < D.g.nmed1 && D.g.nmed1 <= kWarpTab)
        slot->tab[lane] = make_float2((side ? D.g.gm1 : D.g.g1)[lane], (side ? D.g.gm2 : D.g.g2)[lane]);
    __syncwarp();
    return *slot;
}

// Advance_Ex/Ey/Ez + AdvanceelectricCPML (SIDE 0) or Advance_Hx/Hy/Hz +
// AdvanceMagneticCPML (SIDE 1) over every active instance's tiles, with the
// register-marching columns.
template <int SIDE>
__global__ void __launch_bounds__(kBX * kBY, 4)
    k_batch_field(const InstDesc* __restrict__ descs, const FieldItem* __restrict__ items, const int* counts, const int* G) {
    __shared__ WarpView views[kBY];
    const int n_items = counts[SIDE == 0 ? kCntE : kCntH];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const FieldItem w = items[it];
        const InstDesc& D = descs[w.slot];
        bool on;
        inst_step(D, G, &on);
        if (!on) continue;
        const WarpView& V = stage_view(&views[threadIdx.y], D, w.cp != 0, threadIdx.x);
        const KGrid& g = V.g;
        const int i = w.ib + threadIdx.x, j = w.jb + threadIdx.y;
        const int jc = min(max(j, 1), (int)(g.plane / g.pitch) - 2);
        constexpr int MODE = kBulk | kCpml | kAll;
        if (SIDE == 0) {
            const bool vx = col_in(g.sw[0], i, j), vy = col_in(g.sw[1], i, j), vz = col_in(g.sw[2], i, j);
            if (w.cp) efield_column<MODE, true>(g, V.cp, g.g1, g.g2, i, jc, w.kb, w.ke, vx, vy, vz);
            else efield_column<MODE, false>(g, V.cp, g.g1, g.g2, i, jc, w.kb, w.ke, vx, vy, vz);
        } else {
            const bool vx = col_in(g.sw[3], i, j), vy = col_in(g.sw[4], i, j), vz = col_in(g.sw[5], i, j);
            if (w.cp) hfield_column<MODE, true>(g, V.cp, g.gm1, g.gm2, i, jc, w.kb, w.ke, vx, vy, vz);
            else hfield_column<MODE, false>(g, V.cp, g.gm1, g.gm2, i, jc, w.kb, w.ke, vx, vy, vz);
        }
    }
}

// The same half steps through the TMA ring (tma_fields.cuh) as one
// persistent kernel: each CTA's producer warp takes the next work item from a
// counter shared by the launch (so CTAs that draw cheap items take more of
// them and all finish together) and the ring's running plane number carries
// on from item to item, so the producer fetches the next item's planes while
// the consumers finish the current one; each plane names its item, which is
// how the consumer warps follow.
// Each instance's tensor maps live in global memory (written by the host
// before the launch) and are acquired through the tensormap proxy before
// their first use in the CTA.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* m) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((unsigned long long)m) : "memory");
}

// One work item of a consumer warp: the staged-psi, global-psi or bulk form.
template <int SIDE, class TAB>
__device__ __forceinline__ bool consume(const TmaCta& t, unsigned gp, const KGrid& g, const KCpml& cp, const TAB tab, int* err,
                                        PsiRow* rows, unsigned smask, bool cpml) {
    if (SIDE == 0)
        return smask ? e_consume<2>(t, gp, g, cp, tab, err, true, rows)
               : cpml ? e_consume<1>(t, gp, g, cp, tab, err, true, rows)
                      : e_consume<0>(t, gp, g, cp, tab, err, true, rows);
    return smask ? h_consume<2>(t, gp, g, cp, tab, err, true, rows)
           : cpml ? h_consume<1>(t, gp, g, cp, tab, err, true, rows)
                  : h_consume<0>(t, gp, g, cp, tab, err, true, rows);
}

template <int SIDE>
__global__ void __launch_bounds__(kTmaThreads, 3)
    k_batch_tma_field(const InstDesc* __restrict__ descs, const TMaps* __restrict__ maps, const FieldItem* __restrict__ items,
                      const int* counts, const int* G, int* err, long long wait, int drill, int* next) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ WarpView views[kConsumerWarps];
    __shared__ ProdWindow tb;
    __shared__ PsiRow rows[kConsumerWarps][12];
    TmaCta t = tma_cta_setup(smem, 0, 0, 0, 1, wait);
    const int n_items = counts[SIDE == 0 ? kCntE : kCntH];
    const bool producer = t.warp == kConsumerWarps;
    unsigned gp = 0;  // running plane number of the ring
    int fenced = -1;     // the instance whose tensor maps the producer has acquired
    bool facq = false;   // ... and whether this lane has acquired its own map
    int viewed = -1;  // ... whose view the consumer warp holds
    const int c0 = SIDE == 0 ? 0 : 3;
    if (producer) {
        if (drill) return;  // a failure drill: no plane arrives, every consumer wait runs out
        for (;;) {
            int it = 0;
            if (t.lane == 0) it = atomicAdd(next, 1);
            it = __shfl_sync(0xffffffffu, it, 0);
            if (it >= n_items) break;
            const FieldItem w = items[it];
            const InstDesc& D = descs[w.slot];
            bool on;
            inst_step(D, G, &on);
            if (!on) continue;
            t.ib = w.ib;
            t.jb = w.jb;
            t.kb = w.kb;
            t.ke = w.ke;
            const int np = w.ke - w.kb + 2;  // the item's planes, edge plane included
            // CPML items stage their psi tiles through the ring when the tile's
            // slabs fit the kPsiSlots slots (the consumers derive the same mask)
            const int p0 = SIDE == 0 ? w.kb - 1 : w.kb, p1 = SIDE == 0 ? w.ke : w.ke + 1;
            const int edge = SIDE == 0 ? w.kb - 1 : w.ke + 1;
            const unsigned tmask = w.cp ? cpml_tile_mask(D.cp, c0, w.ib, w.ib + kTX - 1, w.jb, w.jb + kTY - 1) : 0u;
            const unsigned smask = w.cp ? staged_mask(D.cp, c0, w.ib, w.jb) : 0u;
            prod_psi(&tb, t, SIDE != 0, D.cp, tmask);
            const PlaneSource src{&D.g, &D.cp, tmask};
            const CUtensorMap* m = maps[2 * w.slot + SIDE].m;
            // each lane acquires the one map it issues through (lane q: map q),
            // once per instance, when this item loads through it
            if (fenced != w.slot) {
                fenced = w.slot;
                facq = false;
            }
            const bool need = t.lane < kPsiMap0 || (t.lane < kPsiMap0 + 12 && ((smask >> (t.lane - kPsiMap0)) & 1u));
            if (need && !facq) {
                tensormap_acquire(&m[t.lane]);
                facq = true;
            }
            const ItemWords iw{{it, w.slot, w.ib, w.jb, w.kb, w.ke, w.cp}};
            const int got = tma_issue_warp(t, m, gp, p0, p1, edge, SIDE != 0, err, &tb, src, smask, iw);
            if (got < np) {
                if (t.lane == 0) tma_drain(t, gp + (unsigned)got, err, 15);
                return;
            }
            gp += (unsigned)np;
        }
        if (t.lane == 0) {
            const bool ended = tma_publish_end(t, gp, err);
            tma_drain(t, gp + (ended ? 1u : 0u), err, 15);
        }
        return;
    }
    for (;;) {
        // the item of the next plane (item -1: no more)
        const unsigned s = gp % kStages;
        if (!warp_wait(t.full0 + 8 * s, (gp / kStages) & 1, err, 5, t.wait)) return;
        const volatile int* iv = (const volatile int*)(t.ring + s * kStageBytes + kOffItem);
        if (iv[0] < 0) return;
        const FieldItem w{iv[1], iv[2], iv[3], iv[4], iv[5], iv[6]};
        const InstDesc& D = descs[w.slot];
        t.ib = w.ib;
        t.jb = w.jb;
        t.kb = w.kb;
        t.ke = w.ke;
        const int np = w.ke - w.kb + 2;
        if (w.slot != viewed) {
            stage_view(&views[t.warp], D, true, t.lane, SIDE);
            viewed = w.slot;
        }
        const WarpView& V = views[t.warp];
        const KGrid& g = V.g;
        const unsigned smask = w.cp ? staged_mask(V.cp, c0, w.ib, w.jb) : 0u;
        bool ok;
        if (g.nmed1 <= kWarpTab)
            ok = consume<SIDE>(t, gp, g, V.cp, TabPairs{V.tab}, err, rows[t.warp], smask, w.cp != 0);
        else
            ok = consume<SIDE>(t, gp, g, V.cp, TabSplit{SIDE == 0 ? g.g1 : g.gm1, SIDE == 0 ? g.g2 : g.gm2}, err,
                               rows[t.warp], smask, w.cp != 0);
        if (!ok) return;
        gp += (unsigned)np;
    }
}

// AdvanceEDispersiveE (MAG false) or AdvanceMdispersiveH (MAG true) over
// node ranges of every active instance.
template <int NU, bool MAG>
__global__ void __launch_bounds__(kPhaseThreads)
    k_batch_ade(const InstDesc* __restrict__ descs, const RangeItem* __restrict__ items, const int* counts, const int* G) {
    const int n_items = counts[MAG ? kCntMNode : kCntNode];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const RangeItem w = items[it];
        const InstDesc& D = descs[w.slot];
        bool on;
        inst_step(D, G, &on);
        if (!on) continue;
        const AdeRefs r = ade_refs<MAG>(D.g, MAG ? D.md : D.d, w.sub);
        // two nodes a thread at a time: both nodes' loads go out before
        // either node's stores
        for (long long q = w.q0 + threadIdx.x; q < w.q1; q += 2 * (long long)blockDim.x) {
            const long long q2 = q + blockDim.x;
            const bool two = q2 < w.q1;
            AdeNode<NU> a, b;
            ade_load<NU, false>(r, q, a);
            if (two) ade_load<NU, false>(r, q2, b);
            ade_update<NU, MAG, false>(r, a);
            if (two) ade_update<NU, MAG, false>(r, b);
            ade_store<NU, false>(r, q, a);
            if (two) ade_store<NU, false>(r, q2, b);
        }
    }
}

// Plane-wave and nodal sources of one half step.
__global__ void __launch_bounds__(kPhaseThreads)
    k_batch_sources(const InstDesc* __restrict__ descs, const RangeItem* __restrict__ items, const int* counts, const int* G,
                    int side) {
    const int n_items = counts[side == 0 ? kCntSrcE : kCntSrcH];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const RangeItem w = items[it];
        const InstDesc& D = descs[w.slot];
        bool on;
        const int n = inst_step(D, G, &on);
        if (!on) continue;  // the same for the whole block: the item is one instance's
        const bool pw_on = pw_switch_block(D.src[side], n, D.tiempo, 0, D.dt, side);
        if (D.src[side].pw_only && !pw_on) continue;  // nothing applies once the switch is down
        const long long r = w.q0 + threadIdx.x;
        if (r < w.q1)
            source_row(D.g, D.src[side], n, D.tiempo, 0, D.dt, side,
                       (1 << kSrcPlaneWave) | (1 << kSrcNodalSoft) | (1 << kSrcNodalHard), (int)r, pw_on);
    }
}

// Point probes, one row per step of each instance (the whole trace stays on
// the device).
__global__ void __launch_bounds__(kPhaseThreads)
    k_batch_probes(const InstDesc* __restrict__ descs, const RangeItem* __restrict__ items, const int* counts, const int* G) {
    const int n_items = counts[kCntProbe];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const RangeItem w = items[it];
        const InstDesc& D = descs[w.slot];
        bool on;
        const int n = inst_step(D, G, &on);
        if (!on) continue;
        const long long q = w.q0 + threadIdx.x;
        if (q < w.q1) probe_one(D.g, D.pr, n, 0, (int)q);
    }
}

// The H-side borders after the H sources: PMC / periodic clones (which 0),
// then Mur (which 1), each over cell ranges of every active instance.
__global__ void __launch_bounds__(kPhaseThreads)
    k_batch_borders(const InstDesc* __restrict__ descs, const RangeItem* __restrict__ items, const int* counts, const int* G,
                    int which) {
    const int n_items = counts[which == 0 ? kCntClone : kCntMur];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const RangeItem w = items[it];
        const InstDesc& D = descs[w.slot];
        bool on;
        inst_step(D, G, &on);
        if (!on) continue;
        for (long long q = w.q0 + threadIdx.x; q < w.q1; q += blockDim.x) {
            if (which == 0) clone_cell(D.g, D.bd, 6, q);
            else mur_cell(D.g, D.bd, q);
        }
    }
}

// The batch counter moves on by one step.
__global__ void k_batch_tick(int* G) { *G += 1; }

struct Slot {
    sgpu_ctx* ctx = nullptr;
    int start = 0;   // batch counter value at the instance's step 0
    int nsteps = 0;  // last step index advanced (steps 0..nsteps)
    int size_class = 0;
    bool reserved = false;  // an instance is being set up for this slot
};

bool touches_any(const KCpml& cp, int c0, int x0, int x1, int y0, int y1, int z0, int z1) {
    if (!cp.on) return false;
    for (int f = c0; f < c0 + 3; ++f)
        for (int w = 0; w < 2; ++w)
            for (int sd = 0; sd < 2; ++sd) {
                const Slab& s = cp.s[f][w][sd];
                if (s.psi && x1 >= s.xlo && x0 <= s.xhi && y1 >= s.ylo && y0 <= s.yhi && z1 >= s.zlo && z0 <= s.zhi)
                    return true;
            }
    return false;
}

}  // namespace
}  // namespace sgpu

constexpr int kNumClasses = 3;

struct sgpu_batch {
    std::string err;
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    sgpu::Arena arena;
    int max_slots = 0;
    std::vector<Slot> slots;
    // device tables (plain cudaMalloc: they outlive every instance)
    InstDesc* d_desc = nullptr;
    TMaps* d_maps = nullptr;  // [slot][E side, H side]
    int* d_err = nullptr;     // bounded-wait error word of the TMA kernels
    int* d_next = nullptr;    // next work item of the E and H field launches
    long long wait_cycles = 4000000000LL;  // bound of a pipeline wait (clock cycles, ~2 s)
    int wait_drill = 0;                    // failure drill: producers issue no loads
    int* d_counts = nullptr;
    int* d_G = nullptr;
    FieldItem* d_field[2] = {};
    RangeItem* d_node = nullptr;
    RangeItem* d_mnode = nullptr;  // magnetic ADE node ranges
    size_t cap_mnode = 0;
    bool any_mnode = false;
    RangeItem* d_src[2] = {};
    RangeItem* d_probe = nullptr;
    RangeItem* d_border[2] = {};  // clone cells, Mur cells
    size_t cap_field[2] = {}, cap_node = 0, cap_src[2] = {}, cap_probe = 0, cap_border[2] = {};
    bool any_border[2] = {};      // some listed instance has clone / Mur cells
    int family = 1;  // 1: TMA-pipelined field kernels, 0: register-marching
    std::vector<char> has_maps;
    bool dirty = true;         // work lists must be rebuilt before the next step
    std::vector<char> listed;  // slots whose work is in the current lists
    int G = 0;                 // host mirror of the device step counter
    int nu_max = 1;
    // launch shape
    int chunk[kNumClasses] = {32, 64, 64};
    int ctas_per_sm = 4;
    // graph of kGraphSteps steps
    cudaGraphExec_t graph = nullptr;
    int graph_nu = 0, graph_ctas = 0;
    bool graph_tma = false, graph_border[2] = {}, graph_mnode = false;
    long long graph_wait = -1;
    int graph_drill = -1;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Every entry point holds this lock while it reads or changes the slots,
    // the step counter, the work lists or the graph.  An instance's set-up
    // runs outside it, on a stream of its own, so several host threads can
    // set up instances at once while the queued steps of the others run.
    mutable std::mutex mu;
};

namespace sgpu {
namespace {

constexpr int kGraphSteps = 32;

sgpu_status berr(sgpu_batch* b, sgpu_status code, const std::string& msg) {
    if (b) b->err = msg;
    return code;
}

#define BTRY(b, call)                                                                                           \
    do {                                                                                                        \
        cudaError_t e_ = (call);                                                                                \
        if (e_ != cudaSuccess) return berr((b), SGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int size_class_of(const sgpu_ctx* c) { return c->nza <= 80 ? 0 : c->nza <= 160 ? 1 : 2; }

InstDesc make_desc(const Slot& s, bool active) {
    InstDesc D{};
    sgpu_ctx* c = s.ctx;
    D.g = kgrid(c);
    D.cp = c->cpml;
    D.d = c->disp;
    if (!c->disp_on) D.d.n[0] = D.d.n[1] = D.d.n[2] = 0;
    D.md = c->mdisp;
    if (!c->mdisp_on) D.md.n[0] = D.md.n[1] = D.md.n[2] = 0;
    D.src[0] = c->src[0];
    D.src[1] = c->src[1];
    D.src[0].h_first = D.src[1].h_first = 0;  // an instance runs from step 0
    D.pr = c->probes;
    D.bd = c->border;
    D.tiempo = c->d_tiempo;
    D.dt = c->dt;
    D.step_off = -s.start;
    D.last_n = active ? s.nsteps : -1;
    return D;
}

template <class T> sgpu_status ensure(sgpu_batch* b, T** p, size_t* cap, size_t n) {
    if (n <= *cap && *p) return SGPU_OK;
    size_t want = std::max<size_t>(std::max<size_t>(n, 2 * *cap), 256);
    T* q = nullptr;
    BTRY(b, cudaStreamSynchronize(b->stream));
    BTRY(b, cudaMalloc((void**)&q, want * sizeof(T)));
    if (*p) cudaFree(*p);
    *p = q;
    *cap = want;
    if (b->graph) {  // a captured graph holds the old pointer
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return SGPU_OK;
}

template <class T> sgpu_status upload(sgpu_batch* b, T* d, const std::vector<T>& h) {
    if (h.empty()) return SGPU_OK;
    BTRY(b, cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, b->stream));
    return SGPU_OK;
}

// An instance still has steps to run at the batch counter value G.
bool running(const Slot& s, int G) { return s.ctx && G - s.start <= s.nsteps; }

// Rebuild the flattened work lists from the instances that still run.
sgpu_status rebuild(sgpu_batch* b) {
    std::vector<FieldItem> fi[2];
    std::vector<RangeItem> node, mnode, src[2], probe, border[2];
    int nu = 1;
    b->listed.assign(b->slots.size(), 0);
    for (int sl = 0; sl < (int)b->slots.size(); ++sl) {
        const Slot& s = b->slots[sl];
        if (!running(s, b->G)) continue;
        b->listed[sl] = 1;
        sgpu_ctx* c = s.ctx;
        const int chunk = b->chunk[s.size_class];
        for (int side = 0; side < 2; ++side) {
            const int c0 = side ? 3 : 0;
            int x1 = -1, y0 = 1 << 30, y1 = -1, z0 = 1 << 30, z1 = -1;
            for (int f = c0; f < c0 + 3; ++f) {
                x1 = std::max(x1, c->sweep[f].xe - c->ox);
                y0 = std::min(y0, c->sweep[f].yi - c->oy);
                y1 = std::max(y1, c->sweep[f].ye - c->oy);
                z0 = std::min(z0, c->sweep[f].zi - c->oz);
                z1 = std::max(z1, c->sweep[f].ze - c->oz);
            }
            for (int kb = z0; kb <= z1; kb += chunk) {
                const int ke = std::min(kb + chunk - 1, z1);
                for (int jb = y0; jb <= y1; jb += kBY)
                    for (int ib = 0; ib <= x1; ib += kBX)
                        fi[side].push_back(FieldItem{sl, ib, jb, kb, ke,
                                                     touches_any(c->cpml, c0, ib, ib + kBX - 1, jb, jb + kBY - 1, kb, ke) ? 1 : 0});
            }
        }
        if (c->disp_on) {
            nu = std::max(nu, c->disp.nu_max);
            for (int comp = 0; comp < 3; ++comp)
                for (long long q = 0; q < c->disp.n[comp]; q += kNodeChunk)
                    node.push_back(RangeItem{sl, comp, q, std::min<long long>(q + kNodeChunk, c->disp.n[comp])});
        }
        if (c->mdisp_on) {
            nu = std::max(nu, c->mdisp.nu_max);
            for (int comp = 0; comp < 3; ++comp)
                for (long long q = 0; q < c->mdisp.n[comp]; q += kNodeChunk)
                    mnode.push_back(RangeItem{sl, comp, q, std::min<long long>(q + kNodeChunk, c->mdisp.n[comp])});
        }
        for (int side = 0; side < 2; ++side)
            for (long long r = 0; r < c->src[side].nrows; r += kRowChunk)
                src[side].push_back(RangeItem{sl, side, r, std::min<long long>(r + kRowChunk, c->src[side].nrows)});
        for (long long q = 0; q < c->probes.n; q += kRowChunk)
            probe.push_back(RangeItem{sl, 0, q, std::min<long long>(q + kRowChunk, c->probes.n)});
        const long long bcells[2] = {c->border.cl_cells, c->border.mur_cells};
        for (int w = 0; w < 2; ++w)
            for (long long q = 0; q < bcells[w]; q += kBorderChunk)
                border[w].push_back(RangeItem{sl, w, q, std::min<long long>(q + kBorderChunk, bcells[w])});
    }
    sgpu_status s;
    for (int side = 0; side < 2; ++side) {
        if ((s = ensure(b, &b->d_field[side], &b->cap_field[side], fi[side].size()))) return s;
        if ((s = ensure(b, &b->d_src[side], &b->cap_src[side], src[side].size()))) return s;
    }
    if ((s = ensure(b, &b->d_node, &b->cap_node, node.size())) || (s = ensure(b, &b->d_probe, &b->cap_probe, probe.size())))
        return s;
    if ((s = ensure(b, &b->d_mnode, &b->cap_mnode, mnode.size())) || (s = upload(b, b->d_mnode, mnode))) return s;
    b->any_mnode = !mnode.empty();
    for (int w = 0; w < 2; ++w) {
        if ((s = ensure(b, &b->d_border[w], &b->cap_border[w], border[w].size()))) return s;
        if ((s = upload(b, b->d_border[w], border[w]))) return s;
        b->any_border[w] = !border[w].empty();
    }
    if ((s = upload(b, b->d_field[0], fi[0])) || (s = upload(b, b->d_field[1], fi[1])) || (s = upload(b, b->d_node, node)) ||
        (s = upload(b, b->d_src[0], src[0])) || (s = upload(b, b->d_src[1], src[1])) || (s = upload(b, b->d_probe, probe)))
        return s;
    std::vector<int> counts(kNumCounts);
    counts[kCntE] = (int)fi[0].size();
    counts[kCntH] = (int)fi[1].size();
    counts[kCntNode] = (int)node.size();
    counts[kCntSrcE] = (int)src[0].size();
    counts[kCntSrcH] = (int)src[1].size();
    counts[kCntProbe] = (int)probe.size();
    counts[kCntClone] = (int)border[0].size();
    counts[kCntMur] = (int)border[1].size();
    counts[kCntMNode] = (int)mnode.size();
    if ((s = upload(b, b->d_counts, counts))) return s;
    if (nu > b->nu_max) b->nu_max = nu;
    // no wait: an asynchronous copy from pageable host memory has staged the
    // data by the time it returns, so the vectors may go out of scope, and
    // the steps already queued keep running meanwhile
    b->dirty = false;
    return SGPU_OK;
}

// Finished instances leave the work lists at the next chunk boundary (their
// memory and results stay until sgpu_batch_remove).
void drop_finished(sgpu_batch* b) {
    if (b->listed.size() != b->slots.size()) {
        b->dirty = true;
        return;
    }
    for (size_t sl = 0; sl < b->slots.size(); ++sl)
        if (b->listed[sl] && !running(b->slots[sl], b->G)) {
            b->dirty = true;
            return;
        }
}

// The TMA kernels serve the batch when every listed instance has tensor maps.
bool use_tma(const sgpu_batch* b) {
    if (b->family != 1) return false;
    for (size_t sl = 0; sl < b->listed.size(); ++sl)
        if (b->listed[sl] && !b->has_maps[sl]) return false;
    return true;
}

template <int NU, bool MAG> void ade_batch(sgpu_batch* b, int grid) {
    k_batch_ade<NU, MAG><<<grid, kPhaseThreads, 0, b->stream>>>(b->d_desc, MAG ? b->d_mnode : b->d_node, b->d_counts, b->d_G);
}

template <bool MAG> void ade_phase(sgpu_batch* b, int grid) {
    switch (b->nu_max) {
        case 1: ade_batch<1, MAG>(b, grid); break;
        case 2: ade_batch<2, MAG>(b, grid); break;
        case 3: ade_batch<3, MAG>(b, grid); break;
        case 4: ade_batch<4, MAG>(b, grid); break;
        default: ade_batch<kMaxPolesPerMedium, MAG>(b, grid); break;
    }
}

// One whole step of every instance in the order of timestepping.F90 (E curl +
// CPML, ADE, E sources, H curl + CPML, magnetic ADE + H sources + borders, probes).  With `marks`, an
// event is recorded after each of the six phases.
sgpu_status enqueue_step(sgpu_batch* b, cudaEvent_t* marks = nullptr) {
    const int grid = b->num_sms * b->ctas_per_sm;
    const int tgrid = b->num_sms * std::min(b->ctas_per_sm, 3);
    const dim3 blk(kBX, kBY);
    const bool tma = use_tma(b);
    auto mark = [&](int q) {
        if (marks) cudaEventRecord(marks[q], b->stream);
    };
    if (tma) {
        cudaMemsetAsync(b->d_next, 0, 2 * sizeof(int), b->stream);  // the launches' item counters
        k_batch_tma_field<0><<<tgrid, kTmaThreads, kTmaSmem, b->stream>>>(b->d_desc, b->d_maps, b->d_field[0], b->d_counts,
                                                                          b->d_G, b->d_err, b->wait_cycles, b->wait_drill,
                                                                          b->d_next);
    }
    else
        k_batch_field<0><<<grid, blk, 0, b->stream>>>(b->d_desc, b->d_field[0], b->d_counts, b->d_G);
    mark(0);
    ade_phase<false>(b, grid);
    mark(1);
    k_batch_sources<<<grid, kPhaseThreads, 0, b->stream>>>(b->d_desc, b->d_src[0], b->d_counts, b->d_G, 0);
    mark(2);
    if (tma)
        k_batch_tma_field<1><<<tgrid, kTmaThreads, kTmaSmem, b->stream>>>(b->d_desc, b->d_maps, b->d_field[1], b->d_counts,
                                                                          b->d_G, b->d_err, b->wait_cycles, b->wait_drill,
                                                                          b->d_next + 1);
    else
        k_batch_field<1><<<grid, blk, 0, b->stream>>>(b->d_desc, b->d_field[1], b->d_counts, b->d_G);
    mark(3);
    if (b->any_mnode) ade_phase<true>(b, grid);
    k_batch_sources<<<grid, kPhaseThreads, 0, b->stream>>>(b->d_desc, b->d_src[1], b->d_counts, b->d_G, 1);
    for (int w = 0; w < 2; ++w)
        if (b->any_border[w])
            k_batch_borders<<<grid, kPhaseThreads, 0, b->stream>>>(b->d_desc, b->d_border[w], b->d_counts, b->d_G, w);
    mark(4);
    k_batch_probes<<<grid, kPhaseThreads, 0, b->stream>>>(b->d_desc, b->d_probe, b->d_counts, b->d_G);
    k_batch_tick<<<1, 1, 0, b->stream>>>(b->d_G);
    mark(5);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return berr(b, SGPU_ERR_CUDA, std::string("batched step launch: ") + cudaGetErrorString(e));
    return SGPU_OK;
}

sgpu_status ensure_graph(sgpu_batch* b) {
    if (b->graph && b->graph_nu == b->nu_max && b->graph_ctas == b->ctas_per_sm && b->graph_tma == use_tma(b) &&
        b->graph_border[0] == b->any_border[0] && b->graph_border[1] == b->any_border[1] &&
        b->graph_mnode == b->any_mnode && b->graph_wait == b->wait_cycles && b->graph_drill == b->wait_drill)
        return SGPU_OK;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    BTRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    sgpu_status s = SGPU_OK;
    for (int q = 0; q < kGraphSteps && !s; ++q) s = enqueue_step(b);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (s) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) return berr(b, SGPU_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->graph = nullptr;
        return berr(b, SGPU_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    b->graph_nu = b->nu_max;
    b->graph_ctas = b->ctas_per_sm;
    b->graph_tma = use_tma(b);
    b->graph_border[0] = b->any_border[0];
    b->graph_border[1] = b->any_border[1];
    b->graph_mnode = b->any_mnode;
    b->graph_wait = b->wait_cycles;
    b->graph_drill = b->wait_drill;
    return SGPU_OK;
}

sgpu_status advance(sgpu_batch* b, int nsteps, bool use_graph) {
    sgpu_status s;
    drop_finished(b);
    if (b->dirty && (s = rebuild(b))) return s;
    int done = 0;
    if (use_graph && nsteps >= kGraphSteps) {
        if ((s = ensure_graph(b))) return s;
        for (; done + kGraphSteps <= nsteps; done += kGraphSteps) BTRY(b, cudaGraphLaunch(b->graph, b->stream));
    }
    for (; done < nsteps; ++done)
        if ((s = enqueue_step(b))) return s;
    b->G += nsteps;
    return SGPU_OK;
}

// The TMA kernels record an expired bounded wait in d_err.
sgpu_status check_err(sgpu_batch* b) {
    int e = 0;
    BTRY(b, cudaMemcpy(&e, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        BTRY(b, cudaMemset(b->d_err, 0, sizeof(int)));
        return berr(b, SGPU_ERR_TIMEOUT, "a bounded wait in a pipelined batch kernel expired (code " + std::to_string(e) + ")");
    }
    return SGPU_OK;
}

bool valid_slot(const sgpu_batch* b, int slot) {
    return b && slot >= 0 && slot < (int)b->slots.size() && b->slots[slot].ctx;
}

}  // namespace
}  // namespace sgpu

extern "C" {

sgpu_status sgpu_batch_create(uint64_t arena_bytes, int max_instances, sgpu_batch** out) {
    if (!out || arena_bytes == 0 || max_instances < 1) return SGPU_ERR_ARG;
    *out = nullptr;
    sgpu_batch* b = new (std::nothrow) sgpu_batch();
    if (!b) return SGPU_ERR_OOM;
    *out = b;
    BTRY(b, cudaGetDevice(&b->device));
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device);
    BTRY(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    void* base = nullptr;
    keep_device_pool(b->device);
    // the arena comes from the device's default memory pool, which keeps the
    // memory solo contexts (or an earlier batch) freed; only when the pool
    // cannot serve it is its unused memory handed back and the request
    // retried.  The pool gets the arena back when the batch is destroyed.
    if (cudaMallocAsync(&base, arena_bytes, b->stream) != cudaSuccess) {
        cudaGetLastError();
        base = nullptr;
        sgpu_trim_device_memory();
        if (cudaMallocAsync(&base, arena_bytes, b->stream) != cudaSuccess) {
            cudaGetLastError();
            return berr(b, SGPU_ERR_OOM, "arena of " + std::to_string(arena_bytes) + " bytes could not be allocated");
        }
    }
    b->arena.base = (char*)base;
    b->arena.cap = arena_bytes / kArenaAlign * kArenaAlign;
    b->arena.free_[0] = b->arena.cap;
    b->max_slots = max_instances;
    b->slots.resize(max_instances);
    b->has_maps.assign(max_instances, 0);
    BTRY(b, cudaMalloc((void**)&b->d_desc, sizeof(InstDesc) * max_instances));
    BTRY(b, cudaMalloc((void**)&b->d_maps, sizeof(TMaps) * 2 * max_instances));
    BTRY(b, cudaMalloc((void**)&b->d_err, sizeof(int)));
    BTRY(b, cudaMalloc((void**)&b->d_next, 2 * sizeof(int)));
    BTRY(b, cudaMalloc((void**)&b->d_counts, sizeof(int) * kNumCounts));
    BTRY(b, cudaMalloc((void**)&b->d_G, sizeof(int)));
    BTRY(b, cudaMemsetAsync(b->d_err, 0, sizeof(int), b->stream));
    BTRY(b, cudaMemsetAsync(b->d_counts, 0, sizeof(int) * kNumCounts, b->stream));
    BTRY(b, cudaMemsetAsync(b->d_G, 0, sizeof(int), b->stream));
    std::vector<InstDesc> off(max_instances);
    for (auto& d : off) d.last_n = -1;
    BTRY(b, cudaMemcpyAsync(b->d_desc, off.data(), sizeof(InstDesc) * max_instances, cudaMemcpyHostToDevice, b->stream));
    BTRY(b, cudaEventCreate(&b->ev0));
    BTRY(b, cudaEventCreate(&b->ev1));
    // the TMA ring (with its psi slots) is above the default dynamic limit
    BTRY(b, cudaFuncSetAttribute(k_batch_tma_field<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmaSmem));
    BTRY(b, cudaFuncSetAttribute(k_batch_tma_field<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmaSmem));
    BTRY(b, cudaStreamSynchronize(b->stream));
    return SGPU_OK;
}

void sgpu_batch_destroy(sgpu_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (Slot& s : b->slots)
        if (s.ctx) sgpu_destroy(s.ctx);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    cudaFree(b->d_desc);
    cudaFree(b->d_maps);
    cudaFree(b->d_err);
    cudaFree(b->d_next);
    cudaFree(b->d_counts);
    cudaFree(b->d_G);
    for (int s = 0; s < 2; ++s) {
        cudaFree(b->d_field[s]);
        cudaFree(b->d_src[s]);
    }
    cudaFree(b->d_node);
    cudaFree(b->d_mnode);
    cudaFree(b->d_probe);
    cudaFree(b->d_border[0]);
    cudaFree(b->d_border[1]);
    if (b->arena.base) {
        cudaFreeAsync(b->arena.base, b->stream);
        cudaStreamSynchronize(b->stream);
    }
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char* sgpu_batch_last_error(const sgpu_batch* b) { return b ? b->err.c_str() : "null batch"; }

sgpu_status sgpu_batch_add(sgpu_batch* b, const sgpu_problem* p, sgpu_ctx* plan, int nsteps, int* slot) {
    if (!b) return SGPU_ERR_ARG;
    if (!slot || (!p && !plan) || nsteps < 0) {
        std::lock_guard<std::mutex> lock(b->mu);
        return berr(b, SGPU_ERR_ARG, "bad sgpu_batch_add arguments");
    }
    *slot = -1;
    int sl = -1;
    {
        std::lock_guard<std::mutex> lock(b->mu);
        for (int q = 0; q < b->max_slots; ++q)
            if (!b->slots[q].ctx && !b->slots[q].reserved) {
                sl = q;
                break;
            }
        if (sl < 0) return berr(b, SGPU_ERR_OOM, "no free instance slot");
        b->slots[sl].reserved = true;
    }
    // Set-up outside the lock, on a stream of its own of the highest
    // priority: it touches only the new instance's arena memory (the arena
    // has its own lock), so the steps queued on the batch stream keep
    // running and other threads may set up other instances meanwhile; the
    // batch stream then waits for it before anything reads the instance.
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    sgpu_ctx* c = nullptr;
    sgpu_status s = SGPU_OK;
    std::string msg;
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, hi) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        s = SGPU_ERR_CUDA;
        msg = "the set-up stream could not be created";
    }
    if (!s) s = host_create_in(p, plan, nsteps, &b->arena, st, &c);
    if (!s) s = rebuild_sources(c);
    if (!s && cudaEventRecord(ev, st) != cudaSuccess) {
        cudaGetLastError();
        s = SGPU_ERR_CUDA;
        msg = "the set-up could not be recorded";
    }
    if (s && msg.empty()) msg = c ? c->err : "instance set-up failed";
    auto release = [&]() {
        if (ev) cudaEventDestroy(ev);
        if (st) cudaStreamDestroy(st);  // released once its work is done
    };
    std::lock_guard<std::mutex> lock(b->mu);
    b->slots[sl].reserved = false;
    if (!s && cudaStreamWaitEvent(b->stream, ev, 0) != cudaSuccess) {
        cudaGetLastError();
        s = SGPU_ERR_CUDA;
        msg = "the batch stream could not wait for the set-up";
    }
    if (s) {
        b->err = msg;
        if (c) sgpu_destroy(c);
        release();
        return s;
    }
    release();
    c->stream = b->stream;
    Slot& S = b->slots[sl];
    S.ctx = c;
    S.start = b->G;
    S.nsteps = nsteps;
    S.size_class = size_class_of(c);
    InstDesc D = make_desc(S, true);
    BTRY(b, cudaMemcpyAsync(b->d_desc + sl, &D, sizeof(InstDesc), cudaMemcpyHostToDevice, b->stream));
    b->has_maps[sl] = tma_usable(c) ? 1 : 0;
    TMaps m2[2] = {c->tme, c->tmh};
    if (c->tma_ready) BTRY(b, cudaMemcpyAsync(b->d_maps + 2 * sl, m2, sizeof(m2), cudaMemcpyHostToDevice, b->stream));
    b->dirty = true;
    *slot = sl;
    return SGPU_OK;
}

sgpu_status sgpu_batch_remove(sgpu_batch* b, int slot) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!valid_slot(b, slot)) return berr(b, SGPU_ERR_ARG, "no instance in that slot");
    BTRY(b, cudaStreamSynchronize(b->stream));
    InstDesc off{};
    off.last_n = -1;
    BTRY(b, cudaMemcpyAsync(b->d_desc + slot, &off, sizeof(InstDesc), cudaMemcpyHostToDevice, b->stream));
    BTRY(b, cudaStreamSynchronize(b->stream));
    sgpu_destroy(b->slots[slot].ctx);
    b->slots[slot] = Slot{};
    b->has_maps[slot] = 0;
    b->dirty = true;
    return SGPU_OK;
}

sgpu_status sgpu_batch_advance(sgpu_batch* b, int nsteps) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b || nsteps < 0) return SGPU_ERR_ARG;
    return advance(b, nsteps, true);
}

sgpu_status sgpu_batch_synchronize(sgpu_batch* b) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b) return SGPU_ERR_ARG;
    BTRY(b, cudaStreamSynchronize(b->stream));
    return check_err(b);
}

sgpu_status sgpu_batch_set_wait_cycles(sgpu_batch* b, int64_t cycles) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b || cycles < 0) return SGPU_ERR_ARG;
    b->wait_cycles = cycles;
    return SGPU_OK;
}

sgpu_status sgpu_batch_set_wait_drill(sgpu_batch* b, int on) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b) return SGPU_ERR_ARG;
    b->wait_drill = on ? 1 : 0;
    return SGPU_OK;
}

sgpu_status sgpu_batch_set_kernel_family(sgpu_batch* b, int family) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b || family < 0 || family > 1) return SGPU_ERR_ARG;
    b->family = family;
    return SGPU_OK;
}

sgpu_status sgpu_batch_elapsed(sgpu_batch* b, int nsteps, float* ms) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b || !ms || nsteps < 0) return SGPU_ERR_ARG;
    sgpu_status s;
    drop_finished(b);
    if (b->dirty && (s = rebuild(b))) return s;
    if (nsteps >= kGraphSteps && (s = ensure_graph(b))) return s;
    BTRY(b, cudaEventRecord(b->ev0, b->stream));
    if ((s = advance(b, nsteps, true))) return s;
    BTRY(b, cudaEventRecord(b->ev1, b->stream));
    BTRY(b, cudaEventSynchronize(b->ev1));
    BTRY(b, cudaEventElapsedTime(ms, b->ev0, b->ev1));
    return check_err(b);
}

sgpu_status sgpu_batch_slot_info(const sgpu_batch* b, int slot, int* steps_done, int* steps_total, int* nprobes) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!valid_slot(b, slot)) return SGPU_ERR_ARG;
    const Slot& S = b->slots[slot];
    const int done = std::min(std::max(b->G - S.start, 0), S.nsteps + 1);
    if (steps_done) *steps_done = done;
    if (steps_total) *steps_total = S.nsteps + 1;
    if (nprobes) *nprobes = S.ctx->probes.n;
    return SGPU_OK;
}

sgpu_status sgpu_batch_read_probes(sgpu_batch* b, int slot, float* out, int max_rows, int* rows) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!valid_slot(b, slot) || !rows) return berr(b, SGPU_ERR_ARG, "bad probe read");
    const Slot& S = b->slots[slot];
    const int done = std::min(std::max(b->G - S.start, 0), S.nsteps + 1);
    const int take = std::min(done, max_rows);
    *rows = take;
    if (take <= 0 || S.ctx->probes.n == 0) return SGPU_OK;
    if (!out) return berr(b, SGPU_ERR_ARG, "null output");
    BTRY(b, cudaStreamSynchronize(b->stream));
    BTRY(b, cudaMemcpy(out, S.ctx->probes.ring, sizeof(float) * (size_t)take * S.ctx->probes.n, cudaMemcpyDeviceToHost));
    return SGPU_OK;
}

sgpu_status sgpu_batch_instance(sgpu_batch* b, int slot, sgpu_ctx** ctx) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!valid_slot(b, slot) || !ctx) return SGPU_ERR_ARG;
    BTRY(b, cudaStreamSynchronize(b->stream));
    *ctx = b->slots[slot].ctx;
    return SGPU_OK;
}

sgpu_status sgpu_batch_memory(sgpu_batch* b, uint64_t* capacity, uint64_t* in_use, uint64_t* largest_free) {
    if (!b) return SGPU_ERR_ARG;
    if (capacity) *capacity = b->arena.cap;
    if (in_use) {
        std::lock_guard<std::mutex> lock(b->arena.mu);
        *in_use = b->arena.in_use;
    }
    if (largest_free) *largest_free = arena_largest(&b->arena);
    return SGPU_OK;
}

sgpu_status sgpu_batch_set_tuning(sgpu_batch* b, const int* chunk3, int ctas_per_sm) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b) return SGPU_ERR_ARG;
    if (chunk3)
        for (int q = 0; q < kNumClasses; ++q) {
            if (chunk3[q] < 1 || chunk3[q] > 1024) return berr(b, SGPU_ERR_ARG, "z chunk out of range (1..1024)");
            if (b->chunk[q] != chunk3[q]) b->dirty = true;
            b->chunk[q] = chunk3[q];
        }
    if (ctas_per_sm) {
        if (ctas_per_sm < 1 || ctas_per_sm > 8) return berr(b, SGPU_ERR_ARG, "CTAs per SM out of range");
        b->ctas_per_sm = ctas_per_sm;
    }
    return SGPU_OK;
}

sgpu_status sgpu_batch_get_tuning(const sgpu_batch* b, int* chunk3, int* ctas_per_sm) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b) return SGPU_ERR_ARG;
    if (chunk3)
        for (int q = 0; q < kNumClasses; ++q) chunk3[q] = b->chunk[q];
    if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
    return SGPU_OK;
}

// Online autotuner: every trial advances the live instances by real steps
// (results do not depend on the launch shape), timed with CUDA events; the
// persistent grid size is chosen first, then each size class's z chunk by
// coordinate descent.
sgpu_status sgpu_batch_autotune(sgpu_batch* b, int steps_per_trial, int* chunk3, int* ctas_per_sm) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b || steps_per_trial < 1) return SGPU_ERR_ARG;
    sgpu_status s;
    auto trial = [&](float* ms) -> sgpu_status {
        sgpu_status r;
        drop_finished(b);
        if (b->dirty && (r = rebuild(b))) return r;
        if ((r = advance(b, 1, false))) return r;  // the first launch of a new shape is not timed
        BTRY(b, cudaEventRecord(b->ev0, b->stream));
        if ((r = advance(b, steps_per_trial, false))) return r;
        BTRY(b, cudaEventRecord(b->ev1, b->stream));
        BTRY(b, cudaEventSynchronize(b->ev1));
        BTRY(b, cudaEventElapsedTime(ms, b->ev0, b->ev1));
        return check_err(b);
    };
    bool present[kNumClasses] = {};
    for (const Slot& sl : b->slots)
        if (sl.ctx) present[sl.size_class] = true;
    float best = 0;
    int best_ctas = b->ctas_per_sm;
    for (int ctas : {2, 3, 4, 6}) {
        b->ctas_per_sm = ctas;
        float ms = 0;
        if ((s = trial(&ms))) return s;
        if (ctas == 2 || ms < best) {
            best = ms;
            best_ctas = ctas;
        }
    }
    b->ctas_per_sm = best_ctas;
    for (int cl = 0; cl < kNumClasses; ++cl) {
        if (!present[cl]) continue;
        // longest chunks first; a shorter one must win by 3 % (fewer items
        // cost less set-up, and a short trial is noisy)
        int best_chunk = b->chunk[cl];
        float best_ms = -1;
        for (int ch : {128, 64, 32, 16, 8}) {
            if (b->chunk[cl] != ch) b->dirty = true;
            b->chunk[cl] = ch;
            float ms = 0;
            if ((s = trial(&ms))) return s;
            if (best_ms < 0 || ms < 0.97f * best_ms) {
                best_ms = ms;
                best_chunk = ch;
            }
        }
        if (b->chunk[cl] != best_chunk) b->dirty = true;
        b->chunk[cl] = best_chunk;
    }
    if (chunk3)
        for (int q = 0; q < kNumClasses; ++q) chunk3[q] = b->chunk[q];
    if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
    return SGPU_OK;
}

// Device time of each phase summed over nsteps steps launched one by one
// (ms6: E field, ADE, E sources, H field, H sources + borders, probes + counter).
// The steps are real steps of the live instances.
sgpu_status sgpu_batch_profile_steps(sgpu_batch* b, int nsteps, float* ms6) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b || !ms6 || nsteps < 0) return SGPU_ERR_ARG;
    sgpu_status s = SGPU_OK;
    drop_finished(b);
    if (b->dirty && (s = rebuild(b))) return s;
    cudaEvent_t ev[7];
    for (auto& e : ev) BTRY(b, cudaEventCreate(&e));
    for (int q = 0; q < 6; ++q) ms6[q] = 0;
    for (int n = 0; n < nsteps && !s; ++n) {
        cudaEventRecord(ev[6], b->stream);
        if ((s = enqueue_step(b, ev))) break;
        b->G += 1;
        if (cudaEventSynchronize(ev[5]) != cudaSuccess) {
            s = berr(b, SGPU_ERR_CUDA, "profiled step failed");
            break;
        }
        float t;
        cudaEventElapsedTime(&t, ev[6], ev[0]);
        ms6[0] += t;
        for (int q = 1; q < 6; ++q) {
            cudaEventElapsedTime(&t, ev[q - 1], ev[q]);
            ms6[q] += t;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return s ? s : check_err(b);
}

sgpu_status sgpu_batch_steps(const sgpu_batch* b, int* counter) {
    if (!b) return SGPU_ERR_ARG;
    std::lock_guard<std::mutex> lock(b->mu);
    if (!b || !counter) return SGPU_ERR_ARG;
    *counter = b->G;
    return SGPU_OK;
}

}  // extern "C"
