// TMA-pipelined curl + CPML kernels (the fused fast path of the E and H half
// steps).  Included by kernels.cu; relies on its Slab/KGrid/KCpml helpers.
//
// Each CTA owns a 32 x 8 tile of (i, j) columns and marches a z chunk.  One
// producer warp streams every plane the tile needs -- the H (or E) tiles with
// their one-cell halos, the tile's own E (or H) values and the three int16
// media tiles -- into a 4-stage shared-memory ring with cp.async.bulk.tensor
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

namespace sgpu {

constexpr int kTX = 32, kTY = 8;          // tile (threads per row, rows)
constexpr int kStages = 4;                // shared-memory ring depth
constexpr int kConsumerWarps = kTY;       // one warp per tile row
constexpr int kTmaThreads = (kConsumerWarps + 1) * 32;
constexpr int kHaloW = kTX + 4;           // haloed row width (x rounded to 16 B)
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at the B200 clock

// byte sizes of the boxes and their 128-byte aligned slots in a stage
constexpr int kBoxA = kTX * (kTY + 1) * 4;      // 32 x 9 floats
constexpr int kBoxB = kHaloW * kTY * 4;         // 36 x 8 floats
constexpr int kBoxC = kHaloW * (kTY + 1) * 4;   // 36 x 9 floats
constexpr int kBoxF = kTX * kTY * 4;            // 32 x 8 floats
constexpr int kBoxM = kTX * kTY * 2;            // 32 x 8 int16
__host__ __device__ constexpr int align128(int b) { return (b + 127) / 128 * 128; }
constexpr int kOffA = 0;
constexpr int kOffB = kOffA + align128(kBoxA);
constexpr int kOffC = kOffB + align128(kBoxB);
constexpr int kOffF = kOffC + align128(kBoxC);
constexpr int kOffM = kOffF + 3 * align128(kBoxF);
constexpr int kStageBytes = kOffM + 3 * align128(kBoxM);
constexpr int kTmaSmem = kStages * kStageBytes + 2 * kStages * 8;
constexpr unsigned kTxFull = kBoxA + kBoxB + kBoxC + 3 * kBoxF + 3 * kBoxM;
constexpr unsigned kTxEdge = kBoxA + kBoxB;  // the extra plane: two arrays only

// TMaps holds the tensor maps in the order the kernels use them:
//   E kernel: Hx(32x9) Hy(36x8) Hz(36x9) Ex Ey Ez (32x8) Mx My Mz (32x8 int16)
//   H kernel: Ex(32x9) Ey(36x8) Ez(36x9) Hx Hy Hz (32x8) Mx My Mz (32x8 int16)

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
// Bounded wait; false (and an error code in *err) when the budget runs out.
__device__ __forceinline__ bool mbar_wait(unsigned a, unsigned parity, int* err, int code) {
    const long long t0 = clock64();
    while (!mbar_try(a, parity)) {
        if (clock64() - t0 > kWaitCycles) {
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

// Shared set-up of the two kernels: barriers, coefficient tables, geometry.
struct TmaCta {
    unsigned char* ring;
    unsigned full0, empty0;  // shared addresses of the barrier arrays
    int ib, jb, kb, ke;
    int warp, lane;
};

__device__ __forceinline__ TmaCta tma_cta_setup(unsigned char* smem, int y0, int z0, int z1, int zchunk) {
    TmaCta t;
    t.ring = smem;
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

// Producer: planes p0 .. p1 into the ring; `edge` is the plane that carries
// only the first two arrays (the E kernel's k-1 plane, the H kernel's k+1).
__device__ __forceinline__ void tma_produce(const TmaCta& t, const TMaps& tm, int p0, int p1, int edge, int* err) {
    if (t.lane != 0) return;
    int issued = 0;
    bool ok = true;
    for (int p = p0; p <= p1 && ok; ++p) {
        const int pidx = p - p0, s = pidx % kStages, u = pidx / kStages;
        if (u >= 1 && !mbar_wait(t.empty0 + 8 * s, (u - 1) & 1, err, 11)) { ok = false; break; }
        const unsigned bar = t.full0 + 8 * s;
        unsigned char* st = t.ring + s * kStageBytes;
        const bool part = p == edge;
        mbar_expect_tx(bar, part ? kTxEdge : kTxFull);
        tma_load3(smem_u32(st + kOffA), &tm.m[0], t.ib, t.jb - 1, p, bar);  // first array (halo in y)
        tma_load3(smem_u32(st + kOffB), &tm.m[1], t.ib - 4, t.jb, p, bar);  // second (halo in x)
        if (!part) {
            tma_load3(smem_u32(st + kOffC), &tm.m[2], t.ib - 4, t.jb - 1, p, bar);
            for (int q = 0; q < 3; ++q) tma_load3(smem_u32(st + kOffF + q * align128(kBoxF)), &tm.m[3 + q], t.ib, t.jb, p, bar);
            for (int q = 0; q < 3; ++q) tma_load3(smem_u32(st + kOffM + q * align128(kBoxM)), &tm.m[6 + q], t.ib, t.jb, p, bar);
        }
        ++issued;
    }
    // nothing may be in flight into this CTA's shared memory when it exits
    const int first = issued > kStages ? issued - kStages : 0;
    for (int pidx = first; pidx < issued; ++pidx)
        mbar_wait(t.full0 + 8 * (pidx % kStages), (pidx / kStages) & 1, err, 12);
}

// The H kernel's tiles start at x = ib (no -x halo) and its y halo is +1, so
// its maps are encoded with those origins; the producer passes coordinates
// through these two helpers.
__device__ __forceinline__ void tma_produce_h(const TmaCta& t, const TMaps& tm, int p0, int p1, int edge, int* err) {
    if (t.lane != 0) return;
    int issued = 0;
    bool ok = true;
    for (int p = p0; p <= p1 && ok; ++p) {
        const int pidx = p - p0, s = pidx % kStages, u = pidx / kStages;
        if (u >= 1 && !mbar_wait(t.empty0 + 8 * s, (u - 1) & 1, err, 13)) { ok = false; break; }
        const unsigned bar = t.full0 + 8 * s;
        unsigned char* st = t.ring + s * kStageBytes;
        const bool part = p == edge;
        mbar_expect_tx(bar, part ? kTxEdge : kTxFull);
        tma_load3(smem_u32(st + kOffA), &tm.m[0], t.ib, t.jb, p, bar);  // Ex rows jb..jb+8
        tma_load3(smem_u32(st + kOffB), &tm.m[1], t.ib, t.jb, p, bar);  // Ey x ib..ib+35
        if (!part) {
            tma_load3(smem_u32(st + kOffC), &tm.m[2], t.ib, t.jb, p, bar);  // Ez x ib..ib+35, rows jb..jb+8
            for (int q = 0; q < 3; ++q) tma_load3(smem_u32(st + kOffF + q * align128(kBoxF)), &tm.m[3 + q], t.ib, t.jb, p, bar);
            for (int q = 0; q < 3; ++q) tma_load3(smem_u32(st + kOffM + q * align128(kBoxM)), &tm.m[6 + q], t.ib, t.jb, p, bar);
        }
        ++issued;
    }
    const int first = issued > kStages ? issued - kStages : 0;
    for (int pidx = first; pidx < issued; ++pidx)
        mbar_wait(t.full0 + 8 * (pidx % kStages), (pidx / kStages) & 1, err, 14);
}

}  // namespace sgpu
