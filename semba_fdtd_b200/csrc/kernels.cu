// libsemba_gpu: device kernels and the level-1 C ABI (see include/semba_gpu.h).
//
// The per-cell arithmetic restates the reference routines named beside each
// kernel, in their operation order, so that a build with -fmad=false
// reproduces the reference FP32 build bit for bit.  All transcendental work
// (exp, log, pow, trig) happens once on the host during set-up; kernels only
// add, subtract, multiply, divide and convert, which CUDA performs with IEEE
// round-to-nearest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <complex>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "sgpu_internal.h"
#include "stencil.cuh"
#include "tma_fields.cuh"

using namespace sgpu;
using namespace sgpu::dev;

namespace sgpu {

sgpu_status set_error(sgpu_ctx* c, sgpu_status code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

KGrid kgrid(const sgpu_ctx* c) {
    KGrid g{};
    for (int f = 0; f < 6; ++f) {
        g.F[f] = c->F[f];
        g.M[f] = c->M[f];
        g.sw[f][0] = c->sweep[f].xi - c->ox;
        g.sw[f][1] = c->sweep[f].xe - c->ox;
        g.sw[f][2] = c->sweep[f].yi - c->oy;
        g.sw[f][3] = c->sweep[f].ye - c->oy;
        g.sw[f][4] = c->sweep[f].zi - c->oz;
        g.sw[f][5] = c->sweep[f].ze - c->oz;
    }
    g.g1 = c->g1; g.g2 = c->g2; g.gm1 = c->gm1; g.gm2 = c->gm2;
    g.idxe = c->idxe; g.idye = c->idye; g.idze = c->idze;
    g.idxh = c->idxh; g.idyh = c->idyh; g.idzh = c->idzh;
    g.pitch = c->pitch;
    g.plane = c->plane;
    g.nmed1 = c->num_media + 1;
    return g;
}

}  // namespace sgpu

#define CUDA_TRY(ctx, call)                                                                   \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return set_error((ctx), SGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

template <int MODE>
__global__ void __launch_bounds__(kBX * kBY, 4) k_efield(KGrid g, KCpml cp, int y0, int z0, int z1, int zchunk) {
    extern __shared__ float sh[];
    const bool use_sh = g.nmed1 <= kShTable;
    if (use_sh) {
        for (int t = threadIdx.x + kBX * threadIdx.y; t < g.nmed1; t += kBX * kBY) {
            sh[t] = g.g1[t];
            sh[g.nmed1 + t] = g.g2[t];
        }
    }
    __syncthreads();
    const float* t1 = use_sh ? sh : g.g1;
    const float* t2 = use_sh ? sh + g.nmed1 : g.g2;
    const int i = blockIdx.x * kBX + threadIdx.x;
    const int jb = y0 + blockIdx.y * kBY;
    const int j = jb + threadIdx.y;
    const int kb = z0 + blockIdx.z * zchunk;
    const int ke = min(kb + zchunk - 1, z1);
    // the warp shuffles need every lane: out-of-range lanes stay in the loop
    // with all three components disabled and clamped (in-bounds) indices
    const bool vx = col_in(g.sw[0], i, j), vy = col_in(g.sw[1], i, j), vz = col_in(g.sw[2], i, j);
    // i < pitch always (grid rounding stays inside the padded row); rows
    // past the last swept row are clamped to a valid one and do no work
    const int ic = i;
    const int jc = min(max(j, 1), (int)(g.plane / g.pitch) - 2);
    bool cpml_block = false;
    if (MODE & kCpml) {
        const int bx0 = blockIdx.x * kBX, bx1 = bx0 + kBX - 1, by1 = jb + kBY - 1;
        for (int f = 0; f < 3; ++f)
            for (int w = 0; w < 2; ++w)
                for (int sd = 0; sd < 2; ++sd) cpml_block |= slab_touches(cp.s[f][w][sd], bx0, bx1, jb, by1, kb, ke);
    }
    if (cpml_block) efield_column<MODE, true>(g, cp, t1, t2, ic, jc, kb, ke, vx, vy, vz);
    else if (MODE & kBulk) efield_column<MODE, false>(g, cp, t1, t2, ic, jc, kb, ke, vx, vy, vz);
}

template <int MODE>
__global__ void __launch_bounds__(kBX * kBY, 4) k_hfield(KGrid g, KCpml cp, int y0, int z0, int z1, int zchunk) {
    extern __shared__ float sh[];
    const bool use_sh = g.nmed1 <= kShTable;
    if (use_sh) {
        for (int t = threadIdx.x + kBX * threadIdx.y; t < g.nmed1; t += kBX * kBY) {
            sh[t] = g.gm1[t];
            sh[g.nmed1 + t] = g.gm2[t];
        }
    }
    __syncthreads();
    const float* t1 = use_sh ? sh : g.gm1;
    const float* t2 = use_sh ? sh + g.nmed1 : g.gm2;
    const int i = blockIdx.x * kBX + threadIdx.x;
    const int jb = y0 + blockIdx.y * kBY;
    const int j = jb + threadIdx.y;
    const int kb = z0 + blockIdx.z * zchunk;
    const int ke = min(kb + zchunk - 1, z1);
    const bool vx = col_in(g.sw[3], i, j), vy = col_in(g.sw[4], i, j), vz = col_in(g.sw[5], i, j);
    // i < pitch always (grid rounding stays inside the padded row); rows
    // past the last swept row are clamped to a valid one and do no work
    const int ic = i;
    const int jc = min(max(j, 1), (int)(g.plane / g.pitch) - 2);
    bool cpml_block = false;
    if (MODE & kCpml) {
        const int bx0 = blockIdx.x * kBX, bx1 = bx0 + kBX - 1, by1 = jb + kBY - 1;
        for (int f = 3; f < 6; ++f)
            for (int w = 0; w < 2; ++w)
                for (int sd = 0; sd < 2; ++sd) cpml_block |= slab_touches(cp.s[f][w][sd], bx0, bx1, jb, by1, kb, ke);
    }
    if (cpml_block) hfield_column<MODE, true>(g, cp, t1, t2, ic, jc, kb, ke, vx, vy, vz);
    else if (MODE & kBulk) hfield_column<MODE, false>(g, cp, t1, t2, ic, jc, kb, ke, vx, vy, vz);
}

// ---------------------------------------------------------------------------
// TMA-pipelined fused kernels (fast path of the E and H half steps).
// Same per-cell arithmetic as efield_column / hfield_column, from shared
// memory instead of global loads.

#ifndef SGPU_TMA_MINB
#define SGPU_TMA_MINB 4
#endif
constexpr int kTmaMinBlocks = SGPU_TMA_MINB;  // CTAs an SM holds of the plain TMA field kernels

// The side's coefficient pairs (G1, G2) or (GM1, GM2) in shared memory after
// the ring; the TMA kernels run only with fewer than 256 media, so the table
// always fits (the launch sizes the shared memory for it).
__device__ __forceinline__ TabPairs tma_tables(unsigned char* smem, const float* a, const float* b, int nmed1) {
    float2* tab = (float2*)(smem + kTmaSmem);
    for (int q = threadIdx.x; q < nmed1; q += blockDim.x) tab[q] = make_float2(a[q], b[q]);
    return TabPairs{tab};
}

__global__ void __launch_bounds__(kTmaThreads, kTmaMinBlocks)
    k_tma_efield(KGrid g, KCpml cp, const __grid_constant__ TMaps tm, int y0, int z0, int z1, int zchunk, int* err,
                 long long wait, int drill) {
    extern __shared__ __align__(128) unsigned char smem[];
    const TabPairs tab = tma_tables(smem, g.g1, g.g2, g.nmed1);
    const TmaCta t = tma_cta_setup(smem, y0, z0, z1, zchunk, wait);
    bool cpml_block = false;
    if (cp.on)
        for (int f = 0; f < 3; ++f)
            for (int w = 0; w < 2; ++w)
                for (int sd = 0; sd < 2; ++sd)
                    cpml_block |= slab_touches(cp.s[f][w][sd], t.ib, t.ib + kTX - 1, t.jb, t.jb + kTY - 1, t.kb, t.ke);
    const unsigned tmask = cpml_block ? cpml_tile_mask(cp, 0, t.ib, t.ib + kTX - 1, t.jb, t.jb + kTY - 1) : 0u;
    const unsigned smask = cpml_block ? staged_mask(cp, 0, t.ib, t.jb) : 0u;
    if (t.warp == kConsumerWarps) {
        if (drill) return;  // a failure drill: no plane arrives, every consumer wait runs out
        __shared__ ProdTable tb;
        prod_prepare(&tb, t, t.kb - 1, t.ke, t.kb - 1, false, g, cp, tmask);
        if (t.lane == 0) tma_drain(t, (unsigned)tma_issue(t, tm.m, 0, t.kb - 1, t.ke, t.kb - 1, false, err, &tb, smask), err, 12);
        return;
    }
    __shared__ PsiRow rows[kConsumerWarps][12];
    if (smask) e_consume<2>(t, 0, g, cp, tab, err, false, rows[t.warp]);
    else if (cpml_block) e_consume<1>(t, 0, g, cp, tab, err, false, rows[t.warp]);
    else e_consume<0>(t, 0, g, cp, tab, err, false, rows[t.warp]);
}

__global__ void __launch_bounds__(kTmaThreads, kTmaMinBlocks)
    k_tma_hfield(KGrid g, KCpml cp, const __grid_constant__ TMaps tm, int y0, int z0, int z1, int zchunk, int* err,
                 long long wait, int drill) {
    extern __shared__ __align__(128) unsigned char smem[];
    const TabPairs tab = tma_tables(smem, g.gm1, g.gm2, g.nmed1);
    const TmaCta t = tma_cta_setup(smem, y0, z0, z1, zchunk, wait);
    bool cpml_block = false;
    if (cp.on)
        for (int f = 3; f < 6; ++f)
            for (int w = 0; w < 2; ++w)
                for (int sd = 0; sd < 2; ++sd)
                    cpml_block |= slab_touches(cp.s[f][w][sd], t.ib, t.ib + kTX - 1, t.jb, t.jb + kTY - 1, t.kb, t.ke);
    const unsigned tmask = cpml_block ? cpml_tile_mask(cp, 3, t.ib, t.ib + kTX - 1, t.jb, t.jb + kTY - 1) : 0u;
    const unsigned smask = cpml_block ? staged_mask(cp, 3, t.ib, t.jb) : 0u;
    if (t.warp == kConsumerWarps) {
        if (drill) return;  // a failure drill: no plane arrives, every consumer wait runs out
        __shared__ ProdTable tb;
        prod_prepare(&tb, t, t.kb, t.ke + 1, t.ke + 1, true, g, cp, tmask);
        if (t.lane == 0) tma_drain(t, (unsigned)tma_issue(t, tm.m, 0, t.kb, t.ke + 1, t.ke + 1, true, err, &tb, smask), err, 14);
        return;
    }
    __shared__ PsiRow rows[kConsumerWarps][12];
    if (smask) h_consume<2>(t, 0, g, cp, tab, err, false, rows[t.warp]);
    else if (cpml_block) h_consume<1>(t, 0, g, cp, tab, err, false, rows[t.warp]);
    else h_consume<0>(t, 0, g, cp, tab, err, false, rows[t.warp]);
}

// One node a thread, 128-thread blocks, 12 blocks an SM (40 registers).
constexpr int kAdeBlock = 128;
template <int NU, bool MAG, bool UNI>
__global__ void __launch_bounds__(kAdeBlock, 12) k_ade(KGrid g, KDisp d, int comp) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q < d.n[comp]) ade_node<NU, MAG, UNI>(ade_refs<MAG>(g, d, comp), q);
}


// AdvancePlaneWaveE/H (planewaves.F90:878-1475) with Incid/evolucion
// (:778-853) and AdvanceNodalE/H (nodalsources.F90:310-777): one thread per
// touched node applies that node's contributions in the reference order.
__global__ void k_sources(KGrid g, KSrc s, StepRef sr, const double* tiempo, int t_n0, double dt, int hside, int mask) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = step_of(sr);
    const bool pw_on = (mask & (1 << kSrcPlaneWave)) ? pw_switch_block(s, n, tiempo, t_n0, dt, hside) : false;
    // with the switch down a row of plane-wave contributions alone changes
    // nothing: the reference calls no plane-wave routine then
    if (s.pw_only && !pw_on) return;
    if (r < s.nrows) source_row(g, s, n, tiempo, t_n0, dt, hside, mask, r, pw_on);
}

// UpdateObservation point probes (observation.F90:2633-2668).
__global__ void k_probes(KGrid g, KProbes p, StepRef sr, int first_n) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < p.n) probe_one(g, p, step_of(sr), first_n, q);
}

// Volume probes, one thread per sampled node (all three components).
// FREQ: the frequency-domain accumulation of observation.F90:3527-3600,
// V = V + w * F in complex(8) per frequency, component and node; else the
// node's three values go into the frame of step n.
template <bool FREQ>
__global__ void k_vol_probe(KGrid g, VolProbe p, StepRef sr, int ox, int oy, int oz) {
    const long long nodes = (long long)p.ni * p.nj * p.nk;
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= nodes) return;
    const int n = step_of(sr);
    const int ii = (int)(q % p.ni), jj = (int)((q / p.ni) % p.nj), kk = (int)(q / ((long long)p.ni * p.nj));
    const long long c = (long long)((p.i0 + ii) * p.tr[0] - ox) + (long long)g.pitch * ((p.j0 + jj) * p.tr[1] - oy) +
                        g.plane * (long long)((p.k0 + kk) * p.tr[2] - oz);
    const int f0 = p.magnetic ? 3 : 0;
    const float v[3] = {g.F[f0][c], g.F[f0 + 1][c], g.F[f0 + 2][c]};
    if (FREQ) {
        const int m = n - p.w_n0;
        if (m < 0 || m >= p.w_steps) return;
        for (int f = 0; f < p.nf; ++f) {
            const double2 w = p.w[(long long)m * p.nf + f];
            for (int comp = 0; comp < 3; ++comp) {
                double2* a = p.acc + (((long long)f * 3 + comp) * nodes + q);
                double2 x = *a;
                x.x = x.x + w.x * (double)v[comp];
                x.y = x.y + w.y * (double)v[comp];
                *a = x;
            }
        }
    } else {
        if (n < p.n_first || n >= p.n_last || (n - p.n_first) % p.every) return;
        const long long slot = (long long)((n - p.n_first) / p.every) % p.cap;
        for (int comp = 0; comp < 3; ++comp) p.ring[(slot * 3 + comp) * nodes + q] = v[comp];
    }
}

// MinusCloneMagneticPMC / CloneMagneticPeriodic (bordersother.F90:65-190)
// for the face kinds in `mask`, and AdvanceMagneticMUR (bordersmur.F90:502).
__global__ void k_clone_h(KGrid g, KBorder b, int mask) {
    clone_cell(g, b, mask, blockIdx.x * (long long)blockDim.x + threadIdx.x);
}
__global__ void k_mur_h(KGrid g, KBorder b) { mur_cell(g, b, blockIdx.x * (long long)blockDim.x + threadIdx.x); }

__global__ void k_fill_i16(int16_t* p, long long n, int v) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        p[q] = (int16_t)v;
}
// The one-byte copy of a media matrix (indices below 256).
__global__ void k_narrow_media(const int16_t* M, uint8_t* M8, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        M8[q] = (uint8_t)M[q];
}
__global__ void k_set_step(int* d, int v) { *d = v; }
__global__ void k_add_step(int* d, int v) { *d += v; }

__global__ void k_count_disp(const int16_t* M, const int16_t* slot, int pitch, long long plane, int x0, int x1, int y0,
                             int y1, int z0, int z1, int* counts) {
    const long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int ny = y1 - y0 + 1, nz = z1 - z0 + 1;
    if (row >= (long long)ny * nz) return;
    const int j = y0 + (int)(row % ny), k = z0 + (int)(row / ny);
    int cnt = 0;
    const long long base = (long long)pitch * j + plane * k;
    for (int i = x0; i <= x1; ++i) cnt += slot[M[base + i]] >= 0;
    counts[row] = cnt;
}

__global__ void k_fill_disp(const int16_t* M, const int16_t* slot, int pitch, long long plane, int x0, int x1, int y0,
                            int y1, int z0, int z1, const long long* offs, int* node, uint8_t* med) {
    const long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int ny = y1 - y0 + 1, nz = z1 - z0 + 1;
    if (row >= (long long)ny * nz) return;
    const int j = y0 + (int)(row % ny), k = z0 + (int)(row / ny);
    long long o = offs[row];
    const long long base = (long long)pitch * j + plane * k;
    for (int i = x0; i <= x1; ++i) {
        const int s = slot[M[base + i]];
        if (s >= 0) {
            node[o] = (int)(base + i);
            med[o] = (uint8_t)s;
            ++o;
        }
    }
}

// The run descriptors of the node groups (32 consecutive nodes each): a run
// is a stretch of nodes on consecutive cells with one medium slot.  Groups of
// more than two runs get z = -1 and are counted in *irregular.
__global__ void k_fill_grp(const int* node, const uint8_t* med, long long n, int4* grp, unsigned long long* irregular) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long q0 = g * 32;
    if (q0 >= n) return;
    const int cnt = (int)min(32LL, n - q0);
    int runs = 1, lane1 = 32;
    for (int l = 1; l < cnt; ++l)
        if (node[q0 + l] != node[q0 + l - 1] + 1 || med[q0 + l] != med[q0 + l - 1]) {
            if (++runs == 2) lane1 = l;
        }
    int4 d;
    if (runs > 2) {
        d = make_int4(0, 0, -1, 0);
        atomicAdd(irregular, 1ULL);
    } else {
        const int l1 = lane1 < cnt ? lane1 : cnt - 1;
        d = make_int4(node[q0], node[q0 + l1] - lane1, lane1, (int)med[q0] | ((int)med[q0 + l1] << 8));
        if (lane1 >= 32) d.y = d.x;  // one run: the second never applies
    }
    grp[g] = d;
}

__global__ void k_nonfinite(const float* a, long long n, unsigned int* flag) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        if (!isfinite(a[q])) {
            atomicOr(flag, 1u);
            return;
        }
}

int zchunk_for(int nz, int blocks_xy) {
    // short chunks: many waves of blocks on 148 SMs, so the last partial wave
    // costs little; 16 planes keep the carried k-1 plane worthwhile
    int chunk = 16;
    while (chunk > 4 && (long long)blocks_xy * ((nz + chunk - 1) / chunk) < 148LL * 4) chunk /= 2;
    return std::min(chunk, nz);
}

struct Launch {
    dim3 grid, block;
    int y0, z0, z1, zchunk;
    size_t smem;
};

Launch plan(const sgpu_ctx* c, int c0, int c1) {
    int x1 = -1, y0 = 1 << 30, y1 = -1, z0 = 1 << 30, z1 = -1;
    for (int f = c0; f <= c1; ++f) {
        x1 = std::max(x1, c->sweep[f].xe - c->ox);
        y0 = std::min(y0, c->sweep[f].yi - c->oy); y1 = std::max(y1, c->sweep[f].ye - c->oy);
        z0 = std::min(z0, c->sweep[f].zi - c->oz); z1 = std::max(z1, c->sweep[f].ze - c->oz);
    }
    Launch L;
    L.block = dim3(kBX, kBY, 1);
    int bx = (x1 + 1 + kBX - 1) / kBX, by = (y1 - y0 + 1 + kBY - 1) / kBY;
    int nz = z1 - z0 + 1;
    L.zchunk = zchunk_for(nz, bx * by);
    L.grid = dim3(bx, by, (nz + L.zchunk - 1) / L.zchunk);
    L.y0 = y0; L.z0 = z0; L.z1 = z1;
    const int n1 = c->num_media + 1;
    L.smem = n1 <= kShTable ? 2 * n1 * sizeof(float) : 0;
    return L;
}

sgpu_status check_launch(sgpu_ctx* c, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(c, SGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return SGPU_OK;
}

template <int MODE> sgpu_status launch_e(sgpu_ctx* c) {
    Launch L = plan(c, 0, 2);
    k_efield<MODE><<<L.grid, L.block, L.smem, c->stream>>>(kgrid(c), c->cpml, L.y0, L.z0, L.z1, L.zchunk);
    return check_launch(c, "k_efield");
}
template <int MODE> sgpu_status launch_h(sgpu_ctx* c) {
    Launch L = plan(c, 3, 5);
    k_hfield<MODE><<<L.grid, L.block, L.smem, c->stream>>>(kgrid(c), c->cpml, L.y0, L.z0, L.z1, L.zchunk);
    return check_launch(c, "k_hfield");
}

// planes per CTA of the TMA field kernels (halved on small grids until the
// grid has four CTAs per SM)
#ifndef SGPU_TMA_CHUNK
#define SGPU_TMA_CHUNK 64
#endif
constexpr int kTmaChunk = SGPU_TMA_CHUNK;

sgpu_status launch_tma(sgpu_ctx* c, bool hside) {
    Launch L = plan(c, hside ? 3 : 0, hside ? 5 : 2);
    int x1 = -1;
    for (int f = hside ? 3 : 0; f < (hside ? 6 : 3); ++f) x1 = std::max(x1, c->sweep[f].xe - c->ox);
    const int bx = (x1 + 1 + kTX - 1) / kTX;
    int y1 = -1;
    for (int f = hside ? 3 : 0; f < (hside ? 6 : 3); ++f) y1 = std::max(y1, c->sweep[f].ye - c->oy);
    const int by = (y1 - L.y0 + 1 + kTY - 1) / kTY;
    const int nz = L.z1 - L.z0 + 1;
    int chunk = kTmaChunk;
    while (chunk > 8 && (long long)bx * by * ((nz + chunk - 1) / chunk) < 148LL * 4) chunk /= 2;
    chunk = std::min(chunk, nz);
    dim3 grid(bx, by, (nz + chunk - 1) / chunk);
    const int n1 = c->num_media + 1;
    const size_t smem = kTmaSmem + n1 * sizeof(float2);  // n1 <= 256: tma_usable
    if (hside)
        k_tma_hfield<<<grid, kTmaThreads, smem, c->stream>>>(kgrid(c), c->cpml, c->tmh, L.y0, L.z0, L.z1, chunk, c->d_err,
                                                             c->wait_cycles, c->wait_drill);
    else
        k_tma_efield<<<grid, kTmaThreads, smem, c->stream>>>(kgrid(c), c->cpml, c->tme, L.y0, L.z0, L.z1, chunk, c->d_err,
                                                             c->wait_cycles, c->wait_drill);
    return check_launch(c, hside ? "k_tma_hfield" : "k_tma_efield");
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                 const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
    // looked up once; a function-local static is initialised once even when
    // several host threads set up contexts at the same time
    static const EncodeTiled fn = []() -> EncodeTiled {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        EncodeTiled f = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            f = (EncodeTiled)p;
        cudaGetLastError();
        return f;
    }();
    return fn;
}

// A 3-D tiled map over one padded array with a (bx, by, 1) box.
bool encode_map(const sgpu_ctx* c, CUtensorMap* m, void* base, bool bytes, int bx, int by) {
    EncodeTiled fn = encoder();
    if (!fn) return false;
    const cuuint64_t esz = bytes ? 1 : 4;
    const cuuint64_t dims[3] = {(cuuint64_t)c->pitch, (cuuint64_t)c->nya, (cuuint64_t)c->nza};
    const cuuint64_t strides[2] = {(cuuint64_t)c->pitch * esz, (cuuint64_t)c->plane * esz};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(m, bytes ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// A psi slab as a 3-D tiled map with a 32 x 8 x 1 box (rows of px floats).
bool encode_psi_map(CUtensorMap* m, const Slab& sl) {
    EncodeTiled fn = encoder();
    if (!fn) return false;
    const cuuint64_t ny = (cuuint64_t)(sl.yhi - sl.ylo + 1), nz = (cuuint64_t)(sl.zhi - sl.zlo + 1);
    const cuuint64_t dims[3] = {(cuuint64_t)sl.px, ny, nz};
    const cuuint64_t strides[2] = {(cuuint64_t)sl.px * 4, (cuuint64_t)sl.px * ny * 4};
    const cuuint32_t box[3] = {(cuuint32_t)kTX, (cuuint32_t)kTY, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, sl.psi, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool build_tensor_maps(sgpu_ctx* c) {
    bool ok = true;
    // E kernel: Hx (32x9), Hy (36x8), Hz (36x9), Ex Ey Ez, Mx My Mz
    ok = ok && encode_map(c, &c->tme.m[0], c->F[3], false, kTX, kTY + 1);
    ok = ok && encode_map(c, &c->tme.m[1], c->F[4], false, kHaloW, kTY);
    ok = ok && encode_map(c, &c->tme.m[2], c->F[5], false, kHaloW, kTY + 1);
    // H kernel: Ex (32x9), Ey (36x8), Ez (36x9), Hx Hy Hz, MHx MHy MHz
    ok = ok && encode_map(c, &c->tmh.m[0], c->F[0], false, kTX, kTY + 1);
    ok = ok && encode_map(c, &c->tmh.m[1], c->F[1], false, kHaloW, kTY);
    ok = ok && encode_map(c, &c->tmh.m[2], c->F[2], false, kHaloW, kTY + 1);
    for (int q = 0; q < 3; ++q) {
        ok = ok && encode_map(c, &c->tme.m[3 + q], c->F[q], false, kTX, kTY);
        ok = ok && encode_map(c, &c->tme.m[6 + q], c->M8[q], true, kTX, kTY);
        ok = ok && encode_map(c, &c->tmh.m[3 + q], c->F[3 + q], false, kTX, kTY);
        ok = ok && encode_map(c, &c->tmh.m[6 + q], c->M8[3 + q], true, kTX, kTY);
    }
    return ok;
}

bool ready(sgpu_ctx* c) {
    for (int f = 0; f < 6; ++f)
        if (!c->media_loaded[f]) return false;
    return true;
}

sgpu_status build_sources(sgpu_ctx* c);

template <int NU, bool MAG> void ade_launch(sgpu_ctx* c, int comp, unsigned blocks) {
    const KDisp& d = MAG ? c->mdisp : c->disp;
    if (d.uniform && d.nu_max == NU) k_ade<NU, MAG, true><<<blocks, kAdeBlock, 0, c->stream>>>(kgrid(c), d, comp);
    else k_ade<NU, MAG, false><<<blocks, kAdeBlock, 0, c->stream>>>(kgrid(c), d, comp);
}

template <bool MAG> sgpu_status launch_ade_side(sgpu_ctx* c) {
    const KDisp& d = MAG ? c->mdisp : c->disp;
    if (!(MAG ? c->mdisp_on : c->disp_on)) return SGPU_OK;
    for (int comp = 0; comp < 3; ++comp) {
        long long n = d.n[comp];
        if (n == 0) continue;
        const unsigned blocks = (unsigned)((n + kAdeBlock - 1) / kAdeBlock);
        switch (d.nu_max) {
            case 1: ade_launch<1, MAG>(c, comp, blocks); break;
            case 2: ade_launch<2, MAG>(c, comp, blocks); break;
            case 3: ade_launch<3, MAG>(c, comp, blocks); break;
            case 4: ade_launch<4, MAG>(c, comp, blocks); break;
            default: ade_launch<kMaxPolesPerMedium, MAG>(c, comp, blocks); break;
        }
        sgpu_status s = check_launch(c, "k_ade");
        if (s) return s;
    }
    return SGPU_OK;
}

sgpu_status launch_edisp(sgpu_ctx* c) { return launch_ade_side<false>(c); }
sgpu_status launch_mdisp(sgpu_ctx* c) { return launch_ade_side<true>(c); }

constexpr int kMaskPW = 1 << kSrcPlaneWave, kMaskNodal = (1 << kSrcNodalSoft) | (1 << kSrcNodalHard),
              kMaskAll = kMaskPW | kMaskNodal;

// The first half step run fixes where the plane-wave switch starts up.
void note_first_half(sgpu_ctx* c, int h) {
    if (c->h_first >= 0) return;
    c->h_first = h;
    c->src[0].h_first = c->src[1].h_first = h;
}

sgpu_status launch_sources(sgpu_ctx* c, int side, StepRef sr, int mask = kMaskAll) {
    if (c->src_dirty) {
        sgpu_status s = build_sources(c);
        if (s) return s;
    }
    if (!sr.dev_n) note_first_half(c, 2 * sr.n + side);
    const KSrc& k = c->src[side];
    if (k.nrows == 0) return SGPU_OK;
    if (!c->d_tiempo) return set_error(c, SGPU_ERR_STATE, "time vector not set (sgpu_set_time)");
    if (!sr.dev_n && (sr.n < c->t_n0 || sr.n >= c->t_n0 + c->d_tiempo_count))
        return set_error(c, SGPU_ERR_ARG, "step outside the time vector");
    int threads = 128;
    int blocks = (k.nrows + threads - 1) / threads;
    k_sources<<<blocks, threads, 0, c->stream>>>(kgrid(c), k, sr, c->d_tiempo, c->t_n0, c->dt, side, mask);
    return check_launch(c, "k_sources");
}

sgpu_status launch_probes(sgpu_ctx* c, StepRef sr) {
    if (!c->farfields.empty()) {
        sgpu_status s = launch_farfields(c, sr);
        if (s) return s;
    }
    for (const VolProbe& p : c->vprobes) {
        const long long nodes = (long long)p.ni * p.nj * p.nk;
        const unsigned blocks = (unsigned)((nodes + 255) / 256);
        if (p.kind == 0) k_vol_probe<true><<<blocks, 256, 0, c->stream>>>(kgrid(c), p, sr, c->ox, c->oy, c->oz);
        else k_vol_probe<false><<<blocks, 256, 0, c->stream>>>(kgrid(c), p, sr, c->ox, c->oy, c->oz);
        sgpu_status s = check_launch(c, "k_vol_probe");
        if (s) return s;
    }
    if (c->probes.n == 0) return SGPU_OK;
    int threads = 128;
    int blocks = (c->probes.n + threads - 1) / threads;
    k_probes<<<blocks, threads, 0, c->stream>>>(kgrid(c), c->probes, sr, c->probe_first_n);
    return check_launch(c, "k_probes");
}

bool has_clone(const sgpu_ctx* c, int mask) {
    for (int a = 0; a < 3; ++a)
        for (int sd = 0; sd < 2; ++sd)
            if (c->border.face_kind[a][sd] & mask) return true;
    return false;
}

sgpu_status launch_clone(sgpu_ctx* c, int mask) {
    if (c->border.cl_cells == 0 || !has_clone(c, mask)) return SGPU_OK;
    const unsigned blocks = (unsigned)((c->border.cl_cells + 255) / 256);
    k_clone_h<<<blocks, 256, 0, c->stream>>>(kgrid(c), c->border, mask);
    return check_launch(c, "k_clone_h");
}

sgpu_status launch_mur(sgpu_ctx* c) {
    if (c->border.mur_cells == 0) return SGPU_OK;
    const unsigned blocks = (unsigned)((c->border.mur_cells + 255) / 256);
    k_mur_h<<<blocks, 256, 0, c->stream>>>(kgrid(c), c->border);
    return check_launch(c, "k_mur_h");
}

// The H-side borders after the H sources: both clone kinds in one launch
// (PMC, then periodic, composed per cell), then Mur.
sgpu_status launch_borders_h(sgpu_ctx* c) {
    sgpu_status s = launch_clone(c, 6);
    if (s) return s;
    return launch_mur(c);
}

sgpu_status field_e(sgpu_ctx* c) {
    if (c->family == 1 && tma_usable(c)) return launch_tma(c, false);
    return c->cpml.on ? launch_e<kBulk | kCpml | kAll>(c) : launch_e<kBulk | kAll>(c);
}

sgpu_status field_h(sgpu_ctx* c) {
    if (c->family == 1 && tma_usable(c)) return launch_tma(c, true);
    return c->cpml.on ? launch_h<kBulk | kCpml | kAll>(c) : launch_h<kBulk | kAll>(c);
}

sgpu_status half_e(sgpu_ctx* c, StepRef sr) {
    sgpu_status s = field_e(c);
    if (s) return s;
    if ((s = launch_edisp(c))) return s;
    return launch_sources(c, 0, sr);
}

sgpu_status half_h(sgpu_ctx* c, StepRef sr) {
    sgpu_status s = field_h(c);
    if (s) return s;
    if ((s = launch_mdisp(c))) return s;
    if ((s = launch_sources(c, 1, sr))) return s;
    return launch_borders_h(c);
}

sgpu_status whole_step(sgpu_ctx* c, StepRef sr) {
    sgpu_status s = half_e(c, sr);
    if (s) return s;
    if ((s = half_h(c, sr))) return s;
    return launch_probes(c, sr);
}

// A context outside a batch takes its device memory from the device's
// default memory pool, stream-ordered on its own stream, and the pool is
// told to keep what is freed: a problem set up after another one (a sweep,
// solves served one at a time) reuses memory already mapped instead of the
// driver unmapping and mapping gigabytes again (measured at 536^3: 0.8 s to
// set up and 0.4 s to tear down the second problem with plain cudaMalloc /
// cudaFree).  sgpu_trim_device_memory hands the kept memory back.
void keep_pool_memory(int device) {
    static std::mutex mu;
    static bool done[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0 || device >= 64 || done[device]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    done[device] = true;
}

void* dev_malloc(sgpu_ctx* c, size_t bytes) {
    if (c->arena) return arena_alloc(c->arena, bytes);
    keep_pool_memory(c->device);
    void* p = nullptr;
    if (cudaMallocAsync(&p, bytes, c->stream) == cudaSuccess) return p;
    cudaGetLastError();
    // memory the pool keeps may be what is missing: hand it back and retry
    cudaMemPool_t pool;
    if (cudaStreamSynchronize(c->stream) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, c->device) == cudaSuccess &&
        cudaMemPoolTrimTo(pool, 0) == cudaSuccess && cudaMallocAsync(&p, bytes, c->stream) == cudaSuccess)
        return p;
    cudaGetLastError();
    return nullptr;
}

void dev_free(sgpu_ctx* c, void* p) {
    if (!p) return;
    if (c->arena) arena_free(c->arena, p);
    else cudaFreeAsync(p, c->stream);
}

template <class T> sgpu_status dalloc(sgpu_ctx* c, T** p, size_t n, std::vector<void*>* track = nullptr) {
    *p = nullptr;
    if (n == 0) return SGPU_OK;
    *p = (T*)dev_malloc(c, n * sizeof(T));
    if (!*p)
        return set_error(c, SGPU_ERR_OOM, std::string(c->arena ? "arena" : "cudaMalloc") + " allocation of " +
                                              std::to_string(n * sizeof(T)) + " bytes failed");
    if (track) track->push_back(*p);
    return SGPU_OK;
}

template <class T> sgpu_status h2d(sgpu_ctx* c, T* d, const T* h, size_t n) {
    if (n == 0) return SGPU_OK;
    CUDA_TRY(c, cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    return SGPU_OK;
}

void free_list(sgpu_ctx* c, std::vector<void*>& v) {
    for (void* p : v) dev_free(c, p);
    v.clear();
}


}  // namespace

// ===========================================================================
// Level-1 C ABI
// ===========================================================================
extern "C" {

const char* sgpu_last_error(const sgpu_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

}  // extern "C"

sgpu_status sgpu::create_in(const sgpu_grid_desc* d, Arena* arena, cudaStream_t stream, sgpu_ctx** out) {
    if (!d || !out) return SGPU_ERR_ARG;
    *out = nullptr;
    sgpu_ctx* c = new (std::nothrow) sgpu_ctx();
    if (!c) return SGPU_ERR_OOM;
    c->arena = arena;
    auto fail = [&](sgpu_status s) {
        // keep the context alive so the caller can read the message
        *out = c;
        return s;
    };
    for (int f = 0; f < 6; ++f) {
        c->alloc[f] = d->alloc[f];
        c->sweep[f] = d->sweep[f];
        const sgpu_lim& a = d->alloc[f];
        const sgpu_lim& w = d->sweep[f];
        if (a.xe < a.xi || a.ye < a.yi || a.ze < a.zi)
            return fail(set_error(c, SGPU_ERR_ARG, "empty Alloc range"));
        if (w.xi <= a.xi || w.xe >= a.xe || w.yi <= a.yi || w.ye >= a.ye || w.zi <= a.zi || w.ze >= a.ze)
            return fail(set_error(c, SGPU_ERR_ARG, "Sweep must lie strictly inside Alloc"));
        if (a.xi != d->alloc[0].xi || a.yi != d->alloc[0].yi || a.zi != d->alloc[0].zi)
            return fail(set_error(c, SGPU_ERR_ARG, "components must share the lower Alloc bounds"));
    }
    if (d->num_media < 1 || d->num_media > 32767)
        return fail(set_error(c, SGPU_ERR_ARG, "num_media out of range"));
    c->ox = d->alloc[0].xi; c->oy = d->alloc[0].yi; c->oz = d->alloc[0].zi;
    for (int f = 0; f < 6; ++f) {
        c->nxa = std::max(c->nxa, d->alloc[f].xe - c->ox + 1);
        c->nya = std::max(c->nya, d->alloc[f].ye - c->oy + 1);
        c->nza = std::max(c->nza, d->alloc[f].ze - c->oz + 1);
    }
    c->pitch = (c->nxa + 31) / 32 * 32;
    c->plane = (long long)c->pitch * c->nya;
    c->vol = c->plane * c->nza;
    if (c->vol >= (1LL << 31)) return fail(set_error(c, SGPU_ERR_UNSUPPORTED, "grid exceeds 2^31 padded cells"));
    c->num_media = d->num_media;
    c->dt = d->dt;
    cudaError_t e = cudaGetDevice(&c->device);
    if (e != cudaSuccess) return fail(set_error(c, SGPU_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e)));
    if (stream) {
        c->stream = stream;
        c->own_stream = false;
    } else {
        e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return fail(set_error(c, SGPU_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e)));
    }
    sgpu_status s;
    for (int f = 0; f < 6; ++f) {
        if ((s = dalloc(c, &c->F[f], c->vol))) return fail(s);
        if ((s = dalloc(c, &c->M[f], c->vol))) return fail(s);
        if ((s = dalloc(c, &c->M8[f], c->vol))) return fail(s);
        CUDA_TRY(c, cudaMemsetAsync(c->F[f], 0, c->vol * sizeof(float), c->stream));
        CUDA_TRY(c, cudaMemsetAsync(c->M8[f], 1, c->vol, c->stream));
        // padding cells keep medium 1 (vacuum), as the reference initialises
        // every media matrix before assigning regions
    }
    const int n1 = d->num_media + 1;
    c->h_g1.assign(d->g1, d->g1 + n1); c->h_g2.assign(d->g2, d->g2 + n1);
    c->h_gm1.assign(d->gm1, d->gm1 + n1); c->h_gm2.assign(d->gm2, d->gm2 + n1);
    c->h_pec.assign(n1, 0);
    if (d->is_pec) c->h_pec.assign(d->is_pec, d->is_pec + n1);
    else c->h_pec[0] = 1;
    if ((s = dalloc(c, &c->g1, n1)) || (s = dalloc(c, &c->g2, n1)) || (s = dalloc(c, &c->gm1, n1)) || (s = dalloc(c, &c->gm2, n1)))
        return fail(s);
    if ((s = h2d(c, c->g1, d->g1, n1)) || (s = h2d(c, c->g2, d->g2, n1)) || (s = h2d(c, c->gm1, d->gm1, n1)) ||
        (s = h2d(c, c->gm2, d->gm2, n1)))
        return fail(s);
    // metric arrays, re-indexed to local coordinates over the padded box
    struct M1 { const float* src; int lo, hi, origin, len; std::vector<float>* h; float** dv; };
    // x metrics span the padded pitch: lanes past the last column read them
    M1 ms[6] = {{d->idxe, d->alloc[3].xi, d->alloc[3].xe, c->ox, c->pitch, &c->h_idxe, &c->idxe},
                {d->idye, d->alloc[4].yi, d->alloc[4].ye, c->oy, c->nya, &c->h_idye, &c->idye},
                {d->idze, d->alloc[5].zi, d->alloc[5].ze, c->oz, c->nza, &c->h_idze, &c->idze},
                {d->idxh, d->alloc[0].xi, d->alloc[0].xe, c->ox, c->pitch, &c->h_idxh, &c->idxh},
                {d->idyh, d->alloc[1].yi, d->alloc[1].ye, c->oy, c->nya, &c->h_idyh, &c->idyh},
                {d->idzh, d->alloc[2].zi, d->alloc[2].ze, c->oz, c->nza, &c->h_idzh, &c->idzh}};
    for (M1& m : ms) {
        if (!m.src) return fail(set_error(c, SGPU_ERR_ARG, "missing metric array"));
        m.h->assign(m.len, 0.0f);
        for (int i = m.lo; i <= m.hi; ++i) (*m.h)[i - m.origin] = m.src[i - m.lo];
        if ((s = dalloc(c, m.dv, m.len))) return fail(s);
        if ((s = h2d(c, *m.dv, m.h->data(), m.len))) return fail(s);
    }
    if ((s = dalloc(c, &c->d_step, 1))) return fail(s);
    if ((s = dalloc(c, &c->d_flag, 1))) return fail(s);
    if ((s = dalloc(c, &c->d_err, 1))) return fail(s);
    CUDA_TRY(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    c->tma_ready = build_tensor_maps(c);
    if (c->tma_ready) {
        const int smax = (int)(kTmaSmem + 2 * kShTable * sizeof(float));
        c->tma_ready = cudaFuncSetAttribute(k_tma_efield, cudaFuncAttributeMaxDynamicSharedMemorySize, smax) == cudaSuccess &&
                       cudaFuncSetAttribute(k_tma_hfield, cudaFuncAttributeMaxDynamicSharedMemorySize, smax) == cudaSuccess;
        cudaGetLastError();
    }
    CUDA_TRY(c, cudaMemsetAsync(c->d_step, 0, sizeof(int), c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    *out = c;
    return SGPU_OK;
}

extern "C" {

sgpu_status sgpu_create(const sgpu_grid_desc* d, sgpu_ctx** out) { return create_in(d, nullptr, nullptr, out); }

void sgpu_destroy(sgpu_ctx* c) {
    if (!c) return;
    if (c->host_only) {
        if (c->host && c->host_free) c->host_free(c->host);
        delete c;
        return;
    }
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    for (int f = 0; f < 6; ++f) {
        dev_free(c, c->F[f]);
        dev_free(c, c->M[f]);
        dev_free(c, c->M8[f]);
    }
    dev_free(c, c->g1); dev_free(c, c->g2); dev_free(c, c->gm1); dev_free(c, c->gm2);
    dev_free(c, c->idxe); dev_free(c, c->idye); dev_free(c, c->idze);
    dev_free(c, c->idxh); dev_free(c, c->idyh); dev_free(c, c->idzh);
    dev_free(c, c->d_tiempo); dev_free(c, c->d_step); dev_free(c, c->d_flag); dev_free(c, c->d_err);
    free_list(c, c->cpml_allocs);
    free_list(c, c->border_allocs);
    free_list(c, c->disp_allocs);
    free_list(c, c->mdisp_allocs);
    free_list(c, c->src_allocs[0]);
    free_list(c, c->src_allocs[1]);
    free_list(c, c->probe_allocs);
    free_list(c, c->vprobe_allocs);
    free_farfields(c);
    if (c->stream && c->own_stream) cudaStreamDestroy(c->stream);
    if (c->host && c->host_free) c->host_free(c->host);
    delete c;
}

sgpu_status sgpu_get_stream(const sgpu_ctx* c, void** stream) {
    if (!c || !stream) return SGPU_ERR_ARG;
    *stream = (void*)c->stream;
    return SGPU_OK;
}

sgpu_status sgpu_synchronize(sgpu_ctx* c) {
    if (!c) return SGPU_ERR_ARG;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (c->d_err) {
        int e = 0;
        CUDA_TRY(c, cudaMemcpy(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) {
            CUDA_TRY(c, cudaMemset(c->d_err, 0, sizeof(int)));
            return set_error(c, SGPU_ERR_TIMEOUT, "a bounded wait in a pipelined kernel expired (code " + std::to_string(e) + ")");
        }
    }
    return SGPU_OK;
}

sgpu_status sgpu_set_wait_cycles(sgpu_ctx* c, int64_t cycles) {
    if (!c || cycles < 0) return set_error(c, SGPU_ERR_ARG, "bad wait budget");
    c->wait_cycles = cycles;
    if (c->graph) {  // captured launches carry the old budget
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    return SGPU_OK;
}

sgpu_status sgpu_set_wait_drill(sgpu_ctx* c, int on) {
    if (!c) return SGPU_ERR_ARG;
    c->wait_drill = on ? 1 : 0;
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    return SGPU_OK;
}

sgpu_status sgpu_set_kernel_family(sgpu_ctx* c, int family) {
    if (!c || family < 0 || family > 1) return SGPU_ERR_ARG;
    if (family == 1 && !c->tma_ready) return set_error(c, SGPU_ERR_UNSUPPORTED, "TMA tensor maps unavailable");
    c->family = family;
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    return SGPU_OK;
}

sgpu_status sgpu_upload_media(sgpu_ctx* c, int comp, const int16_t* mi) { return sgpu::upload_media(c, comp, mi, true); }

}  // extern "C"

sgpu_status sgpu::set_media_tables(sgpu_ctx* c, int num_media, const float* g1, const float* g2, const float* gm1,
                                   const float* gm2, const uint8_t* is_pec) {
    if (!c || num_media < 0 || !g1 || !g2 || !gm1 || !gm2 || !is_pec) return set_error(c, SGPU_ERR_ARG, "bad media tables");
    const int n1 = num_media + 1;
    float** dv[4] = {&c->g1, &c->g2, &c->gm1, &c->gm2};
    const float* src[4] = {g1, g2, gm1, gm2};
    std::vector<float>* hv[4] = {&c->h_g1, &c->h_g2, &c->h_gm1, &c->h_gm2};
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    for (int q = 0; q < 4; ++q) {
        dev_free(c, *dv[q]);
        *dv[q] = nullptr;
        sgpu_status s = dalloc(c, dv[q], n1);
        if (s) return s;
        if ((s = h2d(c, *dv[q], src[q], n1))) return s;
        hv[q]->assign(src[q], src[q] + n1);
    }
    c->h_pec.assign(is_pec, is_pec + n1);
    c->num_media = num_media;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SGPU_OK;
}

sgpu_status sgpu::upload_media(sgpu_ctx* c, int comp, const int16_t* mi, bool check) {
    if (!c || !mi || comp < 0 || comp > 5) return set_error(c, SGPU_ERR_ARG, "bad media upload");
    const sgpu_lim& a = c->alloc[comp];
    const long long ax = a.xe - a.xi + 1, ay = a.ye - a.yi + 1, az = a.ze - a.zi + 1;
    const long long n = check ? ax * ay * az : 0;
    std::mutex mu;
    int lo = 0, hi = 0;
    if (check) lo = 0x7fff;
    host_parallel(n, [&](long long q0, long long q1) {
        int l = 0x7fff, h = 0;
        for (long long q = q0; q < q1; ++q) {
            l = std::min(l, (int)mi[q]);
            h = std::max(h, (int)mi[q]);
        }
        std::lock_guard<std::mutex> g(mu);
        lo = std::min(lo, l);
        hi = std::max(hi, h);
    }, 1 << 20);
    if (lo < 0 || hi > c->num_media) return set_error(c, SGPU_ERR_ARG, "media index outside 0..num_media");
    // the unused padding of the common box is vacuum
    k_fill_i16<<<(unsigned)std::min<long long>((c->vol + 255) / 256, 65535), 256, 0, c->stream>>>(c->M[comp], c->vol, 1);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, box_to_device(c->M[comp], mi, sizeof(int16_t), ax, ay, az, c->pitch, c->plane / c->pitch, c->stream));
    c->media_loaded[comp] = true;
    c->src_dirty = true;
    return narrow_media(c, comp);
}

sgpu_status sgpu::narrow_media(sgpu_ctx* c, int comp) {
    k_narrow_media<<<(unsigned)std::min<long long>((c->vol + 255) / 256, 148 * 16), 256, 0, c->stream>>>(c->M[comp], c->M8[comp],
                                                                                                      c->vol);
    CUDA_TRY(c, cudaGetLastError());
    return SGPU_OK;
}

bool sgpu::tma_usable(const sgpu_ctx* c) { return c->tma_ready && c->num_media < 256; }
void sgpu::keep_device_pool(int device) { keep_pool_memory(device); }

extern "C" {

// The padding outside a component's Alloc range is zero on the device and
// stays zero; only the Alloc box moves.
sgpu_status sgpu_upload_field(sgpu_ctx* c, int comp, const float* f) {
    if (!c || !f || comp < 0 || comp > 5) return set_error(c, SGPU_ERR_ARG, "bad field upload");
    const sgpu_lim& a = c->alloc[comp];
    const long long ax = a.xe - a.xi + 1, ay = a.ye - a.yi + 1, az = a.ze - a.zi + 1;
    CUDA_TRY(c, box_to_device(c->F[comp], f, sizeof(float), ax, ay, az, c->pitch, c->plane / c->pitch, c->stream));
    return SGPU_OK;
}

sgpu_status sgpu_download_field(sgpu_ctx* c, int comp, float* f) {
    if (!c || !f || comp < 0 || comp > 5) return set_error(c, SGPU_ERR_ARG, "bad field download");
    const sgpu_lim& a = c->alloc[comp];
    const long long ax = a.xe - a.xi + 1, ay = a.ye - a.yi + 1, az = a.ze - a.zi + 1;
    CUDA_TRY(c, box_to_host(f, c->F[comp], sizeof(float), ax, ay, az, c->pitch, c->plane / c->pitch, c->stream));
    return SGPU_OK;
}

sgpu_status sgpu_init_cpml(sgpu_ctx* c, const sgpu_cpml_desc* d) {
    if (!c || !d) return set_error(c, SGPU_ERR_ARG, "null cpml descriptor");
    free_list(c, c->cpml_allocs);
    KCpml& k = c->cpml;
    k = KCpml{};
    sgpu_status s;
    const int lens[3] = {c->nxa, c->nya, c->nza};
    const int org[3] = {c->ox, c->oy, c->oz};
    const sgpu_lim* ah[3] = {&c->alloc[3], &c->alloc[4], &c->alloc[5]};
    for (int a = 0; a < 3; ++a) {
        int lo = a == 0 ? ah[a]->xi : (a == 1 ? ah[a]->yi : ah[a]->zi);
        int hi = a == 0 ? ah[a]->xe : (a == 1 ? ah[a]->ye : ah[a]->ze);
        const float* src[4] = {d->p_be[a], d->p_ce[a], d->p_bm[a], d->p_cm[a]};
        const float** dst[4] = {&k.pbe[a], &k.pce[a], &k.pbm[a], &k.pcm[a]};
        for (int w = 0; w < 4; ++w) {
            if (!src[w]) return set_error(c, SGPU_ERR_ARG, "missing CPML coefficient vector");
            std::vector<float> h(lens[a], w == 0 || w == 2 ? 1.0f : 0.0f);
            for (int i = lo; i <= hi; ++i) h[i - org[a]] = src[w][i - lo];
            float* dv;
            if ((s = dalloc(c, &dv, lens[a], &c->cpml_allocs))) return s;
            if ((s = h2d(c, dv, h.data(), h.size()))) return s;
            *dst[w] = dv;
        }
    }
    // psi kinds per component: (region pair of the first correction, of the second)
    // regions: 0 Down 1 Up 2 Left 3 Right 4 Back 5 Front
    const int pairs[6][2] = {{2, 0}, {0, 4}, {2, 4}, {2, 0}, {0, 4}, {2, 4}};
    bool any = false;
    for (int f = 0; f < 6; ++f)
        for (int w = 0; w < 2; ++w)
            for (int side = 0; side < 2; ++side) {
                const sgpu_lim& b = d->pmlc[f][pairs[f][w] + side];
                Slab& sl = k.s[f][w][side];
                sl = Slab{b.xi - c->ox, b.xe - c->ox, b.yi - c->oy, b.ye - c->oy, b.zi - c->oz, b.ze - c->oz, nullptr, 0, 0};
                if (b.xe < b.xi || b.ye < b.yi || b.ze < b.zi) {
                    sl = Slab{1, 0, 1, 0, 1, 0, nullptr, 0, 0};
                    continue;
                }
                sl.xb = sl.xlo & ~3;
                sl.px = (sl.xhi - sl.xb + 1 + 3) & ~3;
                size_t n = (size_t)sl.px * (b.ye - b.yi + 1) * (b.ze - b.zi + 1);
                if ((s = dalloc(c, &sl.psi, n, &c->cpml_allocs))) return s;
                CUDA_TRY(c, cudaMemsetAsync(sl.psi, 0, n * sizeof(float), c->stream));
                any = true;
            }
    k.on = any ? 1 : 0;
    // psi tensor maps of the TMA kernels: map 9+n of a side is slab bit n
    if (c->tma_ready)
        for (int side = 0; side < 2; ++side)
            for (int n = 0; n < 12; ++n) {
                const Slab& sl = k.s[3 * side + (n >> 2)][(n >> 1) & 1][n & 1];
                CUtensorMap* m = &(side ? c->tmh : c->tme).m[kPsiMap0 + n];
                *m = CUtensorMap{};
                if (sl.psi && !encode_psi_map(m, sl)) c->tma_ready = false;
            }
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SGPU_OK;
}

sgpu_status sgpu_init_borders(sgpu_ctx* c, const sgpu_border_desc* d) {
    if (!c || !d) return set_error(c, SGPU_ERR_ARG, "null border descriptor");
    free_list(c, c->border_allocs);
    KBorder& b = c->border;
    b = KBorder{};
    for (int f = 0; f < 6; ++f) {
        const int kinds = (d->pmc[f] != 0) + (d->periodic[f] != 0) + (d->mur[f] != 0);
        if (kinds > 1) return set_error(c, SGPU_ERR_ARG, "a face has more than one border kind");
        if (d->mur[f] && !d->mur_cab1[f]) return set_error(c, SGPU_ERR_ARG, "Mur face without CAB1 table");
        b.face_kind[f / 2][f % 2] = d->pmc[f] ? 2 : (d->periodic[f] ? 4 : 0);
    }
    const int org[3] = {c->ox, c->oy, c->oz};
    for (int q = 0; q < 3; ++q) {
        const sgpu_lim& w = c->sweep[3 + q];
        const sgpu_lim& al = c->alloc[3 + q];
        const int wl[3] = {w.xi, w.yi, w.zi}, wh[3] = {w.xe, w.ye, w.ze};
        const int al0[3] = {al.xi, al.yi, al.zi}, al1[3] = {al.xe, al.ye, al.ze};
        for (int a = 0; a < 3; ++a) {
            b.slo[q][a] = wl[a] - org[a];
            b.shi[q][a] = wh[a] - org[a];
            b.glo[q][a] = b.slo[q][a] - 1;  // inside Alloc: the sweep lies strictly inside it
            b.ghi[q][a] = b.shi[q][a] + 1;
            b.alo[q][a] = al0[a] - org[a];
            b.ahi[q][a] = al1[a] - org[a];
        }
    }
    // clone parts in the order of the reference's assignments
    const int ops[12][3] = {{0, 2, 0}, {0, 2, 1}, {0, 1, 0}, {0, 1, 1}, {1, 0, 0}, {1, 0, 1},
                            {1, 2, 0}, {1, 2, 1}, {2, 0, 0}, {2, 0, 1}, {2, 1, 0}, {2, 1, 1}};
    long long tot = 0;
    for (const auto& op : ops) {
        const int q = op[0], a = op[1], sd = op[2];
        if (!b.face_kind[a][sd]) continue;
        const int ua = a == 0 ? 1 : 0, va = a == 2 ? 1 : 2;
        b.cl[b.ncl++] = ClonePart{q, a, sd, tot};
        tot += (long long)(b.ahi[q][ua] - b.alo[q][ua] + 1) * (b.ahi[q][va] - b.alo[q][va] + 1);
    }
    b.cl_cells = tot;
    // Mur parts: regions left, right, down, up, back, front with the
    // components of regLR (Hx, Hz), regDU (Hy, Hx), regBF (Hz, Hy)
    const int regs[6][3] = {{2, 3, 5}, {3, 3, 5}, {4, 4, 3}, {5, 4, 3}, {0, 5, 4}, {1, 5, 4}};  // face, comps
    const int n1 = c->num_media + 1;
    sgpu_status s;
    tot = 0;
    for (const auto& rg : regs) {
        const int f = rg[0];
        if (!d->mur[f]) continue;
        float* cab;
        if ((s = dalloc(c, &cab, n1, &c->border_allocs))) return s;
        if ((s = h2d(c, cab, d->mur_cab1[f], n1))) return s;
        const int a = f / 2, sd = f % 2;
        for (int t = 1; t <= 2; ++t) {
            const int comp = rg[t], q = comp - 3;
            const int ua = a == 0 ? 1 : 0, va = a == 2 ? 1 : 2;
            MurPart m{};
            m.comp = comp;
            m.axis = a;
            m.inner = sd ? b.shi[q][a] : b.slo[q][a];
            m.outer = sd ? b.ghi[q][a] : b.glo[q][a];
            m.u0 = b.slo[q][ua];
            m.nu = b.shi[q][ua] - b.slo[q][ua] + 1;
            m.v0 = b.slo[q][va];
            m.nv = b.shi[q][va] - b.slo[q][va] + 1;
            const size_t cells = (size_t)m.nu * m.nv;
            if ((s = dalloc(c, &m.past, 2 * cells, &c->border_allocs))) return s;
            CUDA_TRY(c, cudaMemsetAsync(m.past, 0, 2 * cells * sizeof(float), c->stream));
            m.cab1 = cab;
            m.first = tot;
            tot += (long long)cells;
            b.mur[b.nmur++] = m;
        }
    }
    b.mur_cells = tot;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    return SGPU_OK;
}

}  // extern "C"

namespace {
// InitEDispersives / InitMdispersives on the device: the media table, and
// per E (H) component the node list of every swept node whose medium is in
// the table, in k, j, i order, with zero state.
sgpu_status init_ade(sgpu_ctx* c, const sgpu_edisp_desc* d, bool mag) {
    if (!c || !d) return set_error(c, SGPU_ERR_ARG, "null pole-residue descriptor");
    if (!ready(c)) return set_error(c, SGPU_ERR_STATE, "upload the media matrices before the pole-residue set-up");
    std::vector<void*>& allocs = mag ? c->mdisp_allocs : c->disp_allocs;
    bool& on = mag ? c->mdisp_on : c->disp_on;
    const int c0 = mag ? 3 : 0;
    free_list(c, allocs);
    (mag ? c->mdisp : c->disp) = KDisp{};
    c->h_disp_media[mag ? 1 : 0].clear();
    on = false;
    if (d->nmedia <= 0) return SGPU_OK;
    if (d->nmedia > 255) return set_error(c, SGPU_ERR_UNSUPPORTED, "more than 255 dispersive media");
    std::vector<DispMedium> media(d->nmedia);
    std::vector<int16_t> slot(c->num_media + 1, -1);
    int off = 0, nu_max = 0;
    for (int m = 0; m < d->nmedia; ++m) {
        int np = d->npoles[m];
        if (np < 0 || np > kMaxPolesPerMedium) return set_error(c, SGPU_ERR_UNSUPPORTED, "too many poles in a medium");
        int idx = d->medium_index[m];
        if (idx < 1 || idx > c->num_media) return set_error(c, SGPU_ERR_ARG, "dispersive medium index out of range");
        slot[idx] = (int16_t)m;
        DispMedium& dm = media[m];
        dm = DispMedium{};
        dm.np = np;
        dm.nu = 0;
        for (int p = 0; p < np; ++p) {
            const double* K = d->kappa + 2 * (off + p);
            const double* B = d->beta + 2 * (off + p);
            const double* G = d->g3 + 2 * (off + p);
            int found = -1;
            // a pole whose coefficients are the exact conjugates of an earlier
            // pole keeps the conjugate state: fold it onto that slot
            for (int u = 0; u < dm.nu && found < 0; ++u)
                if (dm.kappa[u].x == K[0] && dm.kappa[u].y == -K[1] && dm.beta[u].x == B[0] && dm.beta[u].y == -B[1] &&
                    dm.g3[u].x == G[0] && dm.g3[u].y == -G[1] && K[1] != 0.0)
                    found = u;
            if (found >= 0) {
                dm.map[p] = found;
            } else {
                dm.kappa[dm.nu] = make_double2(K[0], K[1]);
                dm.beta[dm.nu] = make_double2(B[0], B[1]);
                dm.beta_dt[dm.nu] = make_double2(B[0] / c->dt, B[1] / c->dt);
                dm.g3[dm.nu] = make_double2(G[0], G[1]);
                dm.map[p] = dm.nu++;
            }
        }
        nu_max = std::max(nu_max, dm.nu);
        off += np;
    }
    c->h_disp_media[mag ? 1 : 0] = media;
    sgpu_status s;
    DispMedium* dmedia;
    int16_t* dslot;
    if ((s = dalloc(c, &dmedia, media.size(), &allocs))) return s;
    if ((s = h2d(c, dmedia, media.data(), media.size()))) return s;
    if ((s = dalloc(c, &dslot, slot.size(), &allocs))) return s;
    if ((s = h2d(c, dslot, slot.data(), slot.size()))) return s;
    KDisp& k = mag ? c->mdisp : c->disp;
    k.media = dmedia;
    k.slot_of_medium = dslot;
    k.nu_max = nu_max;
    k.uniform = nu_max >= 1;
    for (const DispMedium& dm : media) k.uniform &= dm.nu == nu_max;
    k.dt = c->dt;
    k.inv_dt = 1.0 / c->dt;
    for (int comp = 0; comp < 3; ++comp) {
        const sgpu_lim& w = c->sweep[c0 + comp];
        int x0 = w.xi - c->ox, x1 = w.xe - c->ox;
        int y0 = w.yi - c->oy, y1 = w.ye - c->oy;
        int z0 = w.zi - c->oz, z1 = w.ze - c->oz;
        long long rows = (long long)(y1 - y0 + 1) * (z1 - z0 + 1);
        int* dcount;
        if ((s = dalloc(c, &dcount, rows))) return s;
        k_count_disp<<<(unsigned)((rows + 255) / 256), 256, 0, c->stream>>>(c->M[c0 + comp], dslot, c->pitch, c->plane, x0, x1,
                                                                            y0, y1, z0, z1, dcount);
        if ((s = check_launch(c, "k_count_disp"))) { dev_free(c, dcount); return s; }
        std::vector<int> cnt(rows);
        cudaError_t e = cudaMemcpyAsync(cnt.data(), dcount, rows * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) { dev_free(c, dcount); return set_error(c, SGPU_ERR_CUDA, cudaGetErrorString(e)); }
        dev_free(c, dcount);
        std::vector<long long> offs(rows);
        long long tot = 0;
        for (long long r = 0; r < rows; ++r) { offs[r] = tot; tot += cnt[r]; }
        k.n[comp] = tot;
        if (tot == 0) continue;
        long long* doffs;
        if ((s = dalloc(c, &doffs, rows))) return s;
        if ((s = h2d(c, doffs, offs.data(), rows))) { dev_free(c, doffs); return s; }
        int* node;
        uint8_t* med;
        float* prev;
        double2* J;
        if ((s = dalloc(c, &node, tot, &allocs)) || (s = dalloc(c, &med, tot, &allocs)) ||
            (s = dalloc(c, &prev, tot, &allocs)) || (s = dalloc(c, &J, (size_t)tot * std::max(1, nu_max), &allocs))) {
            dev_free(c, doffs);
            return s;
        }
        k_fill_disp<<<(unsigned)((rows + 255) / 256), 256, 0, c->stream>>>(c->M[c0 + comp], dslot, c->pitch, c->plane, x0, x1, y0,
                                                                           y1, z0, z1, doffs, node, med);
        if ((s = check_launch(c, "k_fill_disp"))) { dev_free(c, doffs); return s; }
        // the run descriptors; one more int4 holds the irregular-group count
        const long long ngrp = (tot + 31) / 32;
        int4* grp;
        if ((s = dalloc(c, &grp, (size_t)ngrp + 1, &allocs))) {
            dev_free(c, doffs);
            return s;
        }
        CUDA_TRY(c, cudaMemsetAsync(grp + ngrp, 0, sizeof(int4), c->stream));
        k_fill_grp<<<(unsigned)((ngrp + 255) / 256), 256, 0, c->stream>>>(node, med, tot, grp,
                                                                         (unsigned long long*)(grp + ngrp));
        if ((s = check_launch(c, "k_fill_grp"))) { dev_free(c, doffs); return s; }
        unsigned long long irr = 0;
        CUDA_TRY(c, cudaMemcpyAsync(&irr, grp + ngrp, sizeof(irr), cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaMemsetAsync(prev, 0, tot * sizeof(float), c->stream));
        CUDA_TRY(c, cudaMemsetAsync(J, 0, (size_t)tot * std::max(1, nu_max) * sizeof(double2), c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        dev_free(c, doffs);
        c->disp_irregular[mag ? 1 : 0][comp] = (long long)irr;
        k.grp[comp] = grp;
        k.node[comp] = node;
        k.med[comp] = med;
        k.prev[comp] = prev;
        k.J[comp] = J;
    }
    on = (k.n[0] + k.n[1] + k.n[2]) > 0;
    return SGPU_OK;
}
}  // namespace

extern "C" {

sgpu_status sgpu_init_edisp(sgpu_ctx* c, const sgpu_edisp_desc* d) { return init_ade(c, d, false); }
sgpu_status sgpu_init_mdisp(sgpu_ctx* c, const sgpu_edisp_desc* d) { return init_ade(c, d, true); }

}  // extern "C"

// ---------------------------------------------------------------------------
// Sources (plane waves and nodal sources)
namespace {

int add_table(sgpu_ctx* c, const float* ev, int numus, float delta, int is_pw) {
    sgpu_ctx::HostSrcTable t;
    t.samples.assign(ev, ev + numus + 1);
    t.numus = numus;
    t.delta = delta;
    t.is_pw = is_pw;
    c->src_tables.push_back(t);
    return (int)c->src_tables.size() - 1;
}

long long lin(const sgpu_ctx* c, int i, int j, int k) {
    return (long long)(i - c->ox) + (long long)c->pitch * (j - c->oy) + c->plane * (long long)(k - c->oz);
}

sgpu_status build_sources(sgpu_ctx* c) {
    for (int side = 0; side < 2; ++side) {
        free_list(c, c->src_allocs[side]);
        c->src[side] = KSrc{};
        const std::vector<sgpu_ctx::HostEntry>& es = c->src_host[side];
        if (es.empty()) continue;
        if (es.size() >= (1u << 30)) return set_error(c, SGPU_ERR_UNSUPPORTED, "too many source contributions");
        // group by (component, node) keeping the reference order inside a
        // group: entries are stored in that order, so a stable sort of their
        // positions by (component, node), an LSD radix sort of 12 bits a
        // pass, is the grouping
        std::vector<uint64_t> gkey(es.size());
        for (size_t q = 0; q < es.size(); ++q) gkey[q] = (uint64_t)es[q].comp * (uint64_t)c->vol + (uint64_t)es[q].node;
        std::vector<uint32_t> ord(es.size()), tmp(es.size());
        for (size_t q = 0; q < es.size(); ++q) ord[q] = (uint32_t)q;
        const uint64_t kmax = 6ull * (uint64_t)c->vol;
        for (int shift = 0; (kmax >> shift) > 0; shift += 12) {
            std::vector<uint32_t> cnt(4097, 0);
            for (uint32_t q : ord) ++cnt[((gkey[q] >> shift) & 4095) + 1];
            for (int b = 0; b < 4096; ++b) cnt[b + 1] += cnt[b];
            for (uint32_t q : ord) tmp[cnt[(gkey[q] >> shift) & 4095]++] = q;
            ord.swap(tmp);
        }
        std::vector<int> rnode, rcomp, rptr;
        std::vector<SrcEntry> ent;
        ent.reserve(es.size());
        for (size_t r = 0; r < ord.size(); ++r) {
            const size_t q = ord[r];
            if (r == 0 || gkey[q] != gkey[ord[r - 1]]) {
                rnode.push_back((int)es[q].node);
                rcomp.push_back(es[q].comp);
                rptr.push_back((int)ent.size());
            }
            ent.push_back(es[q].e);
        }
        rptr.push_back((int)ent.size());
        std::vector<SrcTable> tabs;
        std::vector<float> samples;
        for (const auto& t : c->src_tables) {
            tabs.push_back(SrcTable{t.numus, t.delta, (int)samples.size(), t.is_pw, {t.has[0], t.has[1]},
                                    {t.amax[0], t.amax[1]}});
            samples.insert(samples.end(), t.samples.begin(), t.samples.end());
        }
        KSrc& k = c->src[side];
        sgpu_status s;
        int *drn, *drc, *drp;
        SrcEntry* de;
        SrcTable* dt;
        float* dsm;
        std::vector<void*>& tr = c->src_allocs[side];
        if ((s = dalloc(c, &drn, rnode.size(), &tr)) || (s = dalloc(c, &drc, rcomp.size(), &tr)) ||
            (s = dalloc(c, &drp, rptr.size(), &tr)) || (s = dalloc(c, &de, ent.size(), &tr)) ||
            (s = dalloc(c, &dt, tabs.size(), &tr)) || (s = dalloc(c, &dsm, samples.size(), &tr)))
            return s;
        if ((s = h2d(c, drn, rnode.data(), rnode.size())) || (s = h2d(c, drc, rcomp.data(), rcomp.size())) ||
            (s = h2d(c, drp, rptr.data(), rptr.size())) || (s = h2d(c, de, ent.data(), ent.size())) ||
            (s = h2d(c, dt, tabs.data(), tabs.size())) || (s = h2d(c, dsm, samples.data(), samples.size())))
            return s;
        k.nrows = (int)rnode.size();
        k.row_node = drn;
        k.row_comp = drc;
        k.row_ptr = drp;
        k.e = de;
        k.tab = dt;
        k.samples = dsm;
        k.ntab = (int)tabs.size();
        k.h_first = c->h_first;
        k.pw_only = 1;
        for (const SrcEntry& en : ent) k.pw_only &= en.type == kSrcPlaneWave;
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->src_dirty = false;
    return SGPU_OK;
}

}  // namespace

extern "C" {

sgpu_status sgpu_add_planewave(sgpu_ctx* c, const sgpu_planewave_desc* d) {
    if (!c || !d || !d->evol) return set_error(c, SGPU_ERR_ARG, "bad plane-wave descriptor");
    const int tab = add_table(c, d->evol, d->numus, d->deltaevol, 1);
    enum { EX = 0, EY, EZ, HX, HY, HZ };
    // Per face, per side (E: planewaves.F90:914-1170, H: :1215-1470):
    // {component, incident field, offset along the face normal, sign}.
    struct Part { int comp, fld, off, sign; };
    const Part eparts[6][2] = {{{EZ, HY, -1, -1}, {EY, HZ, -1, +1}},   // back
                               {{EZ, HY, 0, +1}, {EY, HZ, 0, -1}},     // front
                               {{EX, HZ, -1, -1}, {EZ, HX, -1, +1}},   // left
                               {{EZ, HX, 0, -1}, {EX, HZ, 0, +1}},     // right
                               {{EX, HY, -1, +1}, {EY, HX, -1, -1}},   // down
                               {{EX, HY, 0, -1}, {EY, HX, 0, +1}}};    // up
    const Part hparts[6][2] = {{{HZ, EY, +1, +1}, {HY, EZ, +1, -1}},
                               {{HZ, EY, 0, -1}, {HY, EZ, 0, +1}},
                               {{HX, EZ, +1, +1}, {HZ, EX, +1, -1}},
                               {{HX, EZ, 0, -1}, {HZ, EX, 0, +1}},
                               {{HX, EY, +1, -1}, {HY, EX, +1, +1}},
                               {{HX, EY, 0, +1}, {HY, EX, 0, -1}}};
    // The face nodes in the order the reference visits them: side, face, part,
    // then the two in-face axes.  Each block is one (side, face, part) sheet.
    struct Blk {
        int side, axis, fixed;
        Part P;
        const int* L;
        float Id;
        long long nb, count, ord0, row0;  // nodes a row, nodes, first sequence number, first row
    };
    std::vector<Blk> blks;
    long long nodes = 0, rows = 0;
    const int org[3] = {c->ox, c->oy, c->oz};
    const std::vector<float>* idv[2][3] = {{&c->h_idxh, &c->h_idyh, &c->h_idzh}, {&c->h_idxe, &c->h_idye, &c->h_idze}};
    for (int side = 0; side < 2; ++side)
        for (int face = 0; face < 6; ++face) {
            if (!d->active[face]) continue;
            const int axis = face / 2;  // 0 x (back/front), 1 y (left/right), 2 z (down/up)
            for (int pi = 0; pi < 2; ++pi) {
                Blk k;
                k.side = side;
                k.axis = axis;
                k.P = side == 0 ? eparts[face][pi] : hparts[face][pi];
                k.L = d->lim[face][k.P.comp];
                k.fixed = k.L[0];
                // Id of the face: Idxh/Idyh/Idzh (E) or Idxe/Idye/Idze (H) at the fixed index
                k.Id = (*idv[side][axis])[k.fixed - org[axis]];
                const long long na = std::max(0, k.L[2] - k.L[1] + 1);
                k.nb = std::max(0, k.L[4] - k.L[3] + 1);
                k.count = na * k.nb;
                k.ord0 = nodes;
                k.row0 = rows;
                nodes += k.count;
                rows += na;
                blks.push_back(k);
            }
        }
    // One node: its entry and its d/c (Incid: d = (x*px + y*py + z*pz) - d0,
    // the kernel uses d/cluz); false when the node lies outside PhysCoor.
    auto node_entry = [&](const Blk& k, int a, int b, sgpu_ctx::HostEntry& he, float& a_node, int& kk) {
        int i, j, kz;
        if (k.axis == 0) { i = k.fixed; kz = a; j = b; }
        else if (k.axis == 1) { j = k.fixed; kz = a; i = b; }
        else { kz = k.fixed; j = a; i = b; }
        int si = i, sj = j, sk = kz;
        if (k.axis == 0) si += k.P.off; else if (k.axis == 1) sj += k.P.off; else sk += k.P.off;
        const int fl = k.P.fld;
        const int ci[3] = {si, sj, sk};
        float xyz[3];
        for (int ax = 0; ax < 3; ++ax) {
            const int q = ci[ax] - d->phys_lo[fl][ax];
            if (q < 0 || q >= d->phys_n[fl][ax]) return false;
            xyz[ax] = d->phys[fl][ax][q];
        }
        const float dd = (xyz[0] * d->px + xyz[1] * d->py + xyz[2] * d->pz) - d->d0;
        a_node = dd / d->cluz;
        kk = kz;
        he.node = lin(c, i, j, kz);
        he.comp = k.P.comp;
        he.e.comp = k.P.comp;
        he.e.type = kSrcPlaneWave;
        he.e.table = tab;
        he.e.a = a_node;
        he.e.b = d->fpw[fl];
        he.e.c = k.P.sign > 0 ? k.Id : -k.Id;
        return true;
    };
    sgpu_ctx::HostSrcTable& T = c->src_tables[tab];
    auto take_max = [&](int side, float v) {
        T.amax[side] = T.has[side] ? std::max(T.amax[side], v) : v;
        T.has[side] = 1;
    };
    if (c->zslab) {
        // a z slab keeps only its own planes' entries (every node still counts
        // for the switch-off): one pass in the reference's order
        for (const Blk& k : blks)
            for (int a = k.L[1]; a <= k.L[2]; ++a)
                for (int b = k.L[3]; b <= k.L[4]; ++b) {
                    sgpu_ctx::HostEntry he;
                    float an;
                    int kz;
                    if (!node_entry(k, a, b, he, an, kz)) return set_error(c, SGPU_ERR_ARG, "plane-wave node outside PhysCoor");
                    take_max(k.side, an);
                    if (kz < c->sweep[k.P.comp].zi || kz > c->sweep[k.P.comp].ze) continue;
                    he.order = c->src_seq++;
                    c->src_host[k.side].push_back(he);
                }
    } else {
        // every node has an entry: each sheet row is filled by a host thread at
        // its place in the reference's order (the same sequence numbers as one
        // pass), and the switch-off's largest d/c is a maximum, exact in any order
        const int seq0 = c->src_seq;
        std::vector<sgpu_ctx::HostEntry>& e0 = c->src_host[0];
        std::vector<sgpu_ctx::HostEntry>& e1 = c->src_host[1];
        const size_t b0 = e0.size(), b1 = e1.size();
        long long n0 = 0, n1 = 0;
        for (const Blk& k : blks) (k.side ? n1 : n0) += k.count;
        e0.resize(b0 + (size_t)n0);
        e1.resize(b1 + (size_t)n1);
        std::vector<long long> base(blks.size());  // first slot of each block in its side's list
        {
            long long s0 = 0, s1 = 0;
            for (size_t q = 0; q < blks.size(); ++q) {
                long long& sv = blks[q].side ? s1 : s0;
                base[q] = (long long)(blks[q].side ? b1 : b0) + sv;
                sv += blks[q].count;
            }
        }
        std::mutex mu;
        bool bad = false;
        host_parallel(rows, [&](long long r0, long long r1) {
            float mx[2] = {0.0f, 0.0f};
            bool has[2] = {false, false}, oob = false;
            size_t q = (size_t)(std::upper_bound(blks.begin(), blks.end(), r0,
                                                 [](long long r, const Blk& k) { return r < k.row0; }) - blks.begin()) - 1;
            for (long long r = r0; r < r1 && !oob; ++r) {
                while (q + 1 < blks.size() && r >= blks[q + 1].row0) ++q;
                const Blk& k = blks[q];
                const long long ra = r - k.row0;
                const int a = k.L[1] + (int)ra;
                std::vector<sgpu_ctx::HostEntry>& ev = k.side ? e1 : e0;
                for (int b = k.L[3]; b <= k.L[4]; ++b) {
                    const long long loc = ra * k.nb + (b - k.L[3]);
                    sgpu_ctx::HostEntry& he = ev[(size_t)(base[q] + loc)];
                    float an;
                    int kz;
                    if (!node_entry(k, a, b, he, an, kz)) {
                        oob = true;
                        break;
                    }
                    he.order = seq0 + (int)(k.ord0 + loc);
                    mx[k.side] = has[k.side] ? std::max(mx[k.side], an) : an;
                    has[k.side] = true;
                }
            }
            std::lock_guard<std::mutex> g(mu);
            bad = bad || oob;
            for (int sd = 0; sd < 2; ++sd)
                if (has[sd]) take_max(sd, mx[sd]);
        }, 64);
        if (bad) return set_error(c, SGPU_ERR_ARG, "plane-wave node outside PhysCoor");
        c->src_seq = seq0 + (int)nodes;
    }
    c->src_dirty = true;
    return SGPU_OK;
}

sgpu_status sgpu_add_nodal(sgpu_ctx* c, const sgpu_nodal_desc* d) {
    if (!c || !d || !d->evol || d->comp < 0 || d->comp > 5) return set_error(c, SGPU_ERR_ARG, "bad nodal descriptor");
    if (!c->media_loaded[d->comp]) return set_error(c, SGPU_ERR_STATE, "upload the media matrices before sgpu_add_nodal");
    const int tab = add_table(c, d->evol, d->numus, d->deltaevol, 0);
    const bool elec = d->comp < 3;
    const int side = elec ? 0 : 1;
    const sgpu_lim& b = d->box;
    for (int k = b.zi; k <= b.ze; ++k)
        for (int j = b.yi; j <= b.ye; ++j)
            for (int i = b.xi; i <= b.xe; ++i) {
                if (c->zslab && (k < c->sweep[d->comp].zi || k > c->sweep[d->comp].ze)) continue;
                int16_t m;
                long long node = lin(c, i, j, k);
                CUDA_TRY(c, cudaMemcpy(&m, c->M[d->comp] + node, sizeof(int16_t), cudaMemcpyDeviceToHost));
                // electric sources skip PEC media (nodalsources.F90:455-470)
                if (elec && c->h_pec[m]) continue;
                sgpu_ctx::HostEntry he;
                he.node = node;
                he.comp = d->comp;
                he.order = c->src_seq++;
                he.e.comp = d->comp;
                he.e.table = tab;
                he.e.b = 0; he.e.c = 0;
                if (d->hard) {
                    he.e.type = kSrcNodalHard;
                    he.e.a = d->amplitude;
                } else {
                    he.e.type = kSrcNodalSoft;
                    const int a = d->comp % 3;
                    float I1, I2;
                    if (elec) {
                        I1 = a == 0 ? c->h_idyh[j - c->oy] : c->h_idxh[i - c->ox];
                        I2 = a == 2 ? c->h_idyh[j - c->oy] : c->h_idzh[k - c->oz];
                    } else {
                        I1 = a == 0 ? c->h_idye[j - c->oy] : c->h_idxe[i - c->ox];
                        I2 = a == 2 ? c->h_idye[j - c->oy] : c->h_idze[k - c->oz];
                    }
                    const float g = elec ? c->h_g2[m] : c->h_gm2[m];
                    he.e.a = g * I1 * I2 * d->amplitude;
                }
                c->src_host[side].push_back(he);
            }
    c->src_dirty = true;
    return SGPU_OK;
}

sgpu_status sgpu_set_time(sgpu_ctx* c, int n0, int count, const double* t) {
    if (!c || !t || count <= 0) return set_error(c, SGPU_ERR_ARG, "bad time vector");
    dev_free(c, c->d_tiempo);
    c->d_tiempo = nullptr;
    sgpu_status s;
    if ((s = dalloc(c, &c->d_tiempo, count))) return s;
    if ((s = h2d(c, c->d_tiempo, t, count))) return s;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->t_n0 = n0;
    c->d_tiempo_count = count;
    c->h_tiempo.assign(t, t + count);
    return SGPU_OK;
}

sgpu_status sgpu_get_time(const sgpu_ctx* c, int n0, int count, double* t) {
    if (!c || count < 0 || (count > 0 && !t)) return SGPU_ERR_ARG;
    if (n0 < c->t_n0 || (long long)n0 + count > (long long)c->t_n0 + (long long)c->h_tiempo.size())
        return set_error(const_cast<sgpu_ctx*>(c), SGPU_ERR_ARG, "steps outside the time vector");
    for (int q = 0; q < count; ++q) t[q] = c->h_tiempo[n0 - c->t_n0 + q];
    return SGPU_OK;
}

sgpu_status sgpu_set_probes(sgpu_ctx* c, int np, const int* cijk, int cap) {
    if (!c || np < 0 || (np > 0 && (!cijk || cap <= 0))) return set_error(c, SGPU_ERR_ARG, "bad probe set");
    free_list(c, c->probe_allocs);
    c->probes = KProbes{};
    c->probe_written = c->probe_read = 0;
    c->probe_first_n = -1;
    if (np == 0) return SGPU_OK;
    std::vector<int> comp(np);
    std::vector<long long> idx(np);
    for (int q = 0; q < np; ++q) {
        int f = cijk[4 * q];
        if (f < 0 || f > 5) return set_error(c, SGPU_ERR_ARG, "probe component out of range");
        const sgpu_lim& a = c->alloc[f];
        int i = cijk[4 * q + 1], j = cijk[4 * q + 2], k = cijk[4 * q + 3];
        if (i < a.xi || i > a.xe || j < a.yi || j > a.ye || k < a.zi || k > a.ze)
            return set_error(c, SGPU_ERR_ARG, "probe outside Alloc");
        comp[q] = f;
        idx[q] = lin(c, i, j, k);
    }
    sgpu_status s;
    int* dc;
    long long* di;
    float* ring;
    if ((s = dalloc(c, &dc, np, &c->probe_allocs)) || (s = dalloc(c, &di, np, &c->probe_allocs)) ||
        (s = dalloc(c, &ring, (size_t)np * cap, &c->probe_allocs)))
        return s;
    if ((s = h2d(c, dc, comp.data(), np)) || (s = h2d(c, di, idx.data(), np))) return s;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->probes = KProbes{np, dc, di, ring, cap};
    return SGPU_OK;
}

sgpu_status sgpu_read_probes(sgpu_ctx* c, float* out, int max_steps, int* nsteps, int* first_n) {
    if (!c || !nsteps) return set_error(c, SGPU_ERR_ARG, "bad probe read");
    *nsteps = 0;
    if (first_n) *first_n = c->probe_first_n + (int)c->probe_read;
    if (c->probes.n == 0) return SGPU_OK;
    long long pending = c->probe_written - c->probe_read;
    long long take = std::min<long long>(pending, max_steps);
    if (take <= 0) return SGPU_OK;
    if (!out) return set_error(c, SGPU_ERR_ARG, "null output");
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    const int np = c->probes.n, cap = c->probes.cap;
    for (long long r = 0; r < take; ++r) {
        long long row = (c->probe_read + r) % cap;
        CUDA_TRY(c, cudaMemcpy(out + r * np, c->probes.ring + row * np, np * sizeof(float), cudaMemcpyDeviceToHost));
    }
    c->probe_read += take;
    *nsteps = (int)take;
    return SGPU_OK;
}

namespace {
// The sampled index range of one axis: multiples of `tr` in [lo, hi], as
// XItrancos / XEtrancos of observation.F90:318-331 (Fortran integer division
// and MOD, both truncating toward zero like C++).
bool stride_range(int lo, int hi, int tr, int* first, int* count) {
    if (tr < 1 || hi < lo) return false;
    int a = lo / tr, b = hi / tr;
    if (lo % tr != 0) a += 1;
    *first = a;
    *count = b - a + 1;
    return *count > 0;
}

sgpu_status add_volume_probe(sgpu_ctx* c, int kind, int magnetic, const int* box, const int* stride, VolProbe* p) {
    if (magnetic != 0 && magnetic != 1) return set_error(c, SGPU_ERR_ARG, "volume probe: magnetic must be 0 or 1");
    *p = VolProbe{};
    p->kind = kind;
    p->magnetic = magnetic;
    for (int f = 3 * magnetic; f < 3 * magnetic + 3; ++f) {
        const sgpu_lim& a = c->alloc[f];
        if (box[0] < a.xi || box[1] > a.xe || box[2] < a.yi || box[3] > a.ye || box[4] < a.zi || box[5] > a.ze)
            return set_error(c, SGPU_ERR_ARG, "volume probe box outside Alloc");
    }
    if (!stride_range(box[0], box[1], stride[0], &p->i0, &p->ni) || !stride_range(box[2], box[3], stride[1], &p->j0, &p->nj) ||
        !stride_range(box[4], box[5], stride[2], &p->k0, &p->nk))
        return set_error(c, SGPU_ERR_ARG, "volume probe samples no node");
    for (int a = 0; a < 3; ++a) p->tr[a] = stride[a];
    return SGPU_OK;
}

sgpu_status commit_volume_probe(sgpu_ctx* c, const VolProbe& p, int* id) {
    c->vprobes.push_back(p);
    c->vprobe_read.push_back(0);
    if (id) *id = (int)c->vprobes.size() - 1;
    if (c->graph) {  // the captured steps do not launch the new probe
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    return SGPU_OK;
}
}  // namespace

sgpu_status sgpu_add_freq_probe(sgpu_ctx* c, const sgpu_freq_probe_desc* d, int* id) {
    if (!c || !d || d->nfreq < 1 || !d->freq) return set_error(c, SGPU_ERR_ARG, "bad frequency probe");
    if (c->h_tiempo.empty()) return set_error(c, SGPU_ERR_STATE, "set the time vector before a frequency probe");
    VolProbe p;
    sgpu_status s = add_volume_probe(c, 0, d->magnetic, d->box, d->stride, &p);
    if (s) return s;
    p.nf = d->nfreq;
    // observation.F90:3530-3534 with mcPI2 = -(0, 1) * 2 * pi (fdetypes.F90:190),
    // all factors real(4) so that its imaginary part is -(2 * pi_f)
    const double mcpi2_im = -(double)(2.0f * (float)3.14159265358979323846);
    const int steps = (int)c->h_tiempo.size();
    std::vector<double2> w((size_t)steps * p.nf);
    for (int f = 0; f < p.nf; ++f) {
        const double im1 = mcpi2_im * (double)d->freq[f];  // mcPI2 * Freq
        const double re1 = -0.0 * (double)d->freq[f];
        std::complex<double> eh = 0.0;
        if (d->magnetic) eh = std::exp(std::complex<double>(re1 * c->dt * 0.5, im1 * c->dt * 0.5));
        for (int m = 0; m < steps; ++m) {
            const double at = c->h_tiempo[m];
            const std::complex<double> e = std::exp(std::complex<double>(re1 * at, im1 * at));
            // dt * (1, 0) is a complex with a known zero imaginary part, so
            // its product with e is (dt * Re e, dt * Im e)
            double wr = c->dt * e.real();
            double wi = c->dt * e.imag();
            if (d->magnetic) {
                const double hr = wr * eh.real() - wi * eh.imag();
                const double hi = wr * eh.imag() + wi * eh.real();
                wr = hr;
                wi = hi;
            }
            w[(size_t)m * p.nf + f] = make_double2(wr, wi);
        }
    }
    const long long nodes = (long long)p.ni * p.nj * p.nk;
    double2* acc;
    double2* dw;
    if ((s = dalloc(c, &acc, (size_t)nodes * 3 * p.nf, &c->vprobe_allocs)) ||
        (s = dalloc(c, &dw, w.size(), &c->vprobe_allocs)))
        return s;
    CUDA_TRY(c, cudaMemsetAsync(acc, 0, sizeof(double2) * (size_t)nodes * 3 * p.nf, c->stream));
    if ((s = h2d(c, dw, w.data(), w.size()))) return s;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    p.acc = acc;
    p.w = dw;
    p.w_n0 = c->t_n0;
    p.w_steps = steps;
    return commit_volume_probe(c, p, id);
}

sgpu_status sgpu_add_movie_probe(sgpu_ctx* c, const sgpu_movie_probe_desc* d, int* id) {
    if (!c || !d || d->every < 1 || d->capacity < 1 || d->n_last < d->n_first)
        return set_error(c, SGPU_ERR_ARG, "bad movie probe");
    VolProbe p;
    sgpu_status s = add_volume_probe(c, 1, d->magnetic, d->box, d->stride, &p);
    if (s) return s;
    p.n_first = d->n_first;
    p.n_last = d->n_last;
    p.every = d->every;
    p.cap = d->capacity;
    const long long nodes = (long long)p.ni * p.nj * p.nk;
    float* ring;
    if ((s = dalloc(c, &ring, (size_t)nodes * 3 * p.cap, &c->vprobe_allocs))) return s;
    p.ring = ring;
    return commit_volume_probe(c, p, id);
}

sgpu_status sgpu_volume_probe_shape(const sgpu_ctx* c, int id, int* ni, int* nj, int* nk, int* ijk0) {
    if (!c || id < 0 || id >= (int)c->vprobes.size()) return SGPU_ERR_ARG;
    const VolProbe& p = c->vprobes[id];
    if (ni) *ni = p.ni;
    if (nj) *nj = p.nj;
    if (nk) *nk = p.nk;
    if (ijk0) {
        ijk0[0] = p.i0;
        ijk0[1] = p.j0;
        ijk0[2] = p.k0;
    }
    return SGPU_OK;
}

sgpu_status sgpu_read_freq_probe(sgpu_ctx* c, int id, double* out) {
    if (!c || !out || id < 0 || id >= (int)c->vprobes.size() || c->vprobes[id].kind != 0)
        return set_error(c, SGPU_ERR_ARG, "no frequency probe with that id");
    const VolProbe& p = c->vprobes[id];
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    CUDA_TRY(c, cudaMemcpy(out, p.acc, sizeof(double2) * (size_t)p.ni * p.nj * p.nk * 3 * p.nf, cudaMemcpyDeviceToHost));
    return SGPU_OK;
}

sgpu_status sgpu_read_movie_probe(sgpu_ctx* c, int id, float* out, int max_frames, int* frames, int* first_n) {
    if (!c || !frames || id < 0 || id >= (int)c->vprobes.size() || c->vprobes[id].kind != 1)
        return set_error(c, SGPU_ERR_ARG, "no movie probe with that id");
    const VolProbe& p = c->vprobes[id];
    *frames = 0;
    // frames of the steps launched so far
    const int end = std::min(p.n_last, c->steps_hi);
    const long long total = end > p.n_first ? (end - p.n_first + p.every - 1) / p.every : 0;
    long long& read = c->vprobe_read[id];
    if (total - read > p.cap) read = total - p.cap;  // older frames were overwritten
    if (first_n) *first_n = p.n_first + (int)(read * p.every);
    const long long take = std::min<long long>(total - read, max_frames);
    if (take <= 0) return SGPU_OK;
    if (!out) return set_error(c, SGPU_ERR_ARG, "null output");
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    const size_t frame = (size_t)p.ni * p.nj * p.nk * 3;
    for (long long r = 0; r < take; ++r) {
        const long long slot = (read + r) % p.cap;
        CUDA_TRY(c, cudaMemcpy(out + r * frame, p.ring + slot * frame, frame * sizeof(float), cudaMemcpyDeviceToHost));
    }
    read += take;
    *frames = (int)take;
    return SGPU_OK;
}

sgpu_status sgpu_zplane(sgpu_ctx* c, int comp, int z, void** ptr, uint64_t* bytes) {
    if (!c || comp < 0 || comp > 5 || !ptr) return set_error(c, SGPU_ERR_ARG, "bad plane request");
    if (z < c->oz || z >= c->oz + c->nza) return set_error(c, SGPU_ERR_ARG, "plane outside the context's Alloc box");
    *ptr = c->F[comp] + c->plane * (long long)(z - c->oz);
    if (bytes) *bytes = (uint64_t)c->plane * sizeof(float);
    return SGPU_OK;
}

sgpu_status sgpu_copy_zplane(sgpu_ctx* dst, sgpu_ctx* src, int comp, int z) {
    if (!dst || !src) return SGPU_ERR_ARG;
    if (dst->pitch != src->pitch || dst->plane != src->plane || dst->ox != src->ox || dst->oy != src->oy)
        return set_error(dst, SGPU_ERR_ARG, "the two contexts have different x-y layouts");
    void *d, *s;
    uint64_t n;
    sgpu_status st;
    if ((st = sgpu_zplane(dst, comp, z, &d, &n)) || (st = sgpu_zplane(src, comp, z, &s, nullptr))) return st;
    // the copy waits for the work queued on src, and src's later work waits
    // for the copy (the plane is overwritten by src's next half step)
    // (each event is created on the device of the stream that records it)
    int cur = 0;
    cudaGetDevice(&cur);
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaSetDevice(src->device);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(a, src->stream);
    if (e == cudaSuccess) e = cudaSetDevice(dst->device);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(dst->stream, a, 0);
    if (e == cudaSuccess)
        e = dst->device == src->device ? cudaMemcpyAsync(d, s, n, cudaMemcpyDeviceToDevice, dst->stream)
                                       : cudaMemcpyPeerAsync(d, dst->device, s, src->device, n, dst->stream);
    if (e == cudaSuccess) e = cudaEventRecord(b, dst->stream);
    if (e == cudaSuccess) e = cudaSetDevice(src->device);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(src->stream, b, 0);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaSetDevice(cur);
    if (e != cudaSuccess) return set_error(dst, SGPU_ERR_CUDA, std::string("plane copy: ") + cudaGetErrorString(e));
    return SGPU_OK;
}

namespace {
sgpu_status note_probe_rows(sgpu_ctx* c, int n0, int count) {
    if (c->probes.n == 0) return SGPU_OK;
    if (c->probe_first_n < 0) c->probe_first_n = n0;
    if (n0 != c->probe_first_n + c->probe_written)
        return set_error(c, SGPU_ERR_STATE, "probe rows must be recorded for consecutive steps");
    if (c->probe_written + count - c->probe_read > c->probes.cap)
        return set_error(c, SGPU_ERR_STATE, "probe ring full: read the probes first");
    return SGPU_OK;
}
}  // namespace

#define SGPU_READY(c)                                                                            \
    do {                                                                                         \
        if (!(c)) return SGPU_ERR_ARG;                                                           \
        if (!ready(c)) return set_error((c), SGPU_ERR_STATE, "media matrices not uploaded");      \
    } while (0)

sgpu_status sgpu_advance_ex(sgpu_ctx* c) { SGPU_READY(c); return launch_e<kBulk | kCx>(c); }
sgpu_status sgpu_advance_ey(sgpu_ctx* c) { SGPU_READY(c); return launch_e<kBulk | kCy>(c); }
sgpu_status sgpu_advance_ez(sgpu_ctx* c) { SGPU_READY(c); return launch_e<kBulk | kCz>(c); }
sgpu_status sgpu_advance_electric_cpml(sgpu_ctx* c) {
    SGPU_READY(c);
    return c->cpml.on ? launch_e<kCpml | kAll>(c) : SGPU_OK;
}
sgpu_status sgpu_advance_edispersive_e(sgpu_ctx* c) { SGPU_READY(c); return launch_edisp(c); }
sgpu_status sgpu_advance_mdispersive_h(sgpu_ctx* c) { SGPU_READY(c); return launch_mdisp(c); }
sgpu_status sgpu_advance_planewave_e(sgpu_ctx* c, int n) {
    SGPU_READY(c);
    return launch_sources(c, 0, StepRef{nullptr, n}, kMaskPW);
}
sgpu_status sgpu_advance_nodal_e(sgpu_ctx* c, int n) {
    SGPU_READY(c);
    return launch_sources(c, 0, StepRef{nullptr, n}, kMaskNodal);
}
sgpu_status sgpu_advance_hx(sgpu_ctx* c) { SGPU_READY(c); return launch_h<kBulk | kCx>(c); }
sgpu_status sgpu_advance_hy(sgpu_ctx* c) { SGPU_READY(c); return launch_h<kBulk | kCy>(c); }
sgpu_status sgpu_advance_hz(sgpu_ctx* c) { SGPU_READY(c); return launch_h<kBulk | kCz>(c); }
sgpu_status sgpu_advance_magnetic_cpml(sgpu_ctx* c) {
    SGPU_READY(c);
    return c->cpml.on ? launch_h<kCpml | kAll>(c) : SGPU_OK;
}
sgpu_status sgpu_advance_planewave_h(sgpu_ctx* c, int n) {
    SGPU_READY(c);
    return launch_sources(c, 1, StepRef{nullptr, n}, kMaskPW);
}
sgpu_status sgpu_advance_nodal_h(sgpu_ctx* c, int n) {
    SGPU_READY(c);
    return launch_sources(c, 1, StepRef{nullptr, n}, kMaskNodal);
}
sgpu_status sgpu_advance_pmc_h(sgpu_ctx* c) { SGPU_READY(c); return launch_clone(c, 2); }
sgpu_status sgpu_advance_periodic_h(sgpu_ctx* c) { SGPU_READY(c); return launch_clone(c, 4); }
sgpu_status sgpu_advance_magnetic_mur(sgpu_ctx* c) { SGPU_READY(c); return launch_mur(c); }
sgpu_status sgpu_update_observation(sgpu_ctx* c, int n) {
    SGPU_READY(c);
    sgpu_status s = note_probe_rows(c, n, 1);
    if (s) return s;
    s = launch_probes(c, StepRef{nullptr, n});
    if (!s && c->probes.n) c->probe_written += 1;
    if (!s) c->steps_hi = std::max(c->steps_hi, n + 1);
    return s;
}

sgpu_status sgpu_advance_e(sgpu_ctx* c, int n) { SGPU_READY(c); return half_e(c, StepRef{nullptr, n}); }
sgpu_status sgpu_advance_h(sgpu_ctx* c, int n) { SGPU_READY(c); return half_h(c, StepRef{nullptr, n}); }

sgpu_status sgpu_advance_steps(sgpu_ctx* c, int n0, int count) {
    SGPU_READY(c);
    if (count <= 0) return SGPU_OK;
    if (c->src_dirty) {
        sgpu_status s = build_sources(c);
        if (s) return s;
    }
    const bool has_src = c->src[0].nrows + c->src[1].nrows > 0;
    if (has_src && (n0 < c->t_n0 || n0 + count > c->t_n0 + c->d_tiempo_count))
        return set_error(c, SGPU_ERR_ARG, "steps outside the time vector");
    sgpu_status s = note_probe_rows(c, n0, count);
    if (s) return s;
    note_first_half(c, 2 * n0);
    const int chunk = std::min(count, 32);
    if (!c->graph || c->graph_steps != chunk) {
        if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
        cudaGraph_t g;
        CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        sgpu_status cs = SGPU_OK;
        for (int q = 0; q < chunk && !cs; ++q) cs = whole_step(c, StepRef{c->d_step, q});
        if (!cs) {
            k_add_step<<<1, 1, 0, c->stream>>>(c->d_step, chunk);
            cs = check_launch(c, "k_add_step");
        }
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (cs) { if (e == cudaSuccess) cudaGraphDestroy(g); return cs; }
        if (e != cudaSuccess) return set_error(c, SGPU_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&c->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { c->graph = nullptr; return set_error(c, SGPU_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)); }
        c->graph_steps = chunk;
    }
    k_set_step<<<1, 1, 0, c->stream>>>(c->d_step, n0);
    if ((s = check_launch(c, "k_set_step"))) return s;
    int done = 0;
    while (count - done >= chunk) {
        CUDA_TRY(c, cudaGraphLaunch(c->graph, c->stream));
        done += chunk;
    }
    for (; done < count; ++done)
        if ((s = whole_step(c, StepRef{nullptr, n0 + done}))) return s;
    if (c->probes.n) c->probe_written += count;
    c->steps_hi = std::max(c->steps_hi, n0 + count);
    return SGPU_OK;
}

sgpu_status sgpu_elapsed_steps(sgpu_ctx* c, int n0, int count, float* ms) {
    SGPU_READY(c);
    if (!ms) return set_error(c, SGPU_ERR_ARG, "null output");
    cudaEvent_t a, b;
    CUDA_TRY(c, cudaEventCreate(&a));
    CUDA_TRY(c, cudaEventCreate(&b));
    CUDA_TRY(c, cudaEventRecord(a, c->stream));
    sgpu_status s = sgpu_advance_steps(c, n0, count);
    CUDA_TRY(c, cudaEventRecord(b, c->stream));
    CUDA_TRY(c, cudaEventSynchronize(b));
    CUDA_TRY(c, cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return s;
}

sgpu_status sgpu_profile_steps(sgpu_ctx* c, int n0, int count, float* ms6) {
    SGPU_READY(c);
    if (!ms6) return set_error(c, SGPU_ERR_ARG, "null output");
    sgpu_status s = note_probe_rows(c, n0, count);
    if (s) return s;
    if (c->src_dirty && (s = build_sources(c))) return s;
    cudaEvent_t ev[7];
    for (auto& e : ev) CUDA_TRY(c, cudaEventCreate(&e));
    for (int q = 0; q < 6; ++q) ms6[q] = 0.0f;
    for (int n = n0; n < n0 + count && !s; ++n) {
        StepRef sr{nullptr, n};
        cudaEventRecord(ev[0], c->stream);
        s = field_e(c);
        cudaEventRecord(ev[1], c->stream);
        if (!s) s = launch_edisp(c);
        cudaEventRecord(ev[2], c->stream);
        if (!s) s = launch_sources(c, 0, sr);
        cudaEventRecord(ev[3], c->stream);
        if (!s) s = field_h(c);
        cudaEventRecord(ev[4], c->stream);
        if (!s) s = launch_mdisp(c);
        if (!s) s = launch_sources(c, 1, sr);
        if (!s) s = launch_borders_h(c);
        cudaEventRecord(ev[5], c->stream);
        if (!s) s = launch_probes(c, sr);
        cudaEventRecord(ev[6], c->stream);
        CUDA_TRY(c, cudaEventSynchronize(ev[6]));
        for (int q = 0; q < 6; ++q) {
            float t = 0;
            cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
            ms6[q] += t;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (!s && c->probes.n) c->probe_written += count;
    if (!s) c->steps_hi = std::max(c->steps_hi, n0 + count);
    return s;
}

sgpu_status sgpu_algorithmic_bytes(const sgpu_ctx* c, double* b6) {
    if (!c || !b6) return SGPU_ERR_ARG;
    auto cells = [](const sgpu_lim& l) { return (double)(l.xe - l.xi + 1) * (l.ye - l.yi + 1) * (l.ze - l.zi + 1); };
    auto psi_bytes = [&](int c0) {
        double b = 0;
        for (int f = c0; f < c0 + 3; ++f)
            for (int w = 0; w < 2; ++w)
                for (int sd = 0; sd < 2; ++sd) {
                    const Slab& sl = c->cpml.s[f][w][sd];
                    if (sl.psi) b += 8.0 * (sl.xhi - sl.xlo + 1) * (sl.yhi - sl.ylo + 1) * (sl.zhi - sl.zlo + 1);
                }
        return b;
    };
    // E (H) half step: every swept node of the three updated components is
    // read and written once (8 B) with its medium (1 B from the one-byte copy
    // the TMA-pipelined kernels read, else 2 B), and each node of the three
    // other components is read once (4 B); psi points are read and written
    // (8 B).  Neighbour re-reads and coefficient tables are not counted.
    const double node = (c->family == 1 && tma_usable(c)) ? 9.0 : 10.0;
    double e = 0, h = 0;
    for (int f = 0; f < 3; ++f) e += cells(c->sweep[f]) * node + cells(c->sweep[f + 3]) * 4.0;
    for (int f = 3; f < 6; ++f) h += cells(c->sweep[f]) * node + cells(c->sweep[f - 3]) * 4.0;
    b6[0] = e + psi_bytes(0);
    // ADE node: E 8 + previous E 8 + 32 per state slot, its share of the
    // group's run descriptor (16 B per 32 nodes) and, in groups of more than
    // two runs, index 4 + medium slot 1
    auto ade_bytes = [&](const KDisp& d, int side) {
        double b = 0;
        for (int comp = 0; comp < 3; ++comp) {
            const double n = (double)d.n[comp], irr = 32.0 * (double)c->disp_irregular[side][comp];
            b += n * (16.0 + 32.0 * d.nu_max) + 16.0 * std::ceil(n / 32.0) + 5.0 * std::min(n, irr);
        }
        return b;
    };
    b6[1] = c->disp_on ? ade_bytes(c->disp, 0) : 0.0;
    b6[2] = 0;
    b6[3] = h + psi_bytes(3);
    // H sources (not counted) and borders: a clone cell reads and writes 4 B
    // each; a Mur cell reads H, its medium and both Past_ values and writes H
    // and both Past_ values (26 B)
    b6[4] = 8.0 * (double)c->border.cl_cells + 26.0 * (double)c->border.mur_cells +
            (c->mdisp_on ? ade_bytes(c->mdisp, 1) : 0.0);
    b6[5] = 8.0 * c->probes.n;
    return SGPU_OK;
}

sgpu_status sgpu_compulsory_bytes(const sgpu_ctx* c, double* b6) {
    if (!c || !b6) return SGPU_ERR_ARG;
    auto cells = [](const sgpu_lim& l) { return (double)(l.xe - l.xi + 1) * (l.ye - l.yi + 1) * (l.ze - l.zi + 1); };
    auto psi_points = [&](int c0) {
        double n = 0;
        for (int f = c0; f < c0 + 3; ++f)
            for (int w = 0; w < 2; ++w)
                for (int sd = 0; sd < 2; ++sd) {
                    const Slab& sl = c->cpml.s[f][w][sd];
                    if (sl.psi) n += (double)(sl.xhi - sl.xlo + 1) * (sl.yhi - sl.ylo + 1) * (sl.zhi - sl.zlo + 1);
                }
        return n;
    };
    // Each field node is read and written once a step with its int16 medium
    // (10 B), each psi point read and written (8 B), each pole-residue node's
    // previous field read and written (8 B) and each stored current read and
    // written (32 B); the other component's reads, neighbour re-reads, node
    // lists and the field re-read of a separate ADE pass are not counted.
    double e = 0, h = 0, nodes = 0, mnodes = 0;
    for (int f = 0; f < 3; ++f) e += cells(c->sweep[f]) * 10.0;
    for (int f = 3; f < 6; ++f) h += cells(c->sweep[f]) * 10.0;
    for (int comp = 0; comp < 3; ++comp) nodes += (double)c->disp.n[comp];
    for (int comp = 0; comp < 3; ++comp) mnodes += (double)c->mdisp.n[comp];
    b6[0] = e + 8.0 * psi_points(0);
    b6[1] = c->disp_on ? nodes * (8.0 + 32.0 * c->disp.nu_max) : 0.0;
    b6[2] = 0;
    b6[3] = h + 8.0 * psi_points(3);
    b6[4] = 8.0 * (double)c->border.cl_cells + 26.0 * (double)c->border.mur_cells +
            (c->mdisp_on ? mnodes * (8.0 + 32.0 * c->mdisp.nu_max) : 0.0);
    b6[5] = 8.0 * c->probes.n;
    return SGPU_OK;
}

sgpu_status sgpu_trim_device_memory(void) {
    int device = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&device) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess || cudaMemPoolTrimTo(pool, 0) != cudaSuccess) {
        cudaGetLastError();
        return SGPU_ERR_CUDA;
    }
    return SGPU_OK;
}

sgpu_status sgpu_select_device(int device) {
    return cudaSetDevice(device) == cudaSuccess ? SGPU_OK : SGPU_ERR_CUDA;
}

sgpu_status sgpu_kernels_per_step(const sgpu_ctx* c, int* n) {
    if (!c || !n) return SGPU_ERR_ARG;
    int k = 2;  // E and H field kernels
    for (int comp = 0; comp < 3; ++comp) k += c->disp_on && c->disp.n[comp] > 0;
    for (int comp = 0; comp < 3; ++comp) k += c->mdisp_on && c->mdisp.n[comp] > 0;
    k += c->src[0].nrows > 0;
    k += c->src[1].nrows > 0;
    k += c->probes.n > 0;
    k += (int)c->vprobes.size();
    k += c->border.cl_cells > 0;
    k += c->border.mur_cells > 0;
    *n = k;
    return SGPU_OK;
}

sgpu_status sgpu_check_finite(sgpu_ctx* c) {
    if (!c) return SGPU_ERR_ARG;
    CUDA_TRY(c, cudaMemsetAsync(c->d_flag, 0, sizeof(unsigned int), c->stream));
    for (int f = 0; f < 6; ++f) {
        k_nonfinite<<<148 * 8, 256, 0, c->stream>>>(c->F[f], c->vol, c->d_flag);
        sgpu_status s = check_launch(c, "k_nonfinite");
        if (s) return s;
    }
    unsigned int flag = 0;
    CUDA_TRY(c, cudaMemcpyAsync(&flag, c->d_flag, sizeof(flag), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (flag) return set_error(c, SGPU_ERR_NONFINITE, "non-finite field value found");
    return SGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Non-finite scan that allocates nothing.
//
// sgpu_check_finite keeps its result word in memory the context allocated at
// creation.  sgpu_scan_nonfinite_noalloc is the same scan for callers that
// may not allocate device memory when they run it: a Fortran or framework
// host whose device memory belongs to its own pool allocator, a service loop
// that forbids cudaMalloc/cudaFree after start-up, or a watchdog that checks
// a field buffer someone else owns.  Its scratch is the file-scope array
// below: every device that loads this library holds it (8 B per block of
// 4096 elements, 512 KiB in all) until the process exits, and every call
// shares it.
namespace {

constexpr int kScanChunk = 4096;      // elements scanned by one block
constexpr int kScanMaxBlocks = 65536;  // one scratch word per block
constexpr unsigned long long kScanMaxElems = (unsigned long long)kScanChunk * kScanMaxBlocks;  // 268,435,456

// [b] = (non-finite count of block b) << 32 | first offset in the block
//       (0xffffffff when none); [kScanMaxBlocks] = the reduced result.
// Every entry a call reads is written earlier in that call, so nothing has
// to start at zero.
static __device__ __align__(256) unsigned long long g_scan_scratch[kScanMaxBlocks + 1];

__global__ void k_scan_partial(const float* a, unsigned long long n, unsigned long long* part) {
    __shared__ unsigned int cnt, first;
    if (threadIdx.x == 0) {
        cnt = 0;
        first = 0xffffffffu;
    }
    __syncthreads();
    const unsigned long long base = (unsigned long long)blockIdx.x * kScanChunk;
    for (int t = threadIdx.x; t < kScanChunk; t += blockDim.x) {
        const unsigned long long q = base + t;
        if (q < n && !isfinite(a[q])) {
            atomicAdd(&cnt, 1u);
            atomicMin(&first, (unsigned int)t);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) part[blockIdx.x] = ((unsigned long long)cnt << 32) | first;
}

__global__ void k_scan_reduce(unsigned long long* part, int nblocks) {
    __shared__ unsigned int total, first;
    if (threadIdx.x == 0) {
        total = 0;
        first = 0xffffffffu;
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        const unsigned long long v = part[b];
        const unsigned int cnt = (unsigned int)(v >> 32), f = (unsigned int)(v & 0xffffffffu);
        if (cnt) {
            atomicAdd(&total, cnt);
            atomicMin(&first, (unsigned int)b * kScanChunk + f);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) part[kScanMaxBlocks] = ((unsigned long long)total << 32) | first;
}

constexpr int kScanMaxDevices = 64;
std::mutex g_scan_mu;
unsigned long long* g_scan_ptr[kScanMaxDevices] = {};

}  // namespace

extern "C" sgpu_status sgpu_scan_nonfinite_noalloc(const float* data, uint64_t n, void* stream, uint64_t* count,
                                                  int64_t* first_index) {
    if (!count || !first_index || (n > 0 && !data)) return SGPU_ERR_ARG;
    if (n > kScanMaxElems) return SGPU_ERR_SIZE;
    *count = 0;
    *first_index = -1;
    if (n == 0) return SGPU_OK;
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, data) != cudaSuccess) {
        cudaGetLastError();
        return SGPU_ERR_ARG;
    }
    if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) return SGPU_ERR_ARG;
    // The scan runs on the device that holds the data, whichever device the
    // caller's own runtime has selected: this library links the CUDA runtime
    // statically, so its current device is its own; it switches to the
    // data's device for the call and back before returning.
    const int dev = attr.device;
    if (dev < 0 || dev >= kScanMaxDevices) return SGPU_ERR_ARG;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return SGPU_ERR_CUDA;
    struct Restore {
        int d;
        ~Restore() { if (d >= 0) cudaSetDevice(d); }
    } restore{prev != dev ? prev : -1};
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) return SGPU_ERR_CUDA;
    unsigned long long* scratch = nullptr;
    {
        // once per device, with that device current: the device address of
        // the file-scope array (its host-side name is only a stand-in)
        std::lock_guard<std::mutex> lock(g_scan_mu);
        if (!g_scan_ptr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_scan_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return SGPU_ERR_CUDA;
            }
            g_scan_ptr[dev] = (unsigned long long*)p;
        }
        scratch = g_scan_ptr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int nblocks = (int)((n + kScanChunk - 1) / kScanChunk);
    k_scan_partial<<<nblocks, 256, 0, s>>>(data, n, scratch);
    k_scan_reduce<<<1, 1024, 0, s>>>(scratch, nblocks);
    if (cudaGetLastError() != cudaSuccess) return SGPU_ERR_CUDA;
    unsigned long long res = 0;
    if (cudaMemcpyAsync(&res, scratch + kScanMaxBlocks, sizeof(res), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return SGPU_ERR_CUDA;
    *count = res >> 32;
    const unsigned int f = (unsigned int)(res & 0xffffffffu);
    *first_index = (*count > 0 && f != 0xffffffffu) ? (int64_t)f : -1;
    return SGPU_OK;
}

extern "C" {

sgpu_status sgpu_device_bytes(const sgpu_ctx* c, uint64_t* bytes) {
    if (!c || !bytes) return SGPU_ERR_ARG;
    uint64_t b = (uint64_t)c->vol * 6 * (sizeof(float) + sizeof(int16_t) + sizeof(uint8_t));
    for (int f = 0; f < 6; ++f)
        for (int w = 0; w < 2; ++w)
            for (int s = 0; s < 2; ++s) {
                const Slab& sl = c->cpml.s[f][w][s];
                if (sl.psi) b += (uint64_t)sl.px * (sl.yhi - sl.ylo + 1) * (sl.zhi - sl.zlo + 1) * 4;
            }
    for (int comp = 0; comp < 3; ++comp) {
        b += (uint64_t)c->disp.n[comp] * (4 + 1 + 4 + 16 * (uint64_t)std::max(1, c->disp.nu_max));
        b += (uint64_t)c->mdisp.n[comp] * (4 + 1 + 4 + 16 * (uint64_t)std::max(1, c->mdisp.nu_max));
    }
    b += (uint64_t)c->border.mur_cells * 2 * sizeof(float);
    *bytes = b;
    return SGPU_OK;
}

}  // extern "C"

sgpu_status sgpu::rebuild_sources(sgpu_ctx* c) {
    if (!c->src_dirty) return SGPU_OK;
    return build_sources(c);
}
