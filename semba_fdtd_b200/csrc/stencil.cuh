// Per-cell device arithmetic shared by the single-problem kernels
// (kernels.cu) and the batched kernels (batch.cu).  Each function restates
// one reference routine in its operation order; nothing here rounds
// differently from a separate multiply and add, so a -fmad=false build
// reproduces the reference FP32 build bit for bit.
#pragma once
#include "sgpu_internal.h"

namespace sgpu {
namespace dev {

enum : int { kBulk = 1, kCpml = 2, kCx = 4, kCy = 8, kCz = 16, kAll = kCx | kCy | kCz };
constexpr int kShTable = 4096;  // media entries held in shared memory

__device__ __forceinline__ long long slab_index(const Slab& s, int i, int j, int k) {
    return (i - s.xb) + (long long)s.px * ((j - s.ylo) + (long long)(s.yhi - s.ylo + 1) * (k - s.zlo));
}
__device__ __forceinline__ float* slab_ptr(const Slab& s, int i, int j, int k) {
    if (i < s.xlo || i > s.xhi || j < s.ylo || j > s.yhi || k < s.zlo || k > s.zhi) return nullptr;
    return s.psi + slab_index(s, i, j, k);
}

// True when the (x, y) column range [x0,x1]x[y0,y1] or the z range [z0,z1]
// can touch the slab.
__device__ __forceinline__ bool slab_touches(const Slab& s, int x0, int x1, int y0, int y1, int z0, int z1) {
    return s.psi && x1 >= s.xlo && x0 <= s.xhi && y1 >= s.ylo && y0 <= s.yhi && z1 >= s.zlo && z0 <= s.zhi;
}

// Slab masks: a tile only looks up the slabs that can hold its cells.  Bit
// 4*q + 2*kind + side stands for slab cp.s[c0+q][kind][side] of the three
// components c0..c0+2 of a half step.  cpml_tile_mask keeps the slabs whose
// x-y extent meets the tile's columns (once per tile); cpml_plane_mask keeps
// those whose z extent holds plane k (once per plane).  Both are uniform
// over the tile, so a plane that touches no slab runs the bulk path.
__device__ __forceinline__ unsigned cpml_tile_mask(const KCpml& cp, int c0, int x0, int x1, int y0, int y1) {
    unsigned m = 0;
    if (!cp.on) return 0;
#pragma unroll
    for (int n = 0; n < 12; ++n) {
        const Slab& s = cp.s[c0 + (n >> 2)][(n >> 1) & 1][n & 1];
        if (s.psi && x1 >= s.xlo && x0 <= s.xhi && y1 >= s.ylo && y0 <= s.yhi) m |= 1u << n;
    }
    return m;
}
__device__ __forceinline__ unsigned cpml_plane_mask(const KCpml& cp, int c0, unsigned tile, int k) {
    unsigned m = 0;
#pragma unroll
    for (int n = 0; n < 12; ++n) {
        const Slab& s = cp.s[c0 + (n >> 2)][(n >> 1) & 1][n & 1];
        if (((tile >> n) & 1) && k >= s.zlo && k <= s.zhi) m |= 1u << n;
    }
    return m;
}

// Slabs by the axis their coefficients run along (the same for the E and H
// sides): x -- comp 1 kind 1, comp 2 kind 1; y -- comp 0 kind 0, comp 2
// kind 0; z -- comp 0 kind 1, comp 1 kind 0.
constexpr unsigned kCpmlX = 0xCC0u, kCpmlY = 0x303u, kCpmlZ = 0x03Cu;

// Per-thread CPML view of one tile: `col` flags the slabs whose x-y extent
// holds the thread's column (i, j), and the P_b / P_c values indexed by i
// and j are loaded once (only where some slab needs them, so i and j are in
// range).
struct CpmlCol {
    unsigned col;    // slabs holding the column
    unsigned zall;   // ... of them, those holding every plane kb..ke
    float bx, cx, by, cy;
    // slabs holding cell (i, j, k) of the column, kb <= k <= ke
    __device__ __forceinline__ unsigned live(const KCpml& cp, int c0, int k) const {
        const unsigned zsome = col & ~zall;
        return zsome ? zall | cpml_plane_mask(cp, c0, zsome, k) : zall;
    }
};
__device__ __forceinline__ CpmlCol cpml_col(const KCpml& cp, int c0, unsigned tile, int i, int j, int kb, int ke) {
    CpmlCol r;
    r.col = 0;
    r.zall = 0;
#pragma unroll
    for (int n = 0; n < 12; ++n) {
        const Slab& s = cp.s[c0 + (n >> 2)][(n >> 1) & 1][n & 1];
        if (((tile >> n) & 1) && i >= s.xlo && i <= s.xhi && j >= s.ylo && j <= s.yhi) {
            r.col |= 1u << n;
            if (s.zlo <= kb && s.zhi >= ke) r.zall |= 1u << n;
        }
    }
    const bool h = c0 != 0;
    r.bx = r.cx = r.by = r.cy = 0.0f;
    if (r.col & kCpmlX) {
        r.bx = (h ? cp.pbm[0] : cp.pbe[0])[i];
        r.cx = (h ? cp.pcm[0] : cp.pce[0])[i];
    }
    if (r.col & kCpmlY) {
        r.by = (h ? cp.pbm[1] : cp.pbe[1])[j];
        r.cy = (h ? cp.pcm[1] : cp.pce[1])[j];
    }
    return r;
}

// One CPML correction of the reference (borderscpml.F90:584-1176):
//   psi = P_b(c) * psi + diff * P_c(c) ;  F = F +- g * psi
// for the slab pair whose two live bits are `live2` (side 0 first; the two
// sides lie at opposite ends of the axis and share no cell), with the
// P_b(c) / P_c(c) values already loaded.
template <bool ADD>
__device__ __forceinline__ float cpml_pair(const Slab (&s)[2], unsigned live2, int i, int j, int k, float pb, float pc,
                                           float diff, float g, float v, bool& touched) {
    if (live2) {
        const bool a = live2 & 1;
        float* const psi = a ? s[0].psi : s[1].psi;
        const int xb = a ? s[0].xb : s[1].xb, px = a ? s[0].px : s[1].px;
        const int ylo = a ? s[0].ylo : s[1].ylo, yhi = a ? s[0].yhi : s[1].yhi;
        const int zlo = a ? s[0].zlo : s[1].zlo;
        float* p = psi + ((i - xb) + (long long)px * ((j - ylo) + (long long)(yhi - ylo + 1) * (k - zlo)));
        const float ps = pb * (*p) + diff * pc;
        *p = ps;
        v = ADD ? v + g * ps : v - g * ps;
        touched = true;
    }
    return v;
}

// Staged psi slots: a tile's slabs take slots in bit order, except that the
// two sides of the z-normal slab pairs (bits 2/3 and 4/5, the z kinds of the
// side's first two components) share one slot, since a plane lies in at most
// one of them.
__device__ __forceinline__ unsigned psi_slot_groups(unsigned m) { return (m & ~0x28u) | ((m >> 1) & 0x14u); }
__device__ __forceinline__ int psi_slot(unsigned m, int n) {
    const int b = (n == 3 || n == 5) ? n - 1 : n;
    return __popc(psi_slot_groups(m) & ((1u << b) - 1u));
}

// A staged tile's psi rows, per consumer warp and slab bit n: the psi address
// of the warp's first column (ib, row j) at plane 0, the plane stride (a cell's
// psi is base + lane + k * stride) and the first float of the slab's staged
// slot (psi_slot of the tile's slabs `tmask`).  Bits outside tmask get a
// null row at slot 0.
struct PsiRow {
    float* base;
    int stride;
    int slot;
};
__device__ __forceinline__ void psi_rows_fill(PsiRow* rows, const KCpml& cp, int c0, unsigned tmask, int slot_floats,
                                              int ib, int j, int lane) {
    if (lane < 12) {
        PsiRow r{nullptr, 0, 0};
        if ((tmask >> lane) & 1u) {
            const Slab& sl = cp.s[c0 + (lane >> 2)][(lane >> 1) & 1][lane & 1];
            r.stride = sl.px * (sl.yhi - sl.ylo + 1);
            r.base = sl.psi + ((ib - sl.xb) + (long long)sl.px * (j - sl.ylo) - (long long)r.stride * sl.zlo);
            r.slot = psi_slot(tmask, lane) * slot_floats;
        }
        rows[lane] = r;
    }
    __syncwarp();
}

// The same correction with the old psi value taken from a shared-memory
// tile staged by TMA (slab number nbase + side within the side's 12, cell
// offset o in the 32 x 8 tile); the new value goes to global memory with a
// plain store through the warp's psi row table.
template <bool ADD>
__device__ __forceinline__ float cpml_pair_staged(unsigned live2, int nbase, const float* slots, int o, const PsiRow* rows,
                                                  int lane, int k, float pb, float pc, float diff, float g, float v) {
    if (live2) {
        const PsiRow r = rows[nbase + ((live2 & 1) ? 0 : 1)];
        const float ps = pb * slots[r.slot + o] + diff * pc;
        r.base[lane + (long long)k * r.stride] = ps;
        v = ADD ? v + g * ps : v - g * ps;
    }
    return v;
}

// Block geometry shared by the two field kernels: 32 x BY threads, each
// owning one (i, j) column and marching over a z chunk.  x starts at local 0
// so every warp load covers one aligned 128-byte line.
constexpr int kBX = 32, kBY = 8;

// Advance_Ex/Ey/Ez (timestepping.F90:2165-2285) fused with
// AdvanceelectricCPML (borderscpml.F90:584-876).  Each field value is read
// once per cell; the curl update and, in blocks that touch a PML slab, the
// CPML corrections (in the reference's region order) are applied to the
// register value before a single store.  Hx and Hy of plane k-1 are carried
// in registers from the previous iteration; the i-1 neighbours come from the
// next lower lane.
template <int MODE, bool CP>
__device__ __forceinline__ void efield_column(const KGrid& g, const KCpml& cp, const float* t1, const float* t2, int i, int j,
                                              int kb, int ke, bool vx, bool vy, bool vz) {
    const long long pitch = g.pitch, plane = g.plane;
    float* __restrict__ Ex = g.F[0];
    float* __restrict__ Ey = g.F[1];
    float* __restrict__ Ez = g.F[2];
    const float* __restrict__ Hx = g.F[3];
    const float* __restrict__ Hy = g.F[4];
    const float* __restrict__ Hz = g.F[5];
    const int16_t* __restrict__ Mx = g.M[0];
    const int16_t* __restrict__ My = g.M[1];
    const int16_t* __restrict__ Mz = g.M[2];
    const bool lane0 = (threadIdx.x & 31) == 0;
    const float idyh = g.idyh[j], idxh = g.idxh[i];
    long long c = i + pitch * j + plane * kb;
    float hx_km = __ldg(Hx + c - plane), hy_km = __ldg(Hy + c - plane);
    // slabs that can hold this block's cells (its 32 x blockDim.y columns);
    // threads on clamped rows store nothing, so their mask does not matter
    const int bx0 = i & ~31, by0 = j - (int)threadIdx.y;
    const unsigned tmask = CP ? cpml_tile_mask(cp, 0, bx0, bx0 + 31, by0, by0 + (int)blockDim.y - 1) : 0u;
    const CpmlCol cc = CP ? cpml_col(cp, 0, tmask, i, j, kb, ke) : CpmlCol{};
    for (int k = kb; k <= ke; ++k, c += plane) {
        const unsigned pm = CP ? cc.live(cp, 0, k) : 0u;
        float bz = 0.0f, cz = 0.0f;
        if (CP && (pm & kCpmlZ)) {
            bz = cp.pbe[2][k];
            cz = cp.pce[2][k];
        }
        const float hx = __ldg(Hx + c), hy = __ldg(Hy + c), hz = __ldg(Hz + c);
        float hz_im = __shfl_up_sync(0xffffffffu, hz, 1);
        float hy_im = __shfl_up_sync(0xffffffffu, hy, 1);
        if (lane0) {
            hz_im = __ldg(Hz + c - 1);
            hy_im = __ldg(Hy + c - 1);
        }
        const float idzh = g.idzh[k];
        if ((MODE & kCx) && vx && k >= g.sw[0][4] && k <= g.sw[0][5]) {
            float e = Ex[c];
            const int m = __ldg(Mx + c);
            const float dy = hz - __ldg(Hz + c - pitch);
            const float dz = hy - hy_km;
            bool st = (MODE & kBulk) != 0;
            if (MODE & kBulk) e = t1[m] * e + t2[m] * (dy * idyh - dz * idzh);
            if (CP && pm) {
                const float gg = t2[m];
                e = cpml_pair<true>(cp.s[0][0], pm & 3, i, j, k, cc.by, cc.cy, dy, gg, e, st);
                e = cpml_pair<false>(cp.s[0][1], (pm >> 2) & 3, i, j, k, bz, cz, dz, gg, e, st);
            }
            if (st) Ex[c] = e;
        }
        if ((MODE & kCy) && vy && k >= g.sw[1][4] && k <= g.sw[1][5]) {
            float e = Ey[c];
            const int m = __ldg(My + c);
            const float dz = hx - hx_km;
            const float dx = hz - hz_im;
            bool st = (MODE & kBulk) != 0;
            if (MODE & kBulk) e = t1[m] * e + t2[m] * (dz * idzh - dx * idxh);
            if (CP && pm) {
                const float gg = t2[m];
                e = cpml_pair<true>(cp.s[1][0], (pm >> 4) & 3, i, j, k, bz, cz, dz, gg, e, st);
                e = cpml_pair<false>(cp.s[1][1], (pm >> 6) & 3, i, j, k, cc.bx, cc.cx, dx, gg, e, st);
            }
            if (st) Ey[c] = e;
        }
        if ((MODE & kCz) && vz && k >= g.sw[2][4] && k <= g.sw[2][5]) {
            float e = Ez[c];
            const int m = __ldg(Mz + c);
            const float dx = hy - hy_im;
            const float dy = hx - __ldg(Hx + c - pitch);
            bool st = (MODE & kBulk) != 0;
            if (MODE & kBulk) e = t1[m] * e + t2[m] * (dx * idxh - dy * idyh);
            if (CP && pm) {
                const float gg = t2[m];
                e = cpml_pair<false>(cp.s[2][0], (pm >> 8) & 3, i, j, k, cc.by, cc.cy, dy, gg, e, st);
                e = cpml_pair<true>(cp.s[2][1], (pm >> 10) & 3, i, j, k, cc.bx, cc.cx, dx, gg, e, st);
            }
            if (st) Ez[c] = e;
        }
        hx_km = hx;
        hy_km = hy;
    }
}


__device__ __forceinline__ bool col_in(const int* s, int i, int j) { return i >= s[0] && i <= s[1] && j >= s[2] && j <= s[3]; }

// Advance_Hx/Hy/Hz (timestepping.F90:2294-2409) fused with
// AdvanceMagneticCPML (borderscpml.F90:881-1176).  Ex and Ey of plane k+1
// are loaded once and carried to the next iteration; the i+1 neighbours come
// from the next higher lane.
template <int MODE, bool CP>
__device__ __forceinline__ void hfield_column(const KGrid& g, const KCpml& cp, const float* t1, const float* t2, int i, int j,
                                              int kb, int ke, bool vx, bool vy, bool vz) {
    const long long pitch = g.pitch, plane = g.plane;
    const float* __restrict__ Ex = g.F[0];
    const float* __restrict__ Ey = g.F[1];
    const float* __restrict__ Ez = g.F[2];
    float* __restrict__ Hx = g.F[3];
    float* __restrict__ Hy = g.F[4];
    float* __restrict__ Hz = g.F[5];
    const int16_t* __restrict__ Mx = g.M[3];
    const int16_t* __restrict__ My = g.M[4];
    const int16_t* __restrict__ Mz = g.M[5];
    const bool lane31 = (threadIdx.x & 31) == 31;
    const float idye = g.idye[j], idxe = g.idxe[i];
    long long c = i + pitch * j + plane * kb;
    float ex_k = __ldg(Ex + c), ey_k = __ldg(Ey + c);
    const int bx0 = i & ~31, by0 = j - (int)threadIdx.y;
    const unsigned tmask = CP ? cpml_tile_mask(cp, 3, bx0, bx0 + 31, by0, by0 + (int)blockDim.y - 1) : 0u;
    const CpmlCol cc = CP ? cpml_col(cp, 3, tmask, i, j, kb, ke) : CpmlCol{};
    for (int k = kb; k <= ke; ++k, c += plane) {
        const unsigned pm = CP ? cc.live(cp, 3, k) : 0u;
        float bz = 0.0f, cz = 0.0f;
        if (CP && (pm & kCpmlZ)) {
            bz = cp.pbm[2][k];
            cz = cp.pcm[2][k];
        }
        const float ez = __ldg(Ez + c);
        const float ex_kp = __ldg(Ex + c + plane), ey_kp = __ldg(Ey + c + plane);
        float ez_ip = __shfl_down_sync(0xffffffffu, ez, 1);
        float ey_ip = __shfl_down_sync(0xffffffffu, ey_k, 1);
        if (lane31) {
            ez_ip = __ldg(Ez + c + 1);
            ey_ip = __ldg(Ey + c + 1);
        }
        const float idze = g.idze[k];
        if ((MODE & kCx) && vx && k >= g.sw[3][4] && k <= g.sw[3][5]) {
            float h = Hx[c];
            const int m = __ldg(Mx + c);
            const float dz = ey_kp - ey_k;
            const float dy = __ldg(Ez + c + pitch) - ez;
            bool st = (MODE & kBulk) != 0;
            if (MODE & kBulk) h = t1[m] * h + t2[m] * (dz * idze - dy * idye);
            if (CP && pm) {
                const float gg = t2[m];
                h = cpml_pair<false>(cp.s[3][0], pm & 3, i, j, k, cc.by, cc.cy, dy, gg, h, st);
                h = cpml_pair<true>(cp.s[3][1], (pm >> 2) & 3, i, j, k, bz, cz, dz, gg, h, st);
            }
            if (st) Hx[c] = h;
        }
        if ((MODE & kCy) && vy && k >= g.sw[4][4] && k <= g.sw[4][5]) {
            float h = Hy[c];
            const int m = __ldg(My + c);
            const float dx = ez_ip - ez;
            const float dz = ex_kp - ex_k;
            bool st = (MODE & kBulk) != 0;
            if (MODE & kBulk) h = t1[m] * h + t2[m] * (dx * idxe - dz * idze);
            if (CP && pm) {
                const float gg = t2[m];
                h = cpml_pair<false>(cp.s[4][0], (pm >> 4) & 3, i, j, k, bz, cz, dz, gg, h, st);
                h = cpml_pair<true>(cp.s[4][1], (pm >> 6) & 3, i, j, k, cc.bx, cc.cx, dx, gg, h, st);
            }
            if (st) Hy[c] = h;
        }
        if ((MODE & kCz) && vz && k >= g.sw[5][4] && k <= g.sw[5][5]) {
            float h = Hz[c];
            const int m = __ldg(Mz + c);
            const float dy = __ldg(Ex + c + pitch) - ex_k;
            const float dx = ey_ip - ey_k;
            bool st = (MODE & kBulk) != 0;
            if (MODE & kBulk) h = t1[m] * h + t2[m] * (dy * idye - dx * idxe);
            if (CP && pm) {
                const float gg = t2[m];
                h = cpml_pair<true>(cp.s[5][0], (pm >> 8) & 3, i, j, k, cc.by, cc.cy, dy, gg, h, st);
                h = cpml_pair<false>(cp.s[5][1], (pm >> 10) & 3, i, j, k, cc.bx, cc.cx, dx, gg, h, st);
            }
            if (st) Hz[c] = h;
        }
        ex_k = ex_kp;
        ey_k = ey_kp;
    }
}


// a / dt, correctly rounded, from y = RN(1/dt): q = RN(a*y), the exact
// residual r = a - dt*q by FMA, then RN(q + r*y) -- Markstein's correction,
// which returns RN(a/dt) whenever y is the correctly rounded reciprocal and
// no intermediate underflows (P. Markstein, IBM J. Res. Dev. 34(1), 1990;
// J.-M. Muller et al., Handbook of Floating-Point Arithmetic, section 4.7).
// Two FMAs and a multiply replace the IEEE division sequence; the oracle's
// tests check it against IEEE division on random operands.
__device__ __forceinline__ double div_dt(double a, double dt, double inv_dt) {
    const double q = a * inv_dt;
    const double r = fma(-q, dt, a);
    return fma(r, inv_dt, q);
}

// AdvanceEDispersiveE (electricdispersive.F90:304-362) and, with MAG,
// AdvanceMdispersiveH (magneticdispersive.F90:298-360): one thread per node.
// Conjugate poles share one state slot; the subtraction still runs once
// per pole of the reference, in its order, and Re(conj(g)*conj(J)) equals
// Re(g*J) exactly.  The electric current takes (Beta*(E-Eprev))/dt, the
// magnetic one (Beta/dt)*(H-Hprev), as the two routines are written.  NU
// (the largest number of state slots of any medium) is a template parameter
// so the states stay in registers.
// One component's node arrays and field, gathered once per launch or work
// item so the per-node code reads no descriptor.
struct AdeRefs {
    const int* node;
    const uint8_t* med;
    const int4* grp;
    float* prev;
    double2* J;  // [node][state slot], ju slots a node
    long long n;
    int ju;
    const DispMedium* media;
    float* F;
    double dt, inv_dt;
};
template <bool MAG> __device__ __forceinline__ AdeRefs ade_refs(const KGrid& g, const KDisp& d, int comp) {
    return AdeRefs{d.node[comp], d.med[comp], d.grp[comp], d.prev[comp], d.J[comp], d.n[comp], max(1, d.nu_max),
                   d.media, g.F[MAG ? 3 + comp : comp], d.dt, d.inv_dt};
}

// Node q's cell and medium slot.  Nodes are numbered in cell order, so the 32
// nodes of a group usually form one or two runs of consecutive cells of one
// medium each; the group's descriptor then gives both (one 16-byte load the
// warp shares), and only groups of more than two runs read the per-node
// index and slot arrays.
__device__ __forceinline__ void ade_where(const AdeRefs& d, long long q, int& idx, int& slot) {
    if (d.grp) {
        const int4 gd = __ldg(d.grp + (q >> 5));
        if (gd.z >= 0) {
            const int lane = (int)(q & 31);
            const bool second = lane >= gd.z;
            idx = (second ? gd.y : gd.x) + lane;
            slot = second ? (gd.w >> 8) & 255 : gd.w & 255;
            return;
        }
    }
    idx = d.node[q];
    slot = d.med[q];
}

// The node's update in three parts (loads, arithmetic, stores), so a thread
// can issue the loads of several nodes before any store.  With UNI (every
// medium has NU state slots) the state loads depend on nothing but q.
template <int NU> struct AdeNode {
    int idx;
    const DispMedium* md;
    float e, prev;
    double2 st[NU];
};

template <int NU, bool UNI>
__device__ __forceinline__ void ade_load(const AdeRefs& d, long long q, AdeNode<NU>& a) {
    if (UNI) {
#pragma unroll
        for (int u = 0; u < NU; ++u) a.st[u] = d.J[q * d.ju + u];
        a.prev = d.prev[q];
    }
    int slot;
    ade_where(d, q, a.idx, slot);
    a.md = d.media + slot;
    if (!UNI) {
        const int nu = a.md->nu;
#pragma unroll
        for (int u = 0; u < NU; ++u) a.st[u] = u < nu ? d.J[q * d.ju + u] : make_double2(0.0, 0.0);
        a.prev = d.prev[q];
    }
    a.e = d.F[a.idx];
}

template <int NU, bool MAG, bool UNI>
__device__ __forceinline__ void ade_update(const AdeRefs& d, AdeNode<NU>& a) {
    const DispMedium* __restrict__ md = a.md;
    const int nu = UNI ? NU : md->nu;
    float e = a.e;
    for (int p = 0; p < md->np; ++p) {
        const int up = md->map[p];
        double jr = 0.0, ji = 0.0;
#pragma unroll
        for (int u = 0; u < NU; ++u)
            if (u == up) { jr = a.st[u].x; ji = a.st[u].y; }
        const double2 g3 = md->g3[up];
        const double re = g3.x * jr - g3.y * ji;
        e = (float)((double)e - re);
    }
    const double dd = (double)(e - a.prev);
#pragma unroll
    for (int u = 0; u < NU; ++u) {
        if (u < nu) {
            const double2 kp = md->kappa[u], bt = md->beta[u];
            const double kr = kp.x * a.st[u].x - kp.y * a.st[u].y;
            const double ki = kp.x * a.st[u].y + kp.y * a.st[u].x;
            double br, bi;
            if (MAG) {
                // (Beta/dt)*(H - Hprev): Beta/dt is the same quotient for every
                // node, formed once on the host
                const double2 bd = md->beta_dt[u];
                br = bd.x * dd;
                bi = bd.y * dd;
            } else {
                br = div_dt(bt.x * dd, d.dt, d.inv_dt);
                bi = div_dt(bt.y * dd, d.dt, d.inv_dt);
            }
            a.st[u] = make_double2(kr + br, ki + bi);
        }
    }
    a.e = e;
}

template <int NU, bool UNI>
__device__ __forceinline__ void ade_store(const AdeRefs& d, long long q, const AdeNode<NU>& a) {
    const int nu = UNI ? NU : a.md->nu;
#pragma unroll
    for (int u = 0; u < NU; ++u)
        if (u < nu) d.J[q * d.ju + u] = a.st[u];
    d.prev[q] = a.e;
    d.F[a.idx] = a.e;
}

template <int NU, bool MAG, bool UNI>
__device__ __forceinline__ void ade_node(const AdeRefs& d, long long q) {
    AdeNode<NU> a;
    ade_load<NU, UNI>(d, q, a);
    ade_update<NU, MAG, UNI>(d, a);
    ade_store<NU, UNI>(d, q, a);
}

__device__ __forceinline__ int step_of(const StepRef& s) { return (s.dev_n ? *s.dev_n : 0) + s.n; }

// Whether one half step of side `side` (0: E, evaluated at time t) keeps the
// global plane-wave switch up: Incid raises still_planewave_time for every
// face node whose retarded time is still inside its waveform table, nprev + 1
// <= numus (planewaves.F90:830-832).  nprev = int((t - d/c) / delta) never
// decreases with t and never increases with d, so some node of a wave keeps
// the switch up exactly when its node of largest d/c does.
__device__ __forceinline__ bool pw_side_active(const KSrc& s, int side, float t) {
    for (int q = 0; q < s.ntab; ++q) {
        const SrcTable tb = s.tab[q];
        if (!tb.is_pw || !tb.has[side]) continue;
        const long long nprev = (long long)((t - tb.amax[side]) / tb.delta);
        if (nprev + 1 <= tb.numus) return true;
    }
    return false;
}

// still_planewave_time before half step h = 2n + hside (timestepping.F90:1219,
// :1251-1267, :1423, :1596): up at the first half step run, then lowered by
// every AdvancePlaneWaveE/H (planewaves.F90:904, :1204) and raised again by
// its active nodes, and once down no plane-wave routine runs again.  So it is
// up iff every half step from h_first to h - 1 kept it up; each side's
// activity only falls as its time grows, so that is iff the last E half and
// the last H half before h (those at or after h_first) did.
__device__ __forceinline__ bool pw_switch_up(const KSrc& s, int n, const double* tiempo, int t_n0, double dt, int hside) {
    const int mE = hside ? n : n - 1, mH = n - 1;
    if (2 * mE >= s.h_first && !pw_side_active(s, 0, (float)tiempo[mE - t_n0])) return false;
    if (2 * mH + 1 >= s.h_first && !pw_side_active(s, 1, (float)(tiempo[mH - t_n0] + (double)0.5f * dt)))
        return false;
    return true;
}

// The switch for a whole block of source rows of one half step: thread 0
// evaluates it, every thread of the block returns it (all must call).
__device__ __forceinline__ bool pw_switch_block(const KSrc& s, int n, const double* tiempo, int t_n0, double dt, int hside) {
    __shared__ int on;
    __syncthreads();  // the previous call's value has been read
    if (threadIdx.x == 0) on = pw_switch_up(s, n, tiempo, t_n0, dt, hside) ? 1 : 0;
    __syncthreads();
    return on != 0;
}

// AdvancePlaneWaveE/H (planewaves.F90:878-1475) with Incid/evolucion
// (:778-853) and AdvanceNodalE/H (nodalsources.F90:310-777): source row r
// (one touched node) applies that node's contributions in the reference
// order; plane-wave contributions only while the global switch (pw_on) is up.
__device__ __forceinline__ void source_row(const KGrid& g, const KSrc& s, int n, const double* tiempo, int t_n0, double dt,
                                           int hside, int mask, int r, bool pw_on) {
    const double tn = tiempo[n - t_n0];
    const float t = hside ? (float)(tn + (double)0.5f * dt) : (float)tn;
    const float G21 = hside ? g.gm2[1] : g.g2[1];
    float* F = g.F[s.row_comp[r]];
    const int node = s.row_node[r];
    float v = F[node];
    for (int p = s.row_ptr[r]; p < s.row_ptr[r + 1]; ++p) {
        const SrcEntry en = s.e[p];
        if (!((1 << en.type) & mask)) continue;
        const SrcTable tb = s.tab[en.table];
        const float* ev0 = s.samples + tb.offset;
        if (en.type == kSrcPlaneWave) {
            if (!pw_on) continue;
            float ev = 0.0f;
            const long long nprev = (long long)((t - en.a) / tb.delta);
            if (nprev + 1 <= tb.numus && nprev > 0)
                ev = (ev0[nprev + 1] - ev0[nprev]) / tb.delta * ((t - en.a) - (float)nprev * tb.delta) + ev0[nprev];
            const float inc = 0.0f + en.b * ev;
            v = v + G21 * inc * en.c;
        } else {
            float ev = 0.0f;
            const long long nprev = (long long)(t / tb.delta);
            if (!((nprev + 1 > tb.numus) || (nprev + 1 <= 0)))
                ev = (ev0[nprev + 1] - ev0[nprev]) / tb.delta * ((t) - (float)nprev * tb.delta) + ev0[nprev];
            if (en.type == kSrcNodalSoft) v = v - en.a * ev;
            else v = en.a * ev;
        }
    }
    F[node] = v;
}

// UpdateObservation point probes (observation.F90:2633-2668).
__device__ __forceinline__ void probe_one(const KGrid& g, const KProbes& p, int n, int first_n, int q) {
    const long long row = (long long)(n - first_n) % p.cap;
    p.ring[row * p.n + q] = g.F[p.comp[q]][p.idx[q]];
}

// Cell q of the flattened clone planes, for the face kinds in `mask` (2 PMC,
// 4 periodic, 6 both).  MinusCloneMagneticPMC and CloneMagneticPeriodic
// (bordersother.F90:65-190) assign whole planes one face after another, each
// spanning the component's Alloc extent, so a cell outside two or three such
// faces ends up with the composition of their maps (the later assignment
// reads the value the earlier one wrote in the same call).  Each cell here
// computes that composition directly from swept cells -- a PMC face maps the
// outer layer to the first swept one with a sign flip, a periodic face to the
// swept layer at the other end -- so no cell reads a cell another thread of
// the launch writes, and each cell is written once (by the first of its
// faces in part order).
__device__ __forceinline__ void clone_cell(const KGrid& g, const KBorder& b, int mask, long long q) {
    if (q >= b.cl_cells) return;
    int p = 0;
    while (p + 1 < b.ncl && q >= b.cl[p + 1].first) ++p;
    const ClonePart& cp = b.cl[p];
    if (!(b.face_kind[cp.axis][cp.side] & mask)) return;
    const int c = cp.comp;
    const int ua = cp.axis == 0 ? 1 : 0, va = cp.axis == 2 ? 1 : 2;
    const long long r = q - cp.first;
    const int nu = b.ahi[c][ua] - b.alo[c][ua] + 1;
    int pos[3];
    pos[cp.axis] = cp.side ? b.ghi[c][cp.axis] : b.glo[c][cp.axis];
    pos[ua] = b.alo[c][ua] + (int)(r % nu);
    pos[va] = b.alo[c][va] + (int)(r / nu);
    for (int e = 0; e < p; ++e) {
        const ClonePart& o = b.cl[e];
        if (o.comp == c && (b.face_kind[o.axis][o.side] & mask) &&
            pos[o.axis] == (o.side ? b.ghi[c][o.axis] : b.glo[c][o.axis]))
            return;
    }
    int src[3] = {pos[0], pos[1], pos[2]};
    bool neg = false;
    for (int a = 0; a < 3; ++a) {
        if (a == c) continue;  // only the faces tangential to the component
        for (int sd = 0; sd < 2; ++sd) {
            const int k = b.face_kind[a][sd];
            if (!(k & mask) || pos[a] != (sd ? b.ghi[c][a] : b.glo[c][a])) continue;
            if (k == 2) {
                src[a] = sd ? b.shi[c][a] : b.slo[c][a];
                neg = !neg;
            } else {
                src[a] = sd ? b.slo[c][a] : b.shi[c][a];
            }
        }
    }
    float* F = g.F[3 + c];
    const float v = F[src[0] + (long long)g.pitch * src[1] + g.plane * src[2]];
    F[pos[0] + (long long)g.pitch * pos[1] + g.plane * pos[2]] = neg ? -v : v;
}

// Cell q of the flattened Mur layers: AdvanceMagneticMUR, first order
// (bordersmur.F90:1129-1383), and the storage of Past_ (:1396-1650):
//   H(outer) = Past(inner) + CAB1(medium of the inner node) * (H(inner) - Past(outer))
//   Past(outer) = H(outer), Past(inner) = H(inner)
// A part reads its inner layer, which no part writes, so the store can
// follow the update in the same thread.
__device__ __forceinline__ void mur_cell(const KGrid& g, const KBorder& b, long long q) {
    if (q >= b.mur_cells) return;
    int p = 0;
    while (p + 1 < b.nmur && q >= b.mur[p + 1].first) ++p;
    const MurPart& m = b.mur[p];
    const long long r = q - m.first;
    const int ua = m.axis == 0 ? 1 : 0, va = m.axis == 2 ? 1 : 2;
    int pos[3];
    pos[ua] = m.u0 + (int)(r % m.nu);
    pos[va] = m.v0 + (int)(r / m.nu);
    pos[m.axis] = m.outer;
    const long long no = pos[0] + (long long)g.pitch * pos[1] + g.plane * pos[2];
    pos[m.axis] = m.inner;
    const long long ni = pos[0] + (long long)g.pitch * pos[1] + g.plane * pos[2];
    float* F = g.F[m.comp];
    const long long layer = (long long)m.nu * m.nv;
    const float past_outer = m.past[r], past_inner = m.past[layer + r];
    const float h_inner = F[ni];
    const float h = past_inner + m.cab1[g.M[m.comp][ni]] * (h_inner - past_outer);
    F[no] = h;
    m.past[r] = h;
    m.past[layer + r] = h_inner;
}

}  // namespace dev
}  // namespace sgpu
