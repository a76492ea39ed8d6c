// Near-to-far-field transform (farfield.F90).
//
// UpdateFarField (farfield.F90:1163-1733) is a running DFT of the tangential
// fields on the six faces of a box: per sampled step m and frequency f,
//   S[f] += w[m][f] * F(node)
// in complex(8), E samples with the electric weights auxExp_E, H samples on
// two planes per face with auxExp_H.  Every sampled array of every face is a
// patch of one accumulator [nf][samples]; one launch per step covers them
// all (one thread per sample, the frequencies in a loop, so each frequency's
// read-modify-write is coalesced).  The weights follow the reference's
// recursion auxExp <- auxExp * expIwdt and are tabulated on the host.
//
// FlushFarfield (:2408-3423) runs once at the end: a first kernel forms the
// equivalent currents M = n x E and J = n x H of every surface cell (the two
// H planes averaged arithmetically and geometrically, farfield.F90:3553), a
// second reduces update_LN (:3426) over all cells for one (frequency,
// direction) per block and writes Etheta, Ephi and the two RCS values.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "sgpu_internal.h"
#include "stencil.cuh"

using namespace sgpu;
using sgpu::dev::step_of;

namespace {

constexpr float kPiF = 3.14159265358979323846f;  // pi of kind RKIND (fdetypes.F90:188)

struct FarArgs {
    FarPatch patch[kFarPatches];
    int npatch, samples, nf, ndecim, w_m;
    double2* acc;
    const double2* wE;
    const double2* wH;
};

__global__ void k_farfield_acc(KGrid g, FarArgs a, StepRef sr, int ox, int oy, int oz) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.samples) return;
    const int n = step_of(sr);
    if ((n - 1) % a.ndecim) return;  // mod(ntime-1, Ndecim) /= 0 (Fortran MOD keeps the dividend's sign)
    // sampled steps before this one since step 0: the weight index
    const int m = a.ndecim == 1 ? n : (n - 1) / a.ndecim;
    if (m < 0 || m >= a.w_m) return;
    int p = 0;
    while (p + 1 < a.npatch && q >= a.patch[p + 1].off) ++p;
    const FarPatch& P = a.patch[p];
    const int r = q - P.off, w2 = P.hi2 - P.lo2 + 1;
    const int o = P.lo1 + r / w2, u = P.lo2 + r % w2;
    int i, j, k;
    if (P.axis == 0) { i = P.plane; j = u; k = o; }
    else if (P.axis == 1) { i = u; j = P.plane; k = o; }
    else { i = u; j = o; k = P.plane; }
    const long long c = (long long)(i - ox) + (long long)g.pitch * (j - oy) + g.plane * (long long)(k - oz);
    const double v = (double)g.F[P.comp][c];
    const double2* w = (P.comp >= 3 ? a.wH : a.wE) + (long long)m * a.nf;
    for (int f = 0; f < a.nf; ++f) {
        double2* s = a.acc + (long long)f * a.samples + q;
        double2 x = *s;
        const double2 wf = w[f];
        x.x = x.x + wf.x * v;
        x.y = x.y + wf.y * v;
        *s = x;
    }
}

// One cell of the transform loops: the two E samples (t1 at position A, t2
// at B), the H partners on their two planes, the cell-size factors and the
// signed normal of each of the four currents (0 where the reference's loop
// leaves that current zero).
struct TCell {
    float pa[3], pb[3];
    int col[6];     // Ma, Mb, JA plane 1, JA plane 2, JB plane 1, JB plane 2 (-1: zero)
    float fac[4][3];  // Ma, Mb, JA, JB: two cell sizes and sign * NORMAL
    int ax_ma, ax_mb;  // axes of Ma / Mb; JA has Mb's axis, JB Ma's
};

// Equivalent currents of one cell: Ma, Mb, then JA, JB with the arithmetic
// mean, then JA, JB with the geometric mean.
struct Currents {
    double2 v[6];
};

__device__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// average() of farfield.F90:3553-3579.
__device__ double2 h_average(int pass, double2 z1, double2 z2) {
    if (pass == 1) return make_double2((z1.x + z2.x) / 2.0, (z1.y + z2.y) / 2.0);
    const float phi1 = (float)atan2(z1.y, z1.x), phi2 = (float)atan2(z2.y, z2.x);
    float n1 = phi1, n2 = phi2;
    const float half = kPiF / 2.0f, two = 2.0f * kPiF;
    if (phi1 < -half && phi2 > half) n1 = phi1 - two;
    if (phi2 < -half && phi1 > half) n2 = phi2 - two;
    const float arg = (n1 + n2) / 2.0f;
    float sn, cs;
    sincosf(arg, &sn, &cs);
    const double2 pr = cmul(z1, z2);
    const double r = sqrt(hypot(pr.x, pr.y));
    return make_double2(r * (double)cs, r * (double)sn);
}

__device__ double2 scaled(double2 z, const float* fac) {
    // value * size1 * size2 * (sign * NORMAL), left to right in complex(8)
    z.x = z.x * (double)fac[0];
    z.y = z.y * (double)fac[0];
    z.x = z.x * (double)fac[1];
    z.y = z.y * (double)fac[1];
    z.x = z.x * (double)fac[2];
    z.y = z.y * (double)fac[2];
    return z;
}

__global__ void k_farfield_currents(const TCell* cells, int ncells, const double2* acc, int samples, int nf,
                                    Currents* out) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)ncells * nf) return;
    const int f = (int)(t / ncells), q = (int)(t % ncells);
    const TCell& c = cells[q];
    const double2* A = acc + (long long)f * samples;
    double2 s[6];
    for (int k = 0; k < 6; ++k) s[k] = c.col[k] >= 0 ? A[c.col[k]] : make_double2(0.0, 0.0);
    Currents r;
    const double2 zero = make_double2(0.0, 0.0);
    r.v[0] = c.fac[0][2] != 0.0f ? scaled(s[0], c.fac[0]) : zero;
    r.v[1] = c.fac[1][2] != 0.0f ? scaled(s[1], c.fac[1]) : zero;
    for (int pass = 1; pass <= 2; ++pass) {
        const int o = pass == 1 ? 2 : 4;
        r.v[o] = c.fac[2][2] != 0.0f ? scaled(h_average(pass, s[2], s[3]), c.fac[2]) : zero;
        r.v[o + 1] = c.fac[3][2] != 0.0f ? scaled(h_average(pass, s[4], s[5]), c.fac[3]) : zero;
    }
    out[t] = r;
}

// Direction table: the real(4) trigonometry of FlushFarfield per direction.
struct Dir {
    float theta, phi;
    float stcp, stsp, ct, ctcp, ctsp, st, sp, cp;
};

__device__ __forceinline__ double2 add_scaled(double2 acc, double2 v, double c, double2 e) {
    // acc + (v * c) * e
    const double2 vc = make_double2(v.x * c, v.y * c);
    const double2 p = cmul(vc, e);
    return make_double2(acc.x + p.x, acc.y + p.y);
}

constexpr int kDirThreads = 256;

__global__ void __launch_bounds__(kDirThreads) k_farfield_dir(const TCell* cells, int ncells, const Currents* cur,
                                                                const Dir* dirs, int ndir, const float* freq,
                                                                const double2* dft, float cluz, float zvac,
                                                                double* rows) {
    const int d = blockIdx.x, f = blockIdx.y;
    const Dir D = dirs[d];
    const float fr = freq[f];
    // comun = (0,1) * 2 * pi * freq / cluz in complex(4)
    const double kc = (double)(((2.0f * kPiF) * fr) / cluz);
    const float ctc[3] = {D.ctcp, D.ctsp, -D.st}, cpc[3] = {-D.sp, D.cp, 0.0f};
    // L_theta, L_phi, then N_theta, N_phi of the arithmetic and the geometric pass
    double2 s[6];
    for (int k = 0; k < 6; ++k) s[k] = make_double2(0.0, 0.0);
    const Currents* C = cur + (long long)f * ncells;
    for (int q = threadIdx.x; q < ncells; q += kDirThreads) {
        const TCell& c = cells[q];
        const float da = __fadd_rn(__fadd_rn(__fmul_rn(c.pa[0], D.stcp), __fmul_rn(c.pa[1], D.stsp)), __fmul_rn(c.pa[2], D.ct));
        const float db = __fadd_rn(__fadd_rn(__fmul_rn(c.pb[0], D.stcp), __fmul_rn(c.pb[1], D.stsp)), __fmul_rn(c.pb[2], D.ct));
        double2 ea, eb;
        sincos(kc * (double)da, &ea.y, &ea.x);
        sincos(kc * (double)db, &eb.y, &eb.x);
        const Currents& v = C[q];
        const int ma = c.ax_ma, mb = c.ax_mb;
        s[0] = add_scaled(add_scaled(s[0], v.v[0], (double)ctc[ma], ea), v.v[1], (double)ctc[mb], eb);
        s[1] = add_scaled(add_scaled(s[1], v.v[0], (double)cpc[ma], ea), v.v[1], (double)cpc[mb], eb);
        for (int pass = 0; pass < 2; ++pass) {
            const double2 ja = v.v[2 + 2 * pass], jb = v.v[3 + 2 * pass];
            s[2 + 2 * pass] = add_scaled(add_scaled(s[2 + 2 * pass], ja, (double)ctc[mb], ea), jb, (double)ctc[ma], eb);
            s[3 + 2 * pass] = add_scaled(add_scaled(s[3 + 2 * pass], ja, (double)cpc[mb], ea), jb, (double)cpc[ma], eb);
        }
    }
    __shared__ double red[kDirThreads / 32][12];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < 6; ++k)
        for (int off = 16; off; off >>= 1) {
            s[k].x += __shfl_down_sync(0xffffffffu, s[k].x, off);
            s[k].y += __shfl_down_sync(0xffffffffu, s[k].y, off);
        }
    if (lane == 0)
        for (int k = 0; k < 6; ++k) {
            red[w][2 * k] = s[k].x;
            red[w][2 * k + 1] = s[k].y;
        }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double t[12];
    for (int k = 0; k < 12; ++k) {
        t[k] = 0.0;
        for (int ww = 0; ww < kDirThreads / 32; ++ww) t[k] += red[ww][k];
    }
    const double2 lt = make_double2(t[0], t[1]), lp = make_double2(t[2], t[3]);
    double* row = rows + ((long long)f * ndir + d) * 9;
    row[0] = (double)fr;
    row[1] = (double)D.theta;
    row[2] = (double)D.phi;
    const float q = ((2.0f * kPiF) * fr) / cluz;
    const double hd = hypot(dft[f].x, dft[f].y);
    const double den = (double)(4.0f * kPiF) * (hd * hd);
    const float be = -fr / (2.0f * cluz), bp = fr / (2.0f * cluz);
    for (int pass = 1; pass <= 2; ++pass) {
        const int o = pass == 1 ? 4 : 8;
        const double2 nt = make_double2(t[o], t[o + 1]), np = make_double2(t[o + 2], t[o + 3]);
        // X = L_phi + zvac N_theta, Y = L_theta - zvac N_phi
        const double2 X = make_double2(lp.x + (double)zvac * nt.x, lp.y + (double)zvac * nt.y);
        const double2 Y = make_double2(lt.x - (double)zvac * np.x, lt.y - (double)zvac * np.y);
        const double hx = hypot(X.x, X.y), hy = hypot(Y.x, Y.y);
        const float rcs = (float)((double)(q * q) / den * (hx * hx + hy * hy));
        row[6 + pass] = (double)rcs;
        if (pass == 2) {
            // Etheta = -(0,1) freq / (2 cluz) X, Ephi = (0,1) freq / (2 cluz) Y
            const double2 et = make_double2(-((double)be * X.y), (double)be * X.x);
            const double2 ep = make_double2(-((double)bp * Y.y), (double)bp * Y.x);
            row[3] = hypot(et.x, et.y);
            row[4] = atan2(et.y, et.x);
            row[5] = hypot(ep.x, ep.y);
            row[6] = atan2(ep.y, ep.x);
        }
    }
}

// Tangential E components of a face axis (t1, t2) and the H partner of an
// E component c on that axis.
constexpr int kT[3][2] = {{2, 1}, {2, 0}, {1, 0}};
inline int partner(int axis, int c) { return 3 + (3 - axis - c); }

FarArgs args_of(const FarField& F) {
    FarArgs a;
    for (int p = 0; p < F.npatch; ++p) a.patch[p] = F.patch[p];
    a.npatch = F.npatch;
    a.samples = F.samples;
    a.nf = F.nf;
    a.ndecim = F.ndecim;
    a.w_m = F.w_m;
    a.acc = F.acc;
    a.wE = F.wE;
    a.wH = F.wH;
    return a;
}

// complex(8) product as gfortran forms it (no fused operations)
std::complex<double> cmul_h(std::complex<double> a, std::complex<double> b) {
    const double r = a.real() * b.real() - a.imag() * b.imag();
    const double i = a.real() * b.imag() + a.imag() * b.real();
    return {r, i};
}

// Column of sample (outer o, inner u) in patch p, or -1 outside its ranges.
int column(const FarField& F, int p, int o, int u) {
    if (p < 0) return -1;
    const FarPatch& P = F.patch[p];
    if (P.n == 0 || o < P.lo1 || o > P.hi1 || u < P.lo2 || u > P.hi2) return -1;
    return P.off + (o - P.lo1) * (P.hi2 - P.lo2 + 1) + (u - P.lo2);
}

float at(const std::vector<float>& v, int lo, int i) {
    const int q = i - lo;
    return q >= 0 && q < (int)v.size() ? v[q] : 0.0f;
}

}  // namespace

namespace sgpu {

sgpu_status launch_farfields(sgpu_ctx* c, StepRef sr) {
    for (const FarField& F : c->farfields) {
        if (F.samples == 0) continue;
        const unsigned blocks = (unsigned)((F.samples + 255) / 256);
        k_farfield_acc<<<blocks, 256, 0, c->stream>>>(kgrid(c), args_of(F), sr, c->ox, c->oy, c->oz);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_error(c, SGPU_ERR_CUDA, std::string("k_farfield_acc: ") + cudaGetErrorString(e));
    }
    return SGPU_OK;
}

void free_farfields(sgpu_ctx* c) {
    for (FarField& F : c->farfields) {
        cudaFree(F.acc);
        cudaFree(F.wE);
        cudaFree(F.wH);
        F.acc = F.wE = F.wH = nullptr;
    }
    c->farfields.clear();
}

}  // namespace sgpu

extern "C" {

sgpu_status sgpu_add_farfield(sgpu_ctx* c, const sgpu_farfield_desc* d, int* id) {
    if (!c || !d || d->nfreq < 1 || !d->freq || d->ndecim < 1) return set_error(c, SGPU_ERR_ARG, "bad far-field description");
    if (c->arena) return set_error(c, SGPU_ERR_STATE, "far fields are not kept inside a batch");
    if (c->h_tiempo.empty()) return set_error(c, SGPU_ERR_STATE, "set the time vector before a far field");
    FarField F;
    F.nf = d->nfreq;
    F.ndecim = d->ndecim;
    for (int fc = 0; fc < 6; ++fc) {
        F.active[fc] = d->active[fc] != 0;
        for (int s = 0; s < 6; ++s) F.face_patch[fc][s] = -1;
        if (!F.active[fc]) continue;
        const int axis = fc / 2, low = fc % 2 == 0;
        for (int t = 0; t < 2; ++t) {
            const int* L = d->lim[fc][t];
            const int comp = kT[axis][t];
            const int planes[3] = {L[0], low ? L[0] - 1 : L[0], low ? L[0] : L[0] + 1};
            const int slots[3] = {t, 2 + 2 * t, 3 + 2 * t};
            for (int s = 0; s < 3; ++s) {
                FarPatch& P = F.patch[F.npatch];
                P.comp = s == 0 ? comp : partner(axis, comp);
                P.axis = axis;
                P.plane = planes[s];
                P.lo1 = L[1];
                P.hi1 = L[2];
                P.lo2 = L[3];
                P.hi2 = L[4];
                P.off = F.samples;
                P.n = (L[2] >= L[1] && L[4] >= L[3]) ? (L[2] - L[1] + 1) * (L[4] - L[3] + 1) : 0;
                F.samples += P.n;
                F.face_patch[fc][slots[s]] = F.npatch++;
            }
        }
    }
    // the sampled nodes must lie inside the Alloc box
    for (int p = 0; p < F.npatch; ++p) {
        const FarPatch& P = F.patch[p];
        if (P.n == 0) continue;
        int lo[3], hi[3];
        lo[P.axis] = hi[P.axis] = P.plane;
        const int a1 = P.axis == 2 ? 1 : 2, a2 = P.axis == 0 ? 1 : 0;
        lo[a1] = P.lo1; hi[a1] = P.hi1; lo[a2] = P.lo2; hi[a2] = P.hi2;
        const int org[3] = {c->ox, c->oy, c->oz}, ext[3] = {c->nxa, c->nya, c->nza};
        for (int a = 0; a < 3; ++a)
            if (lo[a] < org[a] || hi[a] >= org[a] + ext[a])
                return set_error(c, SGPU_ERR_ARG, "far-field surface outside the Alloc box");
    }
    F.freq.assign(d->freq, d->freq + d->nfreq);
    F.cluz = d->cluz;
    F.zvac = d->zvac;
    for (int k = 0; k < 6; ++k) {
        if (d->cell[k] && d->cell_n[k] > 0) F.cell[k].assign(d->cell[k], d->cell[k] + d->cell_n[k]);
        F.cell_lo[k] = d->cell_lo[k];
    }
    for (int cc = 0; cc < 3; ++cc)
        for (int a = 0; a < 3; ++a) {
            if (d->phys[cc][a] && d->phys_n[cc][a] > 0) F.phys[cc][a].assign(d->phys[cc][a], d->phys[cc][a] + d->phys_n[cc][a]);
            F.phys_lo[cc][a] = d->phys_lo[cc][a];
        }
    // Weights of the sampled steps (all steps from 0, or 1, 1 + ndecim, ...) up to the time vector's
    // end (farfield.F90:1074-1100 and :1723-1728): auxExp_E starts at
    // dtDecim, auxExp_H at dtDecim * exp(-i 2 pi f dt / 2), both multiplied by
    // expIwdt = exp(-i 2 pi f dtDecim) after every sampled step; expIwdt is a
    // complex(4) exponential, the half-step factor a complex(8) one.
    const int steps = (int)c->h_tiempo.size();
    F.w_m = std::max(1, (steps + F.ndecim - 1) / F.ndecim + 1);
    std::vector<double2> wE((size_t)F.w_m * F.nf), wH((size_t)F.w_m * F.nf);
    for (int f = 0; f < F.nf; ++f) {
        const float fr = d->freq[f];
        const float yim = ((-(2.0f * kPiF)) * fr) * d->dtdecim;
        const std::complex<float> e4 = std::exp(std::complex<float>(-0.0f, yim));
        const std::complex<double> ex((double)e4.real(), (double)e4.imag());
        const float yh = (-(2.0f * kPiF)) * fr;
        const double x = c->dt * 0.5;
        const std::complex<double> eh = std::exp(std::complex<double>(-0.0 * x, (double)yh * x));
        const double dd = (double)d->dtdecim;
        std::complex<double> aE(dd, 0.0), aH(dd * eh.real(), dd * eh.imag());
        for (int m = 0; m < F.w_m; ++m) {
            wE[(size_t)m * F.nf + f] = make_double2(aE.real(), aE.imag());
            wH[(size_t)m * F.nf + f] = make_double2(aH.real(), aH.imag());
            aE = cmul_h(aE, ex);
            aH = cmul_h(aH, ex);
        }
    }
    const size_t wbytes = sizeof(double2) * wE.size(), abytes = sizeof(double2) * (size_t)F.nf * std::max(1, F.samples);
    cudaError_t e = cudaMalloc(&F.acc, abytes);
    if (e == cudaSuccess) e = cudaMalloc(&F.wE, wbytes);
    if (e == cudaSuccess) e = cudaMalloc(&F.wH, wbytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(F.acc, 0, abytes, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(F.wE, wE.data(), wbytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(F.wH, wH.data(), wbytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        cudaFree(F.acc);
        cudaFree(F.wE);
        cudaFree(F.wH);
        return set_error(c, SGPU_ERR_CUDA, std::string("far field: ") + cudaGetErrorString(e));
    }
    c->farfields.push_back(std::move(F));
    if (id) *id = (int)c->farfields.size() - 1;
    if (c->graph) {  // the captured steps do not launch the new far field
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    return SGPU_OK;
}

sgpu_status sgpu_farfield_shape(const sgpu_ctx* c, int id, int* nfreq, int* samples) {
    if (!c || id < 0 || id >= (int)c->farfields.size()) return SGPU_ERR_ARG;
    if (nfreq) *nfreq = c->farfields[id].nf;
    if (samples) *samples = c->farfields[id].samples;
    return SGPU_OK;
}

sgpu_status sgpu_read_farfield(sgpu_ctx* c, int id, int face, int slot, int* dims, double* out) {
    if (!c || id < 0 || id >= (int)c->farfields.size() || face < 0 || face > 5 || slot < 0 || slot > 5 || !dims)
        return set_error(c, SGPU_ERR_ARG, "no far-field array with that id, face and slot");
    const FarField& F = c->farfields[id];
    const int p = F.face_patch[face][slot];
    if (p < 0) {
        dims[0] = dims[1] = 0;
        return SGPU_OK;
    }
    const FarPatch& P = F.patch[p];
    dims[0] = P.n ? P.hi1 - P.lo1 + 1 : 0;
    dims[1] = P.n ? P.hi2 - P.lo2 + 1 : 0;
    if (!out || P.n == 0) return SGPU_OK;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    for (int f = 0; f < F.nf && e == cudaSuccess; ++f)
        e = cudaMemcpy(out + (size_t)f * P.n * 2, F.acc + (size_t)f * F.samples + P.off, sizeof(double2) * P.n,
                       cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return set_error(c, SGPU_ERR_CUDA, std::string("far field read: ") + cudaGetErrorString(e));
    return SGPU_OK;
}

sgpu_status sgpu_farfield_transform(sgpu_ctx* c, int id, const sgpu_farfield_angles* an, const float* incident,
                                    int n_incident, double* out, int max_rows, int* rows) {
    if (!c || !an || !rows || id < 0 || id >= (int)c->farfields.size())
        return set_error(c, SGPU_ERR_ARG, "bad far-field transform request");
    if (!(an->theta_step > 0.0f) || !(an->phi_step > 0.0f))
        return set_error(c, SGPU_ERR_ARG, "far-field angle steps must be positive");
    const FarField& F = c->farfields[id];
    // directions in the order of farfield.F90:2520-2525
    std::vector<Dir> dirs;
    float theta = an->theta_start - an->theta_step;
    while (theta < an->theta_stop) {
        theta = std::min(theta + an->theta_step, an->theta_stop);
        float phi = an->phi_start - an->phi_step;
        while (phi < an->phi_stop) {
            phi = std::min(phi + an->phi_step, an->phi_stop);
            Dir D;
            D.theta = theta;
            D.phi = phi;
            const float s_t = std::sin(theta), c_t = std::cos(theta), s_p = std::sin(phi), c_p = std::cos(phi);
            D.stsp = s_t * s_p;
            D.stcp = s_t * c_p;
            D.ct = c_t;
            D.cp = c_p;
            D.ctcp = c_t * c_p;
            D.ctsp = c_t * s_p;
            D.st = s_t;
            D.sp = s_p;
            dirs.push_back(D);
        }
    }
    const long long need = (long long)dirs.size() * F.nf;
    *rows = (int)need;
    if (!out) return SGPU_OK;
    if (max_rows < need) return set_error(c, SGPU_ERR_ARG, "far-field output too small");
    if (!incident || n_incident < 2) return set_error(c, SGPU_ERR_ARG, "the normalisation needs two samples or more");
    // DFT of the normalisation signal (farfield.F90:1021-1070): dtevol from
    // its first two times, the first sample skipped as the reference's read
    // loop skips it.
    std::vector<double2> dft(F.nf);
    {
        const float dtevol = incident[2] - incident[0];
        const double mc = -(double)(2.0f * kPiF);  // mcPI2 (fdetypes.F90:190)
        for (int f = 0; f < F.nf; ++f) {
            const std::complex<double> ex = std::exp(std::complex<double>(-0.0 * (double)F.freq[f] * dtevol,
                                                                          mc * (double)F.freq[f] * (double)dtevol));
            std::complex<double> aux((double)dtevol, 0.0), acc(0.0, 0.0);
            for (int m = 1; m < n_incident; ++m) {
                const double v = (double)incident[2 * m + 1];
                acc = std::complex<double>(acc.real() + v * aux.real(), acc.imag() + v * aux.imag());
                aux = cmul_h(aux, ex);
            }
            dft[f] = make_double2(acc.real(), acc.imag());
        }
    }
    // transform cells, face by face in the reference's loop ranges
    std::vector<TCell> cells;
    for (int fc = 0; fc < 6; ++fc) {
        if (!F.active[fc]) continue;
        const int axis = fc / 2;
        const float normal = fc % 2 == 0 ? -1.0f : 1.0f;
        const int* fp = F.face_patch[fc];
        const FarPatch &P1 = F.patch[fp[0]], &P2 = F.patch[fp[1]];
        // x faces: k in [K%com%Ez, K%fin%Ey], j in [J%com%Ez, J%fin%Ez];
        // y faces: k in [K%com%Ex, K%fin%Ex], i in [I%com%Ex, I%fin%Ez];
        // z faces: j in [J%com%Ey, J%fin%Ex], i in [I%com%Ey, I%fin%Ey]
        int o0, o1, u0, u1, plane;
        if (axis == 0) { o0 = P1.lo1; o1 = P2.hi1; u0 = P1.lo2; u1 = P1.hi2; plane = P1.plane; }
        else if (axis == 1) { o0 = P2.lo1; o1 = P2.hi1; u0 = P2.lo2; u1 = P1.hi2; plane = P2.plane; }
        else { o0 = P1.lo1; o1 = P2.hi1; u0 = P1.lo2; u1 = P1.hi2; plane = P1.plane; }
        // E1 / E2 of the face (as PhysCoor indices 0..2) and the cell sizes
        // of each current: (outer, inner) arrays from dxe..dzh
        const int e1 = kT[axis][0], e2 = kT[axis][1];
        // Ma: t1 present while outer <= hi1 of t1; Mb: t2 while inner <= hi2 of t2;
        // JB (partner of t2) while outer <= hi1 of t2; JA (partner of t1) while inner <= hi2 of t1
        for (int o = o0; o <= o1; ++o)
            for (int u = u0; u <= u1; ++u) {
                TCell t;
                int ijk[3];
                if (axis == 0) { ijk[0] = plane; ijk[1] = u; ijk[2] = o; }
                else if (axis == 1) { ijk[0] = u; ijk[1] = plane; ijk[2] = o; }
                else { ijk[0] = u; ijk[1] = o; ijk[2] = plane; }
                for (int a = 0; a < 3; ++a) {
                    t.pa[a] = at(F.phys[e1][a], F.phys_lo[e1][a], ijk[a]);
                    t.pb[a] = at(F.phys[e2][a], F.phys_lo[e2][a], ijk[a]);
                }
                t.col[0] = column(F, fp[0], o, u);
                t.col[1] = column(F, fp[1], o, u);
                t.col[2] = column(F, fp[2], o, u);
                t.col[3] = column(F, fp[3], o, u);
                t.col[4] = column(F, fp[4], o, u);
                t.col[5] = column(F, fp[5], o, u);
                const bool has_ma = o <= P1.hi1, has_mb = u <= P2.hi2, has_jb = o <= P2.hi1, has_ja = u <= P1.hi2;
                // cell sizes (e: dxe, dye, dze = 0..2; h: dxh, dyh, dzh = 3..5)
                auto cs = [&](int k, int idx) { return at(F.cell[k], F.cell_lo[k], idx); };
                float sgn[4];
                int s1[4], s2[4];  // cell-size arrays of the two factors
                int x1[4], x2[4];  // their indices
                if (axis == 0) {  // My = -Ez dyh dze, Mz = +Ey dye dzh, Jy = +Hz dye dzh, Jz = -Hy dyh dze
                    t.ax_ma = 1; t.ax_mb = 2;
                    sgn[0] = -1; s1[0] = 4; x1[0] = u; s2[0] = 2; x2[0] = o;
                    sgn[1] = +1; s1[1] = 1; x1[1] = u; s2[1] = 5; x2[1] = o;
                    sgn[2] = -1; s1[2] = 4; x1[2] = u; s2[2] = 2; x2[2] = o;
                    sgn[3] = +1; s1[3] = 1; x1[3] = u; s2[3] = 5; x2[3] = o;
                } else if (axis == 1) {  // Mx = +Ez dxh dze, Mz = -Ex dxe dzh, Jx = -Hz dxe dzh, Jz = +Hx dxh dze
                    t.ax_ma = 0; t.ax_mb = 2;
                    sgn[0] = +1; s1[0] = 3; x1[0] = u; s2[0] = 2; x2[0] = o;
                    sgn[1] = -1; s1[1] = 0; x1[1] = u; s2[1] = 5; x2[1] = o;
                    sgn[2] = +1; s1[2] = 3; x1[2] = u; s2[2] = 2; x2[2] = o;
                    sgn[3] = -1; s1[3] = 0; x1[3] = u; s2[3] = 5; x2[3] = o;
                } else {  // Mx = -Ey dxh dye, My = +Ex dxe dyh, Jx = +Hy dxe dyh, Jy = -Hx dxh dye
                    t.ax_ma = 0; t.ax_mb = 1;
                    sgn[0] = -1; s1[0] = 3; x1[0] = u; s2[0] = 1; x2[0] = o;
                    sgn[1] = +1; s1[1] = 0; x1[1] = u; s2[1] = 4; x2[1] = o;
                    sgn[2] = -1; s1[2] = 3; x1[2] = u; s2[2] = 1; x2[2] = o;
                    sgn[3] = +1; s1[3] = 0; x1[3] = u; s2[3] = 4; x2[3] = o;
                }
                const bool has[4] = {has_ma, has_mb, has_ja, has_jb};
                for (int k = 0; k < 4; ++k) {
                    t.fac[k][0] = cs(s1[k], x1[k]);
                    t.fac[k][1] = cs(s2[k], x2[k]);
                    t.fac[k][2] = has[k] ? sgn[k] * normal : 0.0f;
                }
                cells.push_back(t);
            }
    }
    if (cells.empty() || dirs.empty()) {
        std::fill(out, out + need * 9, 0.0);
        return SGPU_OK;
    }
    TCell* d_cells = nullptr;
    Currents* d_cur = nullptr;
    Dir* d_dirs = nullptr;
    float* d_freq = nullptr;
    double2* d_dft = nullptr;
    double* d_rows = nullptr;
    const int nc = (int)cells.size(), nd = (int)dirs.size();
    cudaError_t e = cudaMalloc(&d_cells, sizeof(TCell) * nc);
    if (e == cudaSuccess) e = cudaMalloc(&d_cur, sizeof(Currents) * (size_t)nc * F.nf);
    if (e == cudaSuccess) e = cudaMalloc(&d_dirs, sizeof(Dir) * nd);
    if (e == cudaSuccess) e = cudaMalloc(&d_freq, sizeof(float) * F.nf);
    if (e == cudaSuccess) e = cudaMalloc(&d_dft, sizeof(double2) * F.nf);
    if (e == cudaSuccess) e = cudaMalloc(&d_rows, sizeof(double) * 9 * (size_t)need);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_cells, cells.data(), sizeof(TCell) * nc, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_dirs, dirs.data(), sizeof(Dir) * nd, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_freq, F.freq.data(), sizeof(float) * F.nf, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_dft, dft.data(), sizeof(double2) * F.nf, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        const long long work = (long long)nc * F.nf;
        k_farfield_currents<<<(unsigned)((work + 255) / 256), 256, 0, c->stream>>>(d_cells, nc, F.acc, F.samples, F.nf, d_cur);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_farfield_dir<<<dim3(nd, F.nf), kDirThreads, 0, c->stream>>>(d_cells, nc, d_cur, d_dirs, nd, d_freq, d_dft, F.cluz,
                                                                     F.zvac, d_rows);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_rows, sizeof(double) * 9 * (size_t)need, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_cells);
    cudaFree(d_cur);
    cudaFree(d_dirs);
    cudaFree(d_freq);
    cudaFree(d_dft);
    cudaFree(d_rows);
    if (e != cudaSuccess) return set_error(c, SGPU_ERR_CUDA, std::string("far-field transform: ") + cudaGetErrorString(e));
    return SGPU_OK;
}

}  // extern "C"
