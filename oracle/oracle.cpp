// CPU oracle for the semba-fdtd Yee / CPML / ADE / TF-SF hot path.
// TEST INFRASTRUCTURE ONLY (see oracle.h): the checker for the CUDA path.
//
// Every routine below names the reference routine it restates.  Paths are
// relative to the reference project root.  Arithmetic follows the reference's
// kinds: RKIND (R) for fields, coefficients and metrics, real(8) for dt and
// the time vector, complex(8) for the ADE.  Mixed-kind Fortran expressions are
// written so that C++ promotes and rounds at the same operations.  Build with
// -ffp-contract=off and without -ffast-math (see Makefile).
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum { iEx = 0, iEy, iEz, iHx, iHy, iHz };
// Face indices of the reference (Down=1, Up=2, Left=3, Right=4, Back=5,
// Front=6 in fdetypes.F90:186), stored 0-based.
enum { Down = 0, Up, Left, Right, Back, Front };

// Default-real literals of semba_fdtd.F90:154-155 (no kind suffix, so they
// are rounded to single precision even when RKIND is 8).
const float kEps0 = 8.8541878176203898505365630317107502606083701665994498081024171524053950954599821142852891607182008932e-12f;
const float kMu0 = 1.2566370614359172953850573533118011536788677597500423283899778369231265625144835994512139301368468271e-6f;

// Priorities, fdetypes.F90:675-703 (set_priorities, default switches).
const int prior_BV = 10, prior_IB = 20, prior_FDB = 40, prior_PEC = 150;

struct Lim { int XI, XE, YI, YE, ZI, ZE; };

template <class T> struct A1 {
    int lo = 0, hi = -1;
    std::vector<T> v;
    void alloc(int l, int h, T init) { lo = l; hi = h; v.assign(h >= l ? h - l + 1 : 0, init); }
    T& operator()(int i) { return v[i - lo]; }
    const T& operator()(int i) const { return v[i - lo]; }
};

template <class T> struct A3 {
    Lim b{0, -1, 0, -1, 0, -1};
    long sx = 0, sy = 0;
    std::vector<T> v;
    void alloc(const Lim& l, T init) {
        b = l;
        sx = std::max(0, l.XE - l.XI + 1);
        sy = std::max(0, l.YE - l.YI + 1);
        long sz = std::max(0, l.ZE - l.ZI + 1);
        v.assign(sx * sy * sz, init);
    }
    T& operator()(int i, int j, int k) { return v[(i - b.XI) + sx * ((j - b.YI) + sy * (long)(k - b.ZI))]; }
    const T& operator()(int i, int j, int k) const { return v[(i - b.XI) + sx * ((j - b.YI) + sy * (long)(k - b.ZI))]; }
};

// complex(8) arithmetic as gfortran lowers it under its default Fortran
// complex rules (-fcx-fortran-rules): the plain product formula and Smith's
// (1962) range-reduced quotient.
struct C8 { double re, im; };
inline C8 cmul(C8 a, C8 b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C8 cdiv(C8 a, C8 b) {
    double ratio, div, tr, ti;
    if (std::fabs(b.re) < std::fabs(b.im)) {
        ratio = b.re / b.im;
        div = (b.re * ratio) + b.im;
        tr = (a.re * ratio) + a.im;
        ti = (a.im * ratio) - a.re;
    } else {
        ratio = b.im / b.re;
        div = (b.im * ratio) + b.re;
        tr = (a.im * ratio) + a.re;
        ti = a.im - (a.re * ratio);
    }
    return {tr / div, ti / div};
}

template <class R> struct Medium {
    R Epr = 1, Sigma = 0, Mur = 1, SigmaM = 0;
    int prio = prior_BV;
    bool pec = false, edisp = false, mdisp = false, yee_dummy = false;
    int region = -1;  // source region (dispersive data)
};

// One node of an electric dispersive medium (electricdispersive.F90:41-47).
template <class R> struct DNode {
    int i, j, k;
    R prev;
};

template <class R> struct EDispMedium {
    int indexmed;
    int np;
    std::vector<C8> beta, kappa, g3;
    std::vector<DNode<R>> nodes[3];
    std::vector<C8> J[3];  // Current(1:np) of node q at [q * np + p]
};

struct PWFaces {
    // Face limits per component, planewaves.F90:217-301 (TrFr, IzDe, AbAr).
    int trfr_i_tra[6], trfr_i_fro[6], trfr_j_com[6], trfr_j_fin[6], trfr_k_com[6], trfr_k_fin[6];
    int izde_j_izq[6], izde_j_der[6], izde_i_com[6], izde_i_fin[6], izde_k_com[6], izde_k_fin[6];
    int abar_k_aba[6], abar_k_arr[6], abar_i_com[6], abar_i_fin[6], abar_j_com[6], abar_j_fin[6];
    bool tr, fr, iz, de, ab, ar;
};

template <class R> struct PlaneWave {
    PWFaces f;
    R px, py, pz, fpw[6], d0;
    int numus;
    R deltaevol;
    std::vector<R> evol;
};

template <class R> struct NodalPoint {
    Lim p;
    R amp;
};
template <class R> struct NodalSet {
    std::vector<NodalPoint<R>> pts;
    std::vector<R> evol;
    R deltaevol;
    int numus;
};

template <class R> struct Sim {
    int nthreads = 1;
    // grid
    int nx, ny, nz;
    int L[3][2];        // PML layers [axis][side]
    R order[3][2], refl[3][2];
    R alphamax, alphaorder, kappamax;
    Lim SINPML[6], full[6], Alloc[6], Sweep[6], SINPMLSweep[6];
    A1<R> DX, DY, DZ, LineX, LineY, LineZ;
    double dt;
    std::vector<double> tiempo;
    R eps0, mu0, cluz, zvac;
    // media
    std::vector<Medium<R>> med;
    int NumMedia;
    A3<int16_t> mi[6];
    std::vector<R> G1, G2, GM1, GM2;
    // fields
    A3<R> F[6];
    // metrics
    A1<R> dxe, dye, dze, dxh, dyh, dzh, Idxe, Idye, Idze, Idxh, Idyh, Idzh;
    // CPML
    Lim PMLc[6][6];  // [field][region] as XI..ZE
    A1<R> ce_x, ce_y, ce_z, cm_x, cm_y, cm_z, Ice_x, Ice_y, Ice_z, Icm_x, Icm_y, Icm_z;
    A1<R> P_ce_x, P_ce_y, P_ce_z, P_be_x, P_be_y, P_be_z, P_cm_x, P_cm_y, P_cm_z, P_bm_x, P_bm_y, P_bm_z;
    // psi arrays: [region][which] where which is the reference's member order
    A3<R> psiLR[2][4], psiDU[2][4], psiBF[2][4];
    // border kinds per [axis][side] (sgg%Border, fdetypes.F90:468-497)
    bool isPML[3][2] = {}, isPEC[3][2] = {}, isPMC[3][2] = {}, isPer[3][2] = {}, isMur[3][2] = {};
    // Mur (bordersmur.F90:36-70): MURc limits per H component and region,
    // the Past_ layers of regLR (Hx, Hz), regDU (Hy, Hx), regBF (Hz, Hy) and
    // CAB1 per region and medium.  PastPast_ is read only by the second-order
    // branch, which stops with an error (bordersmur.F90:525), so it is not kept.
    bool anyMur = false;
    Lim MURc[6][6];
    A3<R> pastLR[2][2], pastDU[2][2], pastBF[2][2];
    std::vector<R> CAB1[6];
    // ADE: electric (Dutton) and magnetic (MDutton) media
    std::vector<EDispMedium<R>> dut, mdut;
    // plane waves; still_planewave_time is the global switch of
    // timestepping.F90:1219 and :1251-1267: true at the start of a run, lowered
    // by each AdvancePlaneWaveE/H and raised again by any face node whose
    // waveform is not over, and once it is down no plane-wave routine runs
    std::vector<PlaneWave<R>> pws;
    bool still_planewave_time = true;
    std::vector<R> phys[6][3];
    int phys_lo[6][3];
    // nodal
    NodalSet<R> nodal_soft[6], nodal_hard[6];
    std::vector<int> nodal_seq;  // unused
    // probes
    std::vector<int> probes;
    // frequency-domain volume probes (observation.F90:318-331, 1918-1922)
    struct FreqProbe {
        int mag;
        int i0, ni, j0, nj, k0, nk, tr[3];
        std::vector<float> freq;
        std::vector<std::complex<double>> V;  // [f][comp][k][j][i]
    };
    std::vector<FreqProbe> fprobes;
    // InitFarField / UpdateFarField state (farfield.F90:64-116): per face the
    // E arrays of its two tangential components and the H arrays of their
    // partners on two planes, each over its accumulation range (the
    // reference's arrays span the Alloc plane and stay zero outside it).
    struct FarArr {
        int comp = 0, plane = 0, lo1 = 0, hi1 = -1, lo2 = 0, hi2 = -1;
        std::vector<std::complex<double>> v;  // [f][outer][inner]
    };
    struct FarOrc {
        bool on[6] = {};
        int lim[6][2][5] = {};
        std::vector<R> freq;
        int ndecim = 1;
        R dtDecim = 0;
        std::vector<std::complex<double>> expIwdt, auxE, auxH;
        FarArr arr[6][6];  // [face][t1 E, t2 E, H1 plane 1, H1 plane 2, H2 plane 1, H2 plane 2]
    };
    std::vector<FarOrc> farfields;

    R physc(int field, int axis, int idx) const { return phys[field][axis][idx - phys_lo[field][axis]]; }
    double time(int n) {
        // crea_timevector, timestepping.F90:3230-3240: running FP64 sum.
        while ((int)tiempo.size() <= n) tiempo.push_back(tiempo.back() + dt);
        return tiempo[n];
    }
};

// ---------------------------------------------------------------------------
// read_limits_nogeom, preprocess_geom.F90:5266-5737, and the Alloc/Sweep set-up
// of NFDE2sgg, semba_fdtd.F90:1285-1300 (single layout).
template <class R> void setup_grid(Sim<R>& s, const orc_problem* p) {
    s.nx = p->nx; s.ny = p->ny; s.nz = p->nz;
    // face order back, front, left, right, down, up -> [axis][side]
    const int fa[6] = {0, 0, 1, 1, 2, 2}, fs[6] = {0, 1, 0, 1, 0, 1};
    for (int f = 0; f < 6; ++f) {
        // preprocess_geom.F90:5398-5600: the border flags; only CPML faces
        // carry layers, order and reflection (sgg%PML starts zeroed)
        const int kind = p->border[f] == 0 ? 9 : p->border[f];
        const int a = fa[f], sd = fs[f];
        s.isPML[a][sd] = kind == 9;
        s.isPEC[a][sd] = kind == 1;
        s.isPMC[a][sd] = kind == 2;
        s.isPer[a][sd] = kind == 4;
        s.isMur[a][sd] = kind == 7 || (kind == 9 && p->mur_after_pml);
        s.L[a][sd] = s.isPML[a][sd] ? p->pml_layers[f] : 0;
        float rf = s.isPML[a][sd] ? p->pml_refl[f] : 0.0f;
        if (rf >= 1.0f) rf = (float)0.99999;  // preprocess_geom.F90:5447
        s.refl[a][sd] = (R)rf;
        s.order[a][sd] = s.isPML[a][sd] ? (R)p->pml_order[f] : (R)0;
    }
    s.alphamax = (R)p->alphamax; s.alphaorder = (R)p->alphaorder; s.kappamax = (R)p->kappamax;
    int mx2 = s.nx, my2 = s.ny, mz2 = s.nz;
    for (int f = 0; f < 6; ++f) s.SINPML[f] = Lim{0, mx2, 0, my2, 0, mz2};
    s.SINPML[iEx].XE -= 1; s.SINPML[iEy].YE -= 1; s.SINPML[iEz].ZE -= 1;
    s.SINPML[iHx].YE -= 1; s.SINPML[iHx].ZE -= 1;
    s.SINPML[iHy].ZE -= 1; s.SINPML[iHy].XE -= 1;
    s.SINPML[iHz].XE -= 1; s.SINPML[iHz].YE -= 1;
    for (int f = 0; f < 6; ++f) {
        Lim& a = s.full[f];
        const Lim& q = s.SINPML[f];
        a = Lim{q.XI - s.L[0][0], q.XE + s.L[0][1], q.YI - s.L[1][0], q.YE + s.L[1][1], q.ZI - s.L[2][0], q.ZE + s.L[2][1]};
        s.Alloc[f] = Lim{a.XI - 1, a.XE + 1, a.YI - 1, a.YE + 1, a.ZI - 1, a.ZE + 1};
        s.Sweep[f] = a;
        s.SINPMLSweep[f] = Lim{std::max(q.XI, a.XI), std::min(q.XE, a.XE), std::max(q.YI, a.YI),
                               std::min(q.YE, a.YE), std::max(q.ZI, a.ZI), std::min(q.ZE, a.ZE)};
    }
    // cell sizes with the PML padding replicated (preprocess_geom.F90:5624-5667)
    auto pad = [&](A1<R>& D, const float* des, int n, int Llo, int Lhi) {
        D.alloc(-Llo - 2, n + Lhi + 2, (R)0);
        for (int i = 0; i < n; ++i) D(i) = (R)des[i];
        R delta = D(0);
        for (int i = -1; i >= -1 - Llo - 1; --i) D(i) = delta;
        delta = D(n - 1);
        for (int i = n; i <= n + Lhi + 2; ++i) D(i) = delta;
    };
    pad(s.DX, p->desx, s.nx, s.L[0][0], s.L[0][1]);
    pad(s.DY, p->desy, s.ny, s.L[1][0], s.L[1][1]);
    pad(s.DZ, p->desz, s.nz, s.L[2][0], s.L[2][1]);
    // grid lines (preprocess_geom.F90:5343-5400, 5670-5735)
    auto lines = [&](A1<R>& Ln, const float* des, int n, float origin, int Llo, int Lhi) {
        Ln.alloc(-Llo - 1, n + Lhi + 1, (R)0);
        Ln(0) = (R)origin + (R)0 * (R)des[1 < n ? 1 : 0];
        for (int i = 0; i < n; ++i) Ln(i + 1) = (R)des[i] + Ln(i);
        R delta = Ln(1) - Ln(0);
        for (int i = -1; i >= -1 - Llo; --i) Ln(i) = Ln(i + 1) - delta;
        delta = Ln(n) - Ln(n - 1);
        for (int i = n + 1; i <= n + Lhi + 1; ++i) Ln(i) = Ln(i - 1) + delta;
    };
    lines(s.LineX, p->desx, s.nx, p->originx, s.L[0][0], s.L[0][1]);
    lines(s.LineY, p->desy, s.ny, p->originy, s.L[1][0], s.L[1][1]);
    lines(s.LineZ, p->desz, s.nz, p->originz, s.L[2][0], s.L[2][1]);
}

// dt fix-up of NFDE2sgg, semba_fdtd.F90:1208-1257, and the constants of
// semba_fdtd.F90:154-156.
template <class R> void setup_dt(Sim<R>& s, const orc_problem* p) {
    s.eps0 = (R)kEps0;
    s.mu0 = (R)kMu0;
    s.cluz = (R)1.0 / std::sqrt(s.eps0 * s.mu0);
    s.zvac = std::sqrt(s.mu0 / s.eps0);
    R dxmin = *std::min_element(s.DX.v.begin(), s.DX.v.end());
    R dymin = *std::min_element(s.DY.v.begin(), s.DY.v.end());
    R dzmin = *std::min_element(s.DZ.v.begin(), s.DZ.v.end());
    R ix = (R)1.0 / dxmin, iy = (R)1.0 / dymin, iz = (R)1.0 / dzmin;
    // x**2.0 is folded to x*x by the compiler
    R dtlay = (R)1.0 / (s.cluz * std::sqrt(ix * ix + iy * iy + iz * iz));
    R dtv = dtlay;
    double sdt = p->dt;
    if (sdt < std::fabs((double)(std::numeric_limits<R>::min() * (R)2.0)))
        sdt = (double)(std::numeric_limits<R>::max() / (R)2.0);
    if (p->forcecfl) {
        sdt = (double)(dtv * (R)p->cfl);
    } else {
        const R heurCFL = (R)0.8f;
        if (sdt > (double)(dtv * heurCFL)) sdt = (double)(dtv * heurCFL);
    }
    s.dt = sdt;
    s.tiempo.assign(1, 0.0);
}

// CreateVolumeMM, healer.F90:66-243.
template <class R> void create_volume(Sim<R>& s, Lim point, int indicemedio) {
    const Lim BB{s.Alloc[iHx].XI, s.Alloc[iHx].XE, s.Alloc[iHy].YI, s.Alloc[iHy].YE, s.Alloc[iHz].ZI, s.Alloc[iHz].ZE};
    Lim pu{std::max(point.XI, std::min(BB.XI, BB.XE)), std::min(point.XE, std::max(BB.XI, BB.XE) - 1),
           std::max(point.YI, std::min(BB.YI, BB.YE)), std::min(point.YE, std::max(BB.YI, BB.YE) - 1),
           std::max(point.ZI, std::min(BB.ZI, BB.ZE)), std::min(point.ZE, std::max(BB.ZI, BB.ZE) - 1)};
    int p1XE = std::min(point.XE + 1, std::max(BB.XI, BB.XE));
    int p1YE = std::min(point.YE + 1, std::max(BB.YI, BB.YE));
    int p1ZE = std::min(point.ZE + 1, std::max(BB.ZI, BB.ZE));
    const int pr = s.med[indicemedio].prio;
    auto putE = [&](A3<int16_t>& m, int x0, int x1, int y0, int y1, int z0, int z1) {
        for (int k = z0; k <= z1; ++k)
            for (int j = y0; j <= y1; ++j)
                for (int i = x0; i <= x1; ++i)
                    if (pr > s.med[m(i, j, k)].prio) m(i, j, k) = (int16_t)indicemedio;
    };
    auto putH = [&](A3<int16_t>& m, int x0, int x1, int y0, int y1, int z0, int z1) {
        for (int k = z0; k <= z1; ++k)
            for (int j = y0; j <= y1; ++j)
                for (int i = x0; i <= x1; ++i)
                    if (pr >= s.med[m(i, j, k)].prio) m(i, j, k) = (int16_t)indicemedio;
    };
    putE(s.mi[iEx], pu.XI, pu.XE, pu.YI, p1YE, pu.ZI, p1ZE);
    putE(s.mi[iEy], pu.XI, p1XE, pu.YI, pu.YE, pu.ZI, p1ZE);
    putE(s.mi[iEz], pu.XI, p1XE, pu.YI, p1YE, pu.ZI, pu.ZE);
    putH(s.mi[iHx], pu.XI, p1XE, pu.YI, pu.YE, pu.ZI, pu.ZE);
    putH(s.mi[iHy], pu.XI, pu.XE, pu.YI, p1YE, pu.ZI, pu.ZE);
    putH(s.mi[iHz], pu.XI, pu.XE, pu.YI, pu.YE, pu.ZI, p1ZE);
}

// Index tables `in` and `on` of healer.F90:44-50, as [field][axis][side].
const int kIn[6][3][2] = {{{0, -1}, {1, -1}, {1, -1}}, {{1, -1}, {0, -1}, {1, -1}}, {{1, -1}, {1, -1}, {0, -1}},
                          {{1, -1}, {0, -1}, {0, -1}}, {{0, -1}, {1, -1}, {0, -1}}, {{0, -1}, {0, -1}, {1, -1}}};
const int kOn[6][3][2] = {{{0, -1}, {0, 0}, {0, 0}}, {{0, 0}, {0, -1}, {0, 0}}, {{0, 0}, {0, 0}, {0, -1}},
                          {{0, 0}, {0, -1}, {0, -1}}, {{0, -1}, {0, 0}, {0, -1}}, {{0, -1}, {0, -1}, {0, 0}}};

// CreatePMLmatrix, healer.F90:961-1420: the media touching the PML interface
// are extended outwards and renumbered as copies.
template <class R> void create_pml_matrix(Sim<R>& s) {
    const Lim BBox{s.Alloc[iHx].XI, s.Alloc[iHx].XE, s.Alloc[iHy].YI, s.Alloc[iHy].YE, s.Alloc[iHz].ZI, s.Alloc[iHz].ZE};
    int XIP[6], XEP[6], YIP[6], YEP[6], ZIP[6], ZEP[6];
    for (int f = 0; f < 6; ++f) {
        XIP[f] = std::max(BBox.XI, s.full[iHx].XI);
        XEP[f] = std::min(BBox.XE + kOn[f][0][1], s.full[iHx].XE);
        YIP[f] = std::max(BBox.YI, s.full[iHy].YI);
        YEP[f] = std::min(BBox.YE + kOn[f][1][1], s.full[iHy].YE);
        ZIP[f] = std::max(BBox.ZI, s.full[iHz].ZI);
        ZEP[f] = std::min(BBox.ZE + kOn[f][2][1], s.full[iHz].ZE);
    }
    const Lim BB{std::max(BBox.XI, s.SINPML[iHx].XI), std::min(BBox.XE, s.SINPML[iHx].XE),
                 std::max(BBox.YI, s.SINPML[iHy].YI), std::min(BBox.YE, s.SINPML[iHy].YE),
                 std::max(BBox.ZI, s.SINPML[iHz].ZI), std::min(BBox.ZE, s.SINPML[iHz].ZE)};
    for (int f = 0; f < 6; ++f) {
        A3<int16_t>& m = s.mi[f];
        auto neg = [](int16_t v) { return (int16_t)(-std::abs((int)v)); };
        for (int j = YIP[f]; j <= YEP[f]; ++j)
            for (int k = ZIP[f]; k <= ZEP[f]; ++k) {
                for (int i = XIP[f]; i <= BB.XI + kIn[f][0][1]; ++i) m(i, j, k) = neg(m(BB.XI + kIn[f][0][1] + 1, j, k));
                for (int i = BB.XE + kIn[f][0][0]; i <= XEP[f]; ++i) m(i, j, k) = neg(m(BB.XE + kIn[f][0][0] - 1, j, k));
            }
        for (int i = XIP[f]; i <= XEP[f]; ++i)
            for (int k = ZIP[f]; k <= ZEP[f]; ++k) {
                for (int j = YIP[f]; j <= BB.YI + kIn[f][1][1]; ++j) m(i, j, k) = neg(m(i, BB.YI + kIn[f][1][1] + 1, k));
                for (int j = BB.YE + kIn[f][1][0]; j <= YEP[f]; ++j) m(i, j, k) = neg(m(i, BB.YE + kIn[f][1][0] - 1, k));
            }
        for (int i = XIP[f]; i <= XEP[f]; ++i)
            for (int j = YIP[f]; j <= YEP[f]; ++j) {
                for (int k = ZIP[f]; k <= BB.ZI + kIn[f][2][1]; ++k) m(i, j, k) = neg(m(i, j, BB.ZI + kIn[f][2][1] + 1));
                for (int k = BB.ZE + kIn[f][2][0]; k <= ZEP[f]; ++k) m(i, j, k) = neg(m(i, j, BB.ZE + kIn[f][2][0] - 1));
            }
    }
    int nuevo = s.NumMedia;
    std::vector<int> tempo(s.NumMedia + 1, 0);
    for (int f = 0; f < 6; ++f)
        for (int k = ZIP[f]; k <= ZEP[f]; ++k)
            for (int j = YIP[f]; j <= YEP[f]; ++j)
                for (int i = XIP[f]; i <= XEP[f]; ++i) {
                    int m = s.mi[f](i, j, k);
                    if (m < 0 && tempo[-m] == 0) tempo[-m] = ++nuevo;
                }
    s.med.resize(nuevo + 1);
    for (int f = 0; f < 6; ++f)
        for (int k = ZIP[f]; k <= ZEP[f]; ++k)
            for (int j = YIP[f]; j <= YEP[f]; ++j)
                for (int i = XIP[f]; i <= XEP[f]; ++i) {
                    int m = s.mi[f](i, j, k);
                    if (m < 0) {
                        s.mi[f](i, j, k) = (int16_t)tempo[-m];
                        s.med[tempo[-m]] = s.med[-m];
                    }
                }
    s.NumMedia = nuevo;
    // PEC borders, healer.F90:1442-1617: medium 0 on the boundary plane of
    // the components tangential to it (E) and normal to it (H)
    for (int f = 0; f < 6; ++f) {
        const bool elec = f < 3;
        const int ca = f % 3;  // the component's own axis
        for (int a = 0; a < 3; ++a)
            for (int sd = 0; sd < 2; ++sd) {
                if (!s.isPEC[a][sd] || (elec ? a == ca : a != ca)) continue;
                int lo[3] = {XIP[f], YIP[f], ZIP[f]}, hi[3] = {XEP[f], YEP[f], ZEP[f]};
                lo[a] = hi[a] = sd == 0 ? lo[a] : hi[a];
                for (int k = lo[2]; k <= hi[2]; ++k)
                    for (int j = lo[1]; j <= hi[1]; ++j)
                        for (int i = lo[0]; i <= hi[0]; ++i) s.mi[f](i, j, k) = 0;
            }
    }
}

// Media table and matrices of read_geomData (preprocess_geom.F90:421-760,
// 1085-1110, asignadisper 5055-5248).
template <class R> void setup_media(Sim<R>& s, const orc_problem* p) {
    int contamedia = 1;
    s.med.assign(4, Medium<R>());
    // medium 1: vacuum (preprocess_geom.F90:456-462)
    s.med[1].Epr = (R)kEps0 / s.eps0;
    s.med[1].Mur = (R)kMu0 / s.mu0;
    s.med[1].prio = prior_BV;
    // medium 0: PEC (preprocess_geom.F90:463-469)
    s.med[0].pec = true;
    s.med[0].prio = prior_PEC;
    s.med[0].Epr = (R)kEps0 / s.eps0;
    s.med[0].Sigma = (R)1.0e29;
    s.med[0].Mur = (R)kMu0 / s.mu0;
    // conformal and split dummies (preprocess_geom.F90:599-603)
    contamedia = 3;
    s.med[2].yee_dummy = true;
    s.med[3].yee_dummy = true;
    for (int f = 0; f < 6; ++f) s.mi[f].alloc(s.Alloc[f], (int16_t)1);
    auto boxes = [&](const orc_region& r, int idx) {
        for (int b = 0; b < r.nboxes; ++b) {
            const int* q = r.boxes + 6 * b;
            create_volume(s, Lim{q[0], q[1], q[2], q[3], q[4], q[5]}, idx);
        }
    };
    for (int r = 0; r < p->nregions; ++r)
        if (p->regions[r].kind == 0) boxes(p->regions[r], 0);
    for (int r = 0; r < p->nregions; ++r) {
        const orc_region& g = p->regions[r];
        if (g.kind != 1) continue;
        Medium<R> m;
        m.prio = prior_IB;
        m.Epr = (R)g.eps / s.eps0;
        m.Sigma = (R)g.sigma;
        m.Mur = (R)g.mu / s.mu0;
        m.SigmaM = (R)g.sigmam;
        s.med.push_back(m);
        ++contamedia;
        boxes(g, contamedia);
    }
    for (int r = 0; r < p->nregions; ++r) {
        const orc_region& g = p->regions[r];
        if (g.kind != 2) continue;
        Medium<R> m;
        m.prio = prior_FDB;
        m.Epr = (R)g.eps / s.eps0;
        m.Sigma = (R)g.sigma;
        m.Mur = (R)g.mu / s.mu0;
        m.SigmaM = (R)g.sigmam;
        m.edisp = g.npoles != 0;
        m.mdisp = g.mpoles != 0;
        m.region = r;
        s.med.push_back(m);
        ++contamedia;
        boxes(g, contamedia);
    }
    s.NumMedia = contamedia;
    create_pml_matrix(s);
}

// calc_G1G2Gm1Gm2, calc_constants.F90:36-148 (branches reachable here).
template <class R> void calc_g(Sim<R>& s) {
    const int n = s.NumMedia;
    s.G1.assign(n + 1, 0); s.G2.assign(n + 1, 0); s.GM1.assign(n + 1, 0); s.GM2.assign(n + 1, 0);
    const double dt = s.dt;
    for (int r = 0; r <= n; ++r) {
        const Medium<R>& m = s.med[r];
        R Sigmam = m.SigmaM, Epsilon = s.eps0 * m.Epr, Mu = s.mu0 * m.Mur, Sigma = m.Sigma;
        auto magnetic = [&]() {
            double a = ((double)Sigmam * dt) / (double)((R)2.0 * Mu);
            s.GM1[r] = (R)((1.0 - a) / (1.0 + a));
            s.GM2[r] = (R)((dt / (double)Mu) / (1.0 + a));
            if (s.GM1[r] < (R)0.0) {
                s.GM1[r] = (R)std::exp(-(((double)Sigmam * dt) / (double)Mu));
                s.GM2[r] = ((R)1.0 - s.GM1[r]) / Sigmam;
            }
        };
        auto electric = [&]() {
            double a = ((double)Sigma * dt) / (double)((R)2.0 * Epsilon);
            s.G1[r] = (R)((1.0 - a) / (1.0 + a));
            s.G2[r] = (R)((dt / (double)Epsilon) / (1.0 + a));
            if (s.G1[r] < (R)0.0) {
                s.G1[r] = (R)std::exp(-(((double)Sigma * dt) / (double)Epsilon));
                s.G2[r] = ((R)1.0 - s.G1[r]) / Sigma;
            }
        };
        if (m.yee_dummy) {
            s.G1[r] = 1; s.G2[r] = 0; s.GM1[r] = 1; s.GM2[r] = 0;
        } else if (m.pec || r == 0) {
            s.G1[r] = 0; s.G2[r] = 0; s.GM1[r] = 0; s.GM2[r] = 0;
        } else if (m.edisp && !m.mdisp) {
            s.G1[r] = 0; s.G2[r] = 0;  // InitEDispersives sets them
            magnetic();
        } else if (m.mdisp && !m.edisp) {
            electric();
            s.GM1[r] = 0; s.GM2[r] = 0;  // InitMdispersives sets them
        } else {
            // also a medium with both kinds of poles: both Init routines
            // overwrite these values
            electric();
            magnetic();
        }
    }
}

// Metric arrays, timestepping.F90:314-370.
template <class R> void setup_metrics(Sim<R>& s) {
    const R bad = (R)-1.0e10;
    s.dxe.alloc(s.Alloc[iHx].XI, s.Alloc[iHx].XE, bad);
    s.dye.alloc(s.Alloc[iHy].YI, s.Alloc[iHy].YE, bad);
    s.dze.alloc(s.Alloc[iHz].ZI, s.Alloc[iHz].ZE, bad);
    s.dxh.alloc(s.Alloc[iEx].XI, s.Alloc[iEx].XE, bad);
    s.dyh.alloc(s.Alloc[iEy].YI, s.Alloc[iEy].YE, bad);
    s.dzh.alloc(s.Alloc[iEz].ZI, s.Alloc[iEz].ZE, bad);
    for (int i = s.dxe.lo; i <= s.dxe.hi; ++i) s.dxe(i) = s.DX(i);
    for (int j = s.dye.lo; j <= s.dye.hi; ++j) s.dye(j) = s.DY(j);
    for (int k = s.dze.lo; k <= s.dze.hi; ++k) s.dze(k) = s.DZ(k);
    for (int i = s.dxh.lo; i <= s.dxh.hi; ++i) s.dxh(i) = (s.DX(i) + s.DX(i - 1)) / (R)2.0;
    for (int j = s.dyh.lo; j <= s.dyh.hi; ++j) s.dyh(j) = (s.DY(j) + s.DY(j - 1)) / (R)2.0;
    for (int k = s.dzh.lo; k <= s.dzh.hi; ++k) s.dzh(k) = (s.DZ(k) + s.DZ(k - 1)) / (R)2.0;
    auto inv = [](A1<R>& o, const A1<R>& d) {
        o.alloc(d.lo, d.hi, 0);
        for (int i = d.lo; i <= d.hi; ++i) o(i) = (R)1.0 / d(i);
    };
    inv(s.Idxe, s.dxe); inv(s.Idye, s.dye); inv(s.Idze, s.dze);
    inv(s.Idxh, s.dxh); inv(s.Idyh, s.dyh); inv(s.Idzh, s.dzh);
}

// InitCPMLBorders (borderscpml.F90:90-473) and calc_cpmlconstants
// (borderscpml.F90:1465-1733).
template <class R> void setup_cpml(Sim<R>& s) {
    for (int f = 0; f < 6; ++f) {
        const Lim& w = s.Sweep[f];
        const Lim& q = s.SINPML[f];
        s.PMLc[f][Down] = Lim{w.XI, w.XE, w.YI, w.YE, w.ZI, std::min(q.ZI - 1, w.ZE)};
        s.PMLc[f][Up] = Lim{w.XI, w.XE, w.YI, w.YE, std::max(q.ZE + 1, w.ZI), w.ZE};
        s.PMLc[f][Left] = Lim{w.XI, w.XE, w.YI, std::min(q.YI - 1, w.YE), w.ZI, w.ZE};
        s.PMLc[f][Right] = Lim{w.XI, w.XE, std::max(q.YE + 1, w.YI), w.YE, w.ZI, w.ZE};
        s.PMLc[f][Back] = Lim{w.XI, std::min(q.XI - 1, w.XE), w.YI, w.YE, w.ZI, w.ZE};
        s.PMLc[f][Front] = Lim{std::max(q.XE + 1, w.XI), w.XE, w.YI, w.YE, w.ZI, w.ZE};
    }
    // depth arrays over the Alloc range of Hx/Hy/Hz
    auto depth = [&](A1<R>& ce, A1<R>& Ice, A1<R>& cm, A1<R>& Icm, int lo, int hi, int SI, int SE, int NL1, int NL2) {
        ce.alloc(lo, hi, 0); Ice.alloc(lo, hi, 0); cm.alloc(lo, hi, 0); Icm.alloc(lo, hi, 0);
        for (int i = lo; i <= hi; ++i) {
            if (i <= SI) {
                ce(i) = (R)1.0 * (R)(SI - i) / (R)NL1;
                Ice(i) = (R)1.0 * (R)(NL1 - (SI - i)) / (R)NL1;
            } else if (i >= SE) {
                ce(i) = (R)1.0 * (R)(i - SE) / (R)NL2;
                Ice(i) = (R)1.0 * (R)(NL2 - (i - SE)) / (R)NL2;
            } else {
                ce(i) = 0; Ice(i) = 0;
            }
        }
        for (int i = lo; i <= hi; ++i) {
            if (i <= SI - 1) {
                cm(i) = (R)1.0 * ((R)SI - ((R)i + (R)0.5)) / (R)NL1;
                Icm(i) = (R)1.0 * ((R)NL1 - ((R)SI - ((R)i + (R)0.5))) / (R)NL1;
            } else if (i >= SE) {
                cm(i) = (R)1.0 * ((R)(i - SE) + (R)0.5) / (R)NL2;
                Icm(i) = (R)1.0 * ((R)NL2 - ((R)(i - SE) + (R)0.5)) / (R)NL2;
            } else {
                cm(i) = 0; Icm(i) = 0;
            }
        }
    };
    // without a CPML face InitCPMLBorders returns before the depth vectors
    // and calc_cpmlconstants (borderscpml.F90:140-143)
    bool anyPML = false;
    for (int a = 0; a < 3; ++a) anyPML = anyPML || s.isPML[a][0] || s.isPML[a][1];
    if (anyPML) {
        depth(s.ce_x, s.Ice_x, s.cm_x, s.Icm_x, s.Alloc[iHx].XI, s.Alloc[iHx].XE, s.SINPML[iHx].XI, s.SINPML[iHx].XE, s.L[0][0], s.L[0][1]);
        depth(s.ce_y, s.Ice_y, s.cm_y, s.Icm_y, s.Alloc[iHy].YI, s.Alloc[iHy].YE, s.SINPML[iHy].YI, s.SINPML[iHy].YE, s.L[1][0], s.L[1][1]);
        depth(s.ce_z, s.Ice_z, s.cm_z, s.Icm_z, s.Alloc[iHz].ZI, s.Alloc[iHz].ZE, s.SINPML[iHz].ZI, s.SINPML[iHz].ZE, s.L[2][0], s.L[2][1]);
    }

    // calc_cpmlconstants
    R sig_max[3][2], aPar_max[3][2], kPar_max[3][2];
    const R dels[3][2] = {{s.dxe(s.Alloc[iEx].XI), s.dxe(s.Alloc[iEx].XE)},
                          {s.dye(s.Alloc[iEy].YI), s.dye(s.Alloc[iEy].YE)},
                          {s.dze(s.Alloc[iEz].ZI), s.dze(s.Alloc[iEz].ZE)}};
    for (int o = 0; o < 3; ++o)
        for (int q = 0; q < 2; ++q) {
            R del = dels[o][q];
            if (s.L[o][q] != 0) {
                if (s.L[o][q] == 10 || s.L[o][q] == 5) {
                    sig_max[o][q] = (R)0.8f * (s.order[o][q] + (R)1) / (std::sqrt(s.mu0 / s.eps0) * del);
                } else {
                    sig_max[o][q] = -((std::log(s.refl[o][q]) * (s.order[o][q] + (R)1)) /
                                      ((R)2 * std::sqrt(s.mu0 / s.eps0) * (R)s.L[o][q] * del));
                }
            } else {
                sig_max[o][q] = (R)1.0e29;
            }
        }
    for (int o = 0; o < 3; ++o)
        for (int q = 0; q < 2; ++q) {
            if (s.L[o][q] != 0) {
                aPar_max[o][q] = s.alphamax * sig_max[o][q];
                kPar_max[o][q] = s.kappamax;
            } else {
                aPar_max[o][q] = 0;
                kPar_max[o][q] = 1;
            }
        }
    auto init1 = [](A1<R>& a, int lo, int hi, R v) { a.alloc(lo, hi, v); };
    init1(s.P_ce_x, s.Alloc[iHx].XI, s.Alloc[iHx].XE, 0); init1(s.P_be_x, s.Alloc[iHx].XI, s.Alloc[iHx].XE, 1);
    init1(s.P_cm_x, s.Alloc[iHx].XI, s.Alloc[iHx].XE, 0); init1(s.P_bm_x, s.Alloc[iHx].XI, s.Alloc[iHx].XE, 1);
    init1(s.P_ce_y, s.Alloc[iHy].YI, s.Alloc[iHy].YE, 0); init1(s.P_be_y, s.Alloc[iHy].YI, s.Alloc[iHy].YE, 1);
    init1(s.P_cm_y, s.Alloc[iHy].YI, s.Alloc[iHy].YE, 0); init1(s.P_bm_y, s.Alloc[iHy].YI, s.Alloc[iHy].YE, 1);
    init1(s.P_ce_z, s.Alloc[iHz].ZI, s.Alloc[iHz].ZE, 0); init1(s.P_be_z, s.Alloc[iHz].ZI, s.Alloc[iHz].ZE, 1);
    init1(s.P_cm_z, s.Alloc[iHz].ZI, s.Alloc[iHz].ZE, 0); init1(s.P_bm_z, s.Alloc[iHz].ZI, s.Alloc[iHz].ZE, 1);
    const double dt = s.dt;
    // one electric-node coefficient set (borderscpml.F90:1546-1560 and twins)
    auto eco = [&](int o, int q, R ce, R Ice, R dh, R& Pbe, R& Pce, R& Id) {
        R sigmae, kpare;
        if (s.order[o][q] == (R)0) {
            sigmae = sig_max[o][q];
            kpare = (R)1.0 + (kPar_max[o][q] - (R)1);
        } else {
            sigmae = sig_max[o][q] * std::pow(ce, s.order[o][q]);
            kpare = (R)1.0 + (kPar_max[o][q] - (R)1) * std::pow(ce, s.order[o][q]);
        }
        R apare = aPar_max[o][q] * std::pow(Ice, s.alphaorder);
        Pbe = (R)std::exp(-((double)(sigmae / kpare + apare) * dt) / (double)s.eps0);
        Pce = (sigmae * (Pbe - (R)1.0) / (sigmae + kpare * apare) / kpare) / dh;
        Id = (R)1.0 / (kpare * dh);
    };
    // faces without CPML keep order 0 and kPar_max 1, so the inverse steps of
    // their outer nodes come out unchanged (their P_b/P_c are never read)
    if (anyPML) {
    for (int i = s.Alloc[iEx].XI; i <= s.Alloc[iEx].XE; ++i) {
        if (i <= s.SINPML[iHx].XI - 1) eco(0, 0, s.ce_x(i), s.Ice_x(i), s.dxh(i), s.P_be_x(i), s.P_ce_x(i), s.Idxh(i));
        else if (i >= s.SINPML[iHx].XE + 1) eco(0, 1, s.ce_x(i), s.Ice_x(i), s.dxh(i), s.P_be_x(i), s.P_ce_x(i), s.Idxh(i));
    }
    for (int j = s.Alloc[iEy].YI; j <= s.Alloc[iEy].YE; ++j) {
        if (j <= s.SINPML[iHy].YI - 1) eco(1, 0, s.ce_y(j), s.Ice_y(j), s.dyh(j), s.P_be_y(j), s.P_ce_y(j), s.Idyh(j));
        else if (j >= s.SINPML[iHy].YE + 1) eco(1, 1, s.ce_y(j), s.Ice_y(j), s.dyh(j), s.P_be_y(j), s.P_ce_y(j), s.Idyh(j));
    }
    for (int k = s.Alloc[iEz].ZI; k <= s.Alloc[iEz].ZE; ++k) {
        if (k <= s.SINPML[iHz].ZI - 1) eco(2, 0, s.ce_z(k), s.Ice_z(k), s.dzh(k), s.P_be_z(k), s.P_ce_z(k), s.Idzh(k));
        else if (k >= s.SINPML[iHz].ZE + 1) eco(2, 1, s.ce_z(k), s.Ice_z(k), s.dzh(k), s.P_be_z(k), s.P_ce_z(k), s.Idzh(k));
    }
    // magnetic nodes: note the front/right/up test is >= SINPML%XE here
    for (int i = s.Alloc[iHx].XI; i <= s.Alloc[iHx].XE; ++i) {
        if (i <= s.SINPML[iHx].XI - 1) eco(0, 0, s.cm_x(i), s.Icm_x(i), s.dxe(i), s.P_bm_x(i), s.P_cm_x(i), s.Idxe(i));
        else if (i >= s.SINPML[iHx].XE) eco(0, 1, s.cm_x(i), s.Icm_x(i), s.dxe(i), s.P_bm_x(i), s.P_cm_x(i), s.Idxe(i));
    }
    for (int j = s.Alloc[iHy].YI; j <= s.Alloc[iHy].YE; ++j) {
        if (j <= s.SINPML[iHy].YI - 1) eco(1, 0, s.cm_y(j), s.Icm_y(j), s.dye(j), s.P_bm_y(j), s.P_cm_y(j), s.Idye(j));
        else if (j >= s.SINPML[iHy].YE) eco(1, 1, s.cm_y(j), s.Icm_y(j), s.dye(j), s.P_bm_y(j), s.P_cm_y(j), s.Idye(j));
    }
    for (int k = s.Alloc[iHz].ZI; k <= s.Alloc[iHz].ZE; ++k) {
        if (k <= s.SINPML[iHz].ZI - 1) eco(2, 0, s.cm_z(k), s.Icm_z(k), s.dze(k), s.P_bm_z(k), s.P_cm_z(k), s.Idze(k));
        else if (k >= s.SINPML[iHz].ZE) eco(2, 1, s.cm_z(k), s.Icm_z(k), s.dze(k), s.P_bm_z(k), s.P_cm_z(k), s.Idze(k));
    }
    }  // anyPML
    // absent faces are faked empty (borderscpml.F90:307-314); every face is a
    // PML face here only when its layer count is non-zero.
    const int face_axis_side[6][2] = {{2, 0}, {2, 1}, {1, 0}, {1, 1}, {0, 0}, {0, 1}};
    for (int r = 0; r < 6; ++r)
        if (s.L[face_axis_side[r][0]][face_axis_side[r][1]] == 0)
            for (int f = 0; f < 6; ++f) s.PMLc[f][r].ZI = s.PMLc[f][r].ZE + 100;
    auto box = [&](int f, int r) { return s.PMLc[f][r]; };
    for (int r = 0; r < 2; ++r) {
        int reg = Left + r;
        s.psiLR[r][0].alloc(box(iEx, reg), 0); s.psiLR[r][1].alloc(box(iEz, reg), 0);
        s.psiLR[r][2].alloc(box(iHx, reg), 0); s.psiLR[r][3].alloc(box(iHz, reg), 0);
        reg = Down + r;
        s.psiDU[r][0].alloc(box(iEy, reg), 0); s.psiDU[r][1].alloc(box(iEx, reg), 0);
        s.psiDU[r][2].alloc(box(iHy, reg), 0); s.psiDU[r][3].alloc(box(iHx, reg), 0);
        reg = Back + r;
        s.psiBF[r][0].alloc(box(iEz, reg), 0); s.psiBF[r][1].alloc(box(iEy, reg), 0);
        s.psiBF[r][2].alloc(box(iHz, reg), 0); s.psiBF[r][3].alloc(box(iHy, reg), 0);
    }
}

// Region (Down..Front) -> [axis][side].
const int kRegAxis[6] = {2, 2, 1, 1, 0, 0}, kRegSide[6] = {0, 1, 0, 1, 0, 1};

// InitMURBorders and calc_murconstants, bordersmur.F90:79-363 (fresh start:
// the Past_ layers start at zero).
template <class R> void setup_mur(Sim<R>& s) {
    s.anyMur = false;
    for (int a = 0; a < 3; ++a) s.anyMur = s.anyMur || s.isMur[a][0] || s.isMur[a][1];
    if (!s.anyMur) return;
    // two planes per region: the outer H layer and the first swept one
    for (int f = iHx; f <= iHz; ++f) {
        const Lim& w = s.Sweep[f];
        s.MURc[f][Down] = Lim{w.XI, w.XE, w.YI, w.YE, w.ZI - 1, w.ZI};
        s.MURc[f][Up] = Lim{w.XI, w.XE, w.YI, w.YE, w.ZE, w.ZE + 1};
        s.MURc[f][Left] = Lim{w.XI, w.XE, w.YI - 1, w.YI, w.ZI, w.ZE};
        s.MURc[f][Right] = Lim{w.XI, w.XE, w.YE, w.YE + 1, w.ZI, w.ZE};
        s.MURc[f][Back] = Lim{w.XI - 1, w.XI, w.YI, w.YE, w.ZI, w.ZE};
        s.MURc[f][Front] = Lim{w.XE, w.XE + 1, w.YI, w.YE, w.ZI, w.ZE};
        for (int r = 0; r < 6; ++r)  // bordersmur.F90:163-170
            if (!s.isMur[kRegAxis[r]][kRegSide[r]]) s.MURc[f][r].ZI = s.MURc[f][r].ZE + 100;
    }
    for (int r = 0; r < 2; ++r) {
        s.pastLR[r][0].alloc(s.MURc[iHx][Left + r], (R)0); s.pastLR[r][1].alloc(s.MURc[iHz][Left + r], (R)0);
        s.pastDU[r][0].alloc(s.MURc[iHy][Down + r], (R)0); s.pastDU[r][1].alloc(s.MURc[iHx][Down + r], (R)0);
        s.pastBF[r][0].alloc(s.MURc[iHz][Back + r], (R)0); s.pastBF[r][1].alloc(s.MURc[iHy][Back + r], (R)0);
    }
    // cnum = (1/Id(outer node)) / (dt * cluz / sqrt(Epr*Mur)): RKIND operands,
    // the real(8) dt promotes the denominator, the quotient is stored in RKIND
    const R idh[6] = {s.Idzh(s.Alloc[iEz].ZI), s.Idzh(s.Alloc[iEz].ZE), s.Idyh(s.Alloc[iEy].YI),
                      s.Idyh(s.Alloc[iEy].YE), s.Idxh(s.Alloc[iEx].XI), s.Idxh(s.Alloc[iEx].XE)};
    for (int r = 0; r < 6; ++r) {
        s.CAB1[r].assign(s.NumMedia + 1, (R)0);
        for (int m = 0; m <= s.NumMedia; ++m) {
            const R den = std::sqrt(s.med[m].Epr * s.med[m].Mur);
            const R cnum = (R)((double)((R)1.0 / idh[r]) / ((s.dt * (double)s.cluz) / (double)den));
            s.CAB1[r][m] = ((R)1.0 - cnum) / ((R)1.0 + cnum);
        }
    }
}

// InitEDispersives (electricdispersive.F90:77-298) and, with mag,
// InitMdispersives (magneticdispersive.F90:79-289): the same construction
// with the magnetic poles, mu11 and sigmam11 of the medium, writing GM1/GM2
// and listing the swept H nodes.
template <class R> void setup_disp(Sim<R>& s, const orc_problem* p, bool mag) {
    std::vector<EDispMedium<R>>& list = mag ? s.mdut : s.dut;
    list.clear();
    const double dt = s.dt;
    for (int jmed = 1; jmed <= s.NumMedia; ++jmed) {
        if (!(mag ? s.med[jmed].mdisp : s.med[jmed].edisp)) continue;
        const orc_region& g = p->regions[s.med[jmed].region];
        const int np = mag ? g.mpoles : g.npoles;
        const float* res = mag ? g.mresidues : g.residues;
        const float* bp = mag ? g.mbpoles : g.bpoles;
        EDispMedium<R> d;
        d.indexmed = jmed;
        d.np = np;
        for (int q = 0; q < np; ++q) {
            // complex64 inputs promoted to complex(8); a11 = -b11
            // (preprocess_geom.F90:5196-5199, 5223-5226 for the magnetic ones)
            C8 C{(double)res[2 * q], (double)res[2 * q + 1]};
            C8 a{(double)(-bp[2 * q]), (double)(-bp[2 * q + 1])};
            C8 adt2{(a.re * dt) / 2.0, (a.im * dt) / 2.0};
            C8 num{1.0 + adt2.re, adt2.im};
            C8 den{1.0 - adt2.re, -adt2.im};
            d.kappa.push_back(cdiv(num, den));
            d.beta.push_back(cdiv(C8{C.re * dt, C.im * dt}, den));
        }
        list.push_back(d);
    }
    std::vector<R>& C1 = mag ? s.GM1 : s.G1;
    std::vector<R>& C2 = mag ? s.GM2 : s.G2;
    for (EDispMedium<R>& d : list) {
        const orc_region& g = p->regions[s.med[d.indexmed].region];
        R tempo = 0;
        for (int q = 0; q < d.np; ++q) tempo = (R)((double)tempo + d.beta[q].re);
        // eps11 / sigma11 (electric), mu11 / sigmam11 (magnetic)
        R v11 = mag ? (R)g.mu : (R)g.eps, sig11 = mag ? (R)g.sigmam : (R)g.sigma;
        double den = (double)((R)2.0 * v11 + tempo) + (double)sig11 * dt;
        C1[d.indexmed] = (R)(((double)((R)2.0 * v11 + tempo) - (double)sig11 * dt) / den);
        C2[d.indexmed] = (R)(((double)(R)2.0 * dt) / den);
        for (int q = 0; q < d.np; ++q) {
            double gh = (double)(C2[d.indexmed] / (R)2.0);
            d.g3.push_back(C8{gh * (1.0 + d.kappa[q].re), gh * d.kappa[q].im});
        }
    }
    const int c0 = mag ? 3 : 0;
    for (EDispMedium<R>& d : list) {
        for (int c = 0; c < 3; ++c) {
            const Lim& w = s.Sweep[c0 + c];
            for (int k = w.ZI; k <= w.ZE; ++k)
                for (int j = w.YI; j <= w.YE; ++j)
                    for (int i = w.XI; i <= w.XE; ++i)
                        if (s.mi[c0 + c](i, j, k) == d.indexmed) {
                            DNode<R> n;
                            n.i = i; n.j = j; n.k = k;
                            n.prev = 0;
                            d.nodes[c].push_back(n);
                        }
            d.J[c].assign(d.nodes[c].size() * (size_t)d.np, C8{0.0, 0.0});
        }
    }
}

// InitPlaneWave (planewaves.F90:72-770) with the plane-wave pre-processing of
// read_geomData (preprocess_geom.F90:290-413) and calc_planewaveconstants
// (planewaves.F90:1494-1510).
template <class R> void setup_planewave(Sim<R>& s, const orc_problem* p) {
    // physical coordinates of each component (planewaves.F90:94-159)
    const bool half[6][3] = {{true, false, false}, {false, true, false}, {false, false, true},
                             {false, true, true},  {true, false, true}, {true, true, false}};
    const A1<R>* line[3] = {&s.LineX, &s.LineY, &s.LineZ};
    for (int f = 0; f < 6; ++f) {
        const int lo[3] = {s.Sweep[f].XI - 1, s.Sweep[f].YI - 1, s.Sweep[f].ZI - 1};
        const int hi[3] = {s.Sweep[f].XE + 1, s.Sweep[f].YE + 1, s.Sweep[f].ZE + 1};
        for (int a = 0; a < 3; ++a) {
            s.phys_lo[f][a] = lo[a];
            s.phys[f][a].assign(hi[a] - lo[a] + 1, (R)0);
            int top = half[f][a] ? hi[a] - 1 : hi[a];
            for (int i = lo[a]; i <= top; ++i)
                s.phys[f][a][i - lo[a]] = half[f][a] ? ((*line[a])(i) + (*line[a])(i + 1)) * (R)0.5 : (*line[a])(i);
        }
    }
    for (int w = 0; w < p->npw; ++w) {
        const orc_planewave& in = p->pw[w];
        PlaneWave<R> pw;
        Lim pu{std::min(in.x1, in.x2), std::max(in.x1, in.x2), std::min(in.y1, in.y2), std::max(in.y1, in.y2),
               std::min(in.z1, in.z2), std::max(in.z1, in.z2)};
        if (pu.XI == s.SINPML[iHx].XI) pu.XI = s.SINPML[iHx].XI - 5;
        if (pu.XE == s.SINPML[iHx].XE) pu.XE = s.SINPML[iHx].XE + 5;
        if (pu.YI == s.SINPML[iHy].YI) pu.YI = s.SINPML[iHy].YI - 5;
        if (pu.YE == s.SINPML[iHy].YE) pu.YE = s.SINPML[iHy].YE + 5;
        if (pu.ZI == s.SINPML[iHz].ZI) pu.ZI = s.SINPML[iHz].ZI - 5;
        if (pu.ZE == s.SINPML[iHz].ZE) pu.ZE = s.SINPML[iHz].ZE + 5;
        // preprocess_geom.F90:386-391 (default-kind trig, amplitude 1)
        R amplitud = 1;
        R ez = amplitud * std::cos((R)in.alpha);
        R ey = amplitud * std::sin((R)in.alpha) * std::sin((R)in.beta);
        R ex = amplitud * std::sin((R)in.alpha) * std::cos((R)in.beta);
        R pz = std::cos((R)in.theta);
        R py = std::sin((R)in.theta) * std::sin((R)in.phi);
        R px = std::sin((R)in.theta) * std::cos((R)in.phi);
        const int esqx1 = pu.XI, esqx2 = pu.XE, esqy1 = pu.YI, esqy2 = pu.YE, esqz1 = pu.ZI, esqz2 = pu.ZE;
        PWFaces& F = pw.f;
        const Lim* SS = s.SINPMLSweep;
        F.tr = (esqx1 >= SS[iHx].XI) && (esqx1 <= SS[iHx].XE);
        F.fr = (esqx2 <= SS[iHx].XE) && (esqx2 >= SS[iHx].XI);
        F.iz = (esqy1 >= SS[iHy].YI) && (esqy1 <= SS[iHy].YE);
        F.de = (esqy2 <= SS[iHy].YE) && (esqy2 >= SS[iHy].YI);
        F.ab = (esqz1 >= SS[iHz].ZI) && (esqz1 <= SS[iHz].ZE);
        F.ar = (esqz2 <= SS[iHz].ZE) && (esqz2 >= SS[iHz].ZI);
        // planewaves.F90:217-301
        for (int c : {iEz, iEy}) {
            F.trfr_i_tra[c] = std::max(SS[c].XI, esqx1);
            F.trfr_i_fro[c] = std::min(SS[c].XE, esqx2);
        }
        F.trfr_j_com[iEz] = std::max(SS[iEz].YI, esqy1); F.trfr_j_fin[iEz] = std::min(SS[iEz].YE, esqy2);
        F.trfr_k_com[iEz] = std::max(SS[iEz].ZI, esqz1); F.trfr_k_fin[iEz] = std::min(SS[iEz].ZE, esqz2 - 1);
        F.trfr_j_com[iEy] = std::max(SS[iEy].YI, esqy1); F.trfr_j_fin[iEy] = std::min(SS[iEy].YE, esqy2 - 1);
        F.trfr_k_com[iEy] = std::max(SS[iEy].ZI, esqz1); F.trfr_k_fin[iEy] = std::min(SS[iEy].ZE, esqz2);
        F.trfr_i_tra[iHy] = F.trfr_i_tra[iEz] - 1; F.trfr_i_fro[iHy] = F.trfr_i_fro[iEz];
        F.trfr_j_com[iHy] = F.trfr_j_com[iEz]; F.trfr_j_fin[iHy] = F.trfr_j_fin[iEz];
        F.trfr_k_com[iHy] = F.trfr_k_com[iEz]; F.trfr_k_fin[iHy] = F.trfr_k_fin[iEz];
        F.trfr_i_tra[iHz] = F.trfr_i_tra[iEy] - 1; F.trfr_i_fro[iHz] = F.trfr_i_fro[iEy];
        F.trfr_j_com[iHz] = F.trfr_j_com[iEy]; F.trfr_j_fin[iHz] = F.trfr_j_fin[iEy];
        F.trfr_k_com[iHz] = F.trfr_k_com[iEy]; F.trfr_k_fin[iHz] = F.trfr_k_fin[iEy];

        F.izde_j_izq[iEx] = std::max(SS[iEx].YI, esqy1); F.izde_j_der[iEx] = std::min(SS[iEx].YE, esqy2);
        F.izde_i_com[iEx] = std::max(SS[iEx].XI, esqx1); F.izde_i_fin[iEx] = std::min(SS[iEx].XE, esqx2 - 1);
        F.izde_k_com[iEx] = std::max(SS[iEx].ZI, esqz1); F.izde_k_fin[iEx] = std::min(SS[iEx].ZE, esqz2);
        F.izde_j_izq[iEz] = std::max(SS[iEz].YI, esqy1); F.izde_j_der[iEz] = std::min(SS[iEz].YE, esqy2);
        F.izde_i_com[iEz] = std::max(SS[iEz].XI, esqx1); F.izde_i_fin[iEz] = std::min(SS[iEz].XE, esqx2);
        F.izde_k_com[iEz] = std::max(SS[iEz].ZI, esqz1); F.izde_k_fin[iEz] = std::min(SS[iEz].ZE, esqz2 - 1);
        F.izde_j_izq[iHz] = F.izde_j_izq[iEx] - 1; F.izde_j_der[iHz] = F.izde_j_der[iEx];
        F.izde_i_com[iHz] = F.izde_i_com[iEx]; F.izde_i_fin[iHz] = F.izde_i_fin[iEx];
        F.izde_k_com[iHz] = F.izde_k_com[iEx]; F.izde_k_fin[iHz] = F.izde_k_fin[iEx];
        F.izde_j_izq[iHx] = F.izde_j_izq[iEz] - 1; F.izde_j_der[iHx] = F.izde_j_der[iEz];
        F.izde_i_com[iHx] = F.izde_i_com[iEz]; F.izde_i_fin[iHx] = F.izde_i_fin[iEz];
        F.izde_k_com[iHx] = F.izde_k_com[iEz]; F.izde_k_fin[iHx] = F.izde_k_fin[iEz];

        F.abar_k_aba[iEy] = std::max(SS[iEy].ZI, esqz1); F.abar_k_arr[iEy] = std::min(SS[iEy].ZE, esqz2);
        F.abar_i_com[iEy] = std::max(SS[iEy].XI, esqx1); F.abar_i_fin[iEy] = std::min(SS[iEy].XE, esqx2);
        F.abar_j_com[iEy] = std::max(SS[iEy].YI, esqy1); F.abar_j_fin[iEy] = std::min(SS[iEy].YE, esqy2 - 1);
        F.abar_k_aba[iEx] = std::max(SS[iEx].ZI, esqz1); F.abar_k_arr[iEx] = std::min(SS[iEx].ZE, esqz2);
        F.abar_i_com[iEx] = std::max(SS[iEx].XI, esqx1); F.abar_i_fin[iEx] = std::min(SS[iEx].XE, esqx2 - 1);
        F.abar_j_com[iEx] = std::max(SS[iEx].YI, esqy1); F.abar_j_fin[iEx] = std::min(SS[iEx].YE, esqy2);
        F.abar_k_aba[iHx] = F.abar_k_aba[iEy] - 1; F.abar_k_arr[iHx] = F.abar_k_arr[iEy];
        F.abar_i_com[iHx] = F.abar_i_com[iEy]; F.abar_i_fin[iHx] = F.abar_i_fin[iEy];
        F.abar_j_com[iHx] = F.abar_j_com[iEy]; F.abar_j_fin[iHx] = F.abar_j_fin[iEy];
        F.abar_k_aba[iHy] = F.abar_k_aba[iEx] - 1; F.abar_k_arr[iHy] = F.abar_k_arr[iEx];
        F.abar_i_com[iHy] = F.abar_i_com[iEx]; F.abar_i_fin[iHy] = F.abar_i_fin[iEx];
        F.abar_j_com[iHy] = F.abar_j_com[iEx]; F.abar_j_fin[iHy] = F.abar_j_fin[iEx];

        pw.numus = in.nsamples - 1;
        pw.evol.assign(in.samples, in.samples + in.nsamples);
        pw.deltaevol = (R)in.dsamples;
        // planewaves.F90:330-342: normalised direction
        R modulus = std::sqrt(px * px + py * py + pz * pz);
        pw.px = px / modulus; pw.py = py / modulus; pw.pz = pz / modulus;
        pw.fpw[0] = ex; pw.fpw[1] = ey; pw.fpw[2] = ez;
        // null-phase corner, planewaves.F90:372-411 (INCERT = 0)
        auto LX = [&](int i) { return s.LineX(i); };
        auto LY = [&](int j) { return s.LineY(j); };
        auto LZ = [&](int k) { return s.LineZ(k); };
        int xlo = std::max(esqx1 - 1, s.SINPML[iHx].XI), xhi = std::min(esqx2 + 1, s.SINPML[iHx].XE);
        int ylo = std::max(esqy1 - 1, s.SINPML[iHy].YI), yhi = std::min(esqy2 + 1, s.SINPML[iHy].YE);
        int zlo = std::max(esqz1 - 1, s.SINPML[iHz].ZI), zhi = std::min(esqz2 + 1, s.SINPML[iHz].ZE);
        R X0 = pw.px >= 0 ? LX(xlo) : LX(xhi);
        R Y0 = pw.py >= 0 ? LY(ylo) : LY(yhi);
        R Z0 = pw.pz >= 0 ? LZ(zlo) : LZ(zhi);
        R dx = LX(xlo) - LX(xhi), dy = LY(ylo) - LY(yhi), dz = LZ(zlo) - LZ(zhi);
        R diag = std::sqrt(dx * dx + dy * dy + dz * dz);
        R incert = 0;
        pw.d0 = ((X0 * pw.px + Y0 * pw.py + Z0 * pw.pz)) - incert * diag;
        // calc_planewaveconstants
        pw.fpw[3] = (pw.py * pw.fpw[2] - pw.pz * pw.fpw[1]) / s.zvac;
        pw.fpw[4] = (pw.pz * pw.fpw[0] - pw.px * pw.fpw[2]) / s.zvac;
        pw.fpw[5] = (pw.px * pw.fpw[1] - pw.py * pw.fpw[0]) / s.zvac;
        s.pws.push_back(pw);
    }
}

// Incid + evolucion, planewaves.F90:778-853 (one mode, not from observation).
// evolucion raises still_planewave_time whenever the node's retarded time
// still lies inside the waveform table (nprev + 1 <= numus, :830-832).
template <class R> inline R incid(Sim<R>& s, const PlaneWave<R>& pw, int nfield, R time, int i, int j, int k) {
    R xf = s.physc(nfield, 0, i), yf = s.physc(nfield, 1, j), zf = s.physc(nfield, 2, k);
    R ehi = 0;
    R d = (xf * pw.px + yf * pw.py + zf * pw.pz) - pw.d0;
    R ev = 0;
    R arg = time - d / s.cluz;
    long long nprev = (long long)(arg / pw.deltaevol);
    if (nprev + 1 <= pw.numus) {
        s.still_planewave_time = true;
        if (nprev > 0) {
            ev = (pw.evol[nprev + 1] - pw.evol[nprev]) / pw.deltaevol * ((time - d / s.cluz) - (R)nprev * pw.deltaevol) +
                 pw.evol[nprev];
        }
    }
    ehi = ehi + pw.fpw[nfield] * ev;
    return ehi;
}

// InitNodalSources, nodalsources.F90:76-300 (points clipped to Sweep).
template <class R> void setup_nodal(Sim<R>& s, const orc_problem* p) {
    for (int q = 0; q < p->nnodal; ++q) {
        const orc_nodal& ns = p->nodal[q];
        for (int pt = 0; pt < ns.npoints; ++pt) {
            const int* b = ns.boxes + 6 * pt;
            for (int a = 0; a < 3; ++a) {
                float amp = ns.amp[3 * pt + a];
                if (amp == 0.0f) continue;
                int f = (ns.is_elec ? 0 : 3) + a;
                NodalSet<R>& set = ns.is_hard ? s.nodal_hard[f] : s.nodal_soft[f];
                const Lim& w = s.Sweep[f];
                NodalPoint<R> np;
                np.p = Lim{std::max(b[0], w.XI), std::min(b[1], w.XE), std::max(b[2], w.YI), std::min(b[3], w.YE),
                           std::max(b[4], w.ZI), std::min(b[5], w.ZE)};
                np.amp = (R)amp;
                set.pts.push_back(np);
                set.evol.assign(ns.samples, ns.samples + ns.nsamples);
                set.deltaevol = (R)ns.dsamples;
                set.numus = ns.nsamples - 1;
            }
        }
    }
}

// evolucion of nodalsources.F90:310-361.
template <class R> inline R nodal_evol(const NodalSet<R>& set, R t) {
    long long nprev = (long long)(t / set.deltaevol);
    if ((nprev + 1 > set.numus) || (nprev + 1 <= 0)) return 0;
    return (set.evol[nprev + 1] - set.evol[nprev]) / set.deltaevol * ((t) - (R)nprev * set.deltaevol) + set.evol[nprev];
}

// ---------------------------------------------------------------------------
// Per-step routines.
#define OMP_KJ _Pragma("omp parallel for collapse(2) schedule(static)")

// Advance_Ex/Ey/Ez, timestepping.F90:2165-2285.
template <class R> void advance_e(Sim<R>& s) {
    A3<R>&Ex = s.F[iEx], &Ey = s.F[iEy], &Ez = s.F[iEz], &Hx = s.F[iHx], &Hy = s.F[iHy], &Hz = s.F[iHz];
    const R* g1 = s.G1.data();
    const R* g2 = s.G2.data();
    {
        const Lim w = s.Sweep[iEx];
        OMP_KJ for (int k = w.ZI; k <= w.ZE; ++k) for (int j = w.YI; j <= w.YE; ++j) {
            R Idzhk = s.Idzh(k), Idyhj = s.Idyh(j);
            for (int i = w.XI; i <= w.XE; ++i) {
                int m = s.mi[iEx](i, j, k);
                Ex(i, j, k) = g1[m] * Ex(i, j, k) + g2[m] * ((Hz(i, j, k) - Hz(i, j - 1, k)) * Idyhj - (Hy(i, j, k) - Hy(i, j, k - 1)) * Idzhk);
            }
        }
    }
    {
        const Lim w = s.Sweep[iEy];
        OMP_KJ for (int k = w.ZI; k <= w.ZE; ++k) for (int j = w.YI; j <= w.YE; ++j) {
            R Idzhk = s.Idzh(k);
            for (int i = w.XI; i <= w.XE; ++i) {
                int m = s.mi[iEy](i, j, k);
                Ey(i, j, k) = g1[m] * Ey(i, j, k) + g2[m] * ((Hx(i, j, k) - Hx(i, j, k - 1)) * Idzhk - (Hz(i, j, k) - Hz(i - 1, j, k)) * s.Idxh(i));
            }
        }
    }
    {
        const Lim w = s.Sweep[iEz];
        OMP_KJ for (int k = w.ZI; k <= w.ZE; ++k) for (int j = w.YI; j <= w.YE; ++j) {
            R Idyhj = s.Idyh(j);
            for (int i = w.XI; i <= w.XE; ++i) {
                int m = s.mi[iEz](i, j, k);
                Ez(i, j, k) = g1[m] * Ez(i, j, k) + g2[m] * ((Hy(i, j, k) - Hy(i - 1, j, k)) * s.Idxh(i) - (Hx(i, j, k) - Hx(i, j - 1, k)) * Idyhj);
            }
        }
    }
}

// Advance_Hx/Hy/Hz, timestepping.F90:2294-2409.
template <class R> void advance_h(Sim<R>& s) {
    A3<R>&Ex = s.F[iEx], &Ey = s.F[iEy], &Ez = s.F[iEz], &Hx = s.F[iHx], &Hy = s.F[iHy], &Hz = s.F[iHz];
    const R* gm1 = s.GM1.data();
    const R* gm2 = s.GM2.data();
    {
        const Lim w = s.Sweep[iHx];
        OMP_KJ for (int k = w.ZI; k <= w.ZE; ++k) for (int j = w.YI; j <= w.YE; ++j) {
            R Idzek = s.Idze(k), Idyej = s.Idye(j);
            for (int i = w.XI; i <= w.XE; ++i) {
                int m = s.mi[iHx](i, j, k);
                Hx(i, j, k) = gm1[m] * Hx(i, j, k) + gm2[m] * ((Ey(i, j, k + 1) - Ey(i, j, k)) * Idzek - (Ez(i, j + 1, k) - Ez(i, j, k)) * Idyej);
            }
        }
    }
    {
        const Lim w = s.Sweep[iHy];
        OMP_KJ for (int k = w.ZI; k <= w.ZE; ++k) for (int j = w.YI; j <= w.YE; ++j) {
            R Idzek = s.Idze(k);
            for (int i = w.XI; i <= w.XE; ++i) {
                int m = s.mi[iHy](i, j, k);
                Hy(i, j, k) = gm1[m] * Hy(i, j, k) + gm2[m] * ((Ez(i + 1, j, k) - Ez(i, j, k)) * s.Idxe(i) - (Ex(i, j, k + 1) - Ex(i, j, k)) * Idzek);
            }
        }
    }
    {
        const Lim w = s.Sweep[iHz];
        OMP_KJ for (int k = w.ZI; k <= w.ZE; ++k) for (int j = w.YI; j <= w.YE; ++j) {
            R Idyej = s.Idye(j);
            for (int i = w.XI; i <= w.XE; ++i) {
                int m = s.mi[iHz](i, j, k);
                Hz(i, j, k) = gm1[m] * Hz(i, j, k) + gm2[m] * ((Ex(i, j + 1, k) - Ex(i, j, k)) * Idyej - (Ey(i + 1, j, k) - Ey(i, j, k)) * s.Idxe(i));
            }
        }
    }
}

// One CPML slab pass: psi = Pb*psi + (F(.) - F(.-d))*Pc ; G += sign*g2(m)*psi.
// axis: 0 x, 1 y, 2 z; electric derivative is backward, magnetic forward.
template <class R>
void cpml_pass(Sim<R>& s, A3<R>& psi, const Lim& box, A3<R>& G, const A3<R>& D, const A3<int16_t>& mi, const R* g2,
               const A1<R>& Pb, const A1<R>& Pc, int axis, bool forward, int sign) {
    if (box.ZI > box.ZE || box.YI > box.YE || box.XI > box.XE) return;
    OMP_KJ for (int k = box.ZI; k <= box.ZE; ++k) for (int j = box.YI; j <= box.YE; ++j) {
        for (int i = box.XI; i <= box.XE; ++i) {
            int c = axis == 0 ? i : (axis == 1 ? j : k);
            R diff;
            if (!forward) {
                int di = axis == 0, dj = axis == 1, dk = axis == 2;
                diff = D(i, j, k) - D(i - di, j - dj, k - dk);
            } else {
                int di = axis == 0, dj = axis == 1, dk = axis == 2;
                diff = D(i + di, j + dj, k + dk) - D(i, j, k);
            }
            psi(i, j, k) = Pb(c) * psi(i, j, k) + diff * Pc(c);
            int m = mi(i, j, k);
            if (sign > 0) G(i, j, k) = G(i, j, k) + g2[m] * psi(i, j, k);
            else G(i, j, k) = G(i, j, k) - g2[m] * psi(i, j, k);
        }
    }
}

// AdvanceelectricCPML, borderscpml.F90:584-876.
template <class R> void advance_cpml_e(Sim<R>& s) {
    const R* g2 = s.G2.data();
    for (int r = 0; r < 2; ++r) {  // left, right
        int reg = Left + r;
        cpml_pass(s, s.psiLR[r][0], s.PMLc[iEx][reg], s.F[iEx], s.F[iHz], s.mi[iEx], g2, s.P_be_y, s.P_ce_y, 1, false, +1);
        cpml_pass(s, s.psiLR[r][1], s.PMLc[iEz][reg], s.F[iEz], s.F[iHx], s.mi[iEz], g2, s.P_be_y, s.P_ce_y, 1, false, -1);
    }
    for (int r = 0; r < 2; ++r) {  // down, up
        int reg = Down + r;
        cpml_pass(s, s.psiDU[r][0], s.PMLc[iEy][reg], s.F[iEy], s.F[iHx], s.mi[iEy], g2, s.P_be_z, s.P_ce_z, 2, false, +1);
        cpml_pass(s, s.psiDU[r][1], s.PMLc[iEx][reg], s.F[iEx], s.F[iHy], s.mi[iEx], g2, s.P_be_z, s.P_ce_z, 2, false, -1);
    }
    for (int r = 0; r < 2; ++r) {  // back, front
        int reg = Back + r;
        cpml_pass(s, s.psiBF[r][0], s.PMLc[iEz][reg], s.F[iEz], s.F[iHy], s.mi[iEz], g2, s.P_be_x, s.P_ce_x, 0, false, +1);
        cpml_pass(s, s.psiBF[r][1], s.PMLc[iEy][reg], s.F[iEy], s.F[iHz], s.mi[iEy], g2, s.P_be_x, s.P_ce_x, 0, false, -1);
    }
}

// AdvanceMagneticCPML, borderscpml.F90:881-1176.
template <class R> void advance_cpml_h(Sim<R>& s) {
    const R* gm2 = s.GM2.data();
    for (int r = 0; r < 2; ++r) {
        int reg = Left + r;
        cpml_pass(s, s.psiLR[r][2], s.PMLc[iHx][reg], s.F[iHx], s.F[iEz], s.mi[iHx], gm2, s.P_bm_y, s.P_cm_y, 1, true, -1);
        cpml_pass(s, s.psiLR[r][3], s.PMLc[iHz][reg], s.F[iHz], s.F[iEx], s.mi[iHz], gm2, s.P_bm_y, s.P_cm_y, 1, true, +1);
    }
    for (int r = 0; r < 2; ++r) {
        int reg = Down + r;
        cpml_pass(s, s.psiDU[r][2], s.PMLc[iHy][reg], s.F[iHy], s.F[iEx], s.mi[iHy], gm2, s.P_bm_z, s.P_cm_z, 2, true, -1);
        cpml_pass(s, s.psiDU[r][3], s.PMLc[iHx][reg], s.F[iHx], s.F[iEy], s.mi[iHx], gm2, s.P_bm_z, s.P_cm_z, 2, true, +1);
    }
    for (int r = 0; r < 2; ++r) {
        int reg = Back + r;
        cpml_pass(s, s.psiBF[r][2], s.PMLc[iHz][reg], s.F[iHz], s.F[iEy], s.mi[iHz], gm2, s.P_bm_x, s.P_cm_x, 0, true, -1);
        cpml_pass(s, s.psiBF[r][3], s.PMLc[iHy][reg], s.F[iHy], s.F[iEz], s.mi[iHy], gm2, s.P_bm_x, s.P_cm_x, 0, true, +1);
    }
}

// AdvanceEDispersiveE, electricdispersive.F90:304-362.
template <class R> void advance_edisp(Sim<R>& s) {
    const double dt = s.dt;
    for (EDispMedium<R>& d : s.dut) {
        const int np = d.np;
        for (int c = 0; c < 3; ++c) {
            std::vector<DNode<R>>& nodes = d.nodes[c];
            A3<R>& E = s.F[c];
            const long nn = (long)nodes.size();
#pragma omp parallel for schedule(static)
            for (long q = 0; q < nn; ++q) {
                DNode<R>& n = nodes[q];
                R& E0 = E(n.i, n.j, n.k);
                C8* Jn = &d.J[c][q * np];
                for (int p = 0; p < np; ++p) {
                    double re = d.g3[p].re * Jn[p].re - d.g3[p].im * Jn[p].im;
                    E0 = (R)((double)E0 - re);
                }
                R diff = E0 - n.prev;
                for (int p = 0; p < np; ++p) {
                    C8 kj = cmul(d.kappa[p], Jn[p]);
                    C8 bd{d.beta[p].re * (double)diff, d.beta[p].im * (double)diff};
                    bd.re = bd.re / dt;
                    bd.im = bd.im / dt;
                    Jn[p] = C8{kj.re + bd.re, kj.im + bd.im};
                }
                n.prev = E0;
            }
        }
    }
}

// AdvanceMdispersiveH, magneticdispersive.F90:298-360: as the electric
// update on the H nodes, except that the current takes (Beta/dt)*(H-Hprev),
// dividing before the product.
template <class R> void advance_mdisp(Sim<R>& s) {
    const double dt = s.dt;
    for (EDispMedium<R>& d : s.mdut) {
        const int np = d.np;
        for (int c = 0; c < 3; ++c) {
            std::vector<DNode<R>>& nodes = d.nodes[c];
            A3<R>& H = s.F[3 + c];
            const long nn = (long)nodes.size();
#pragma omp parallel for schedule(static)
            for (long q = 0; q < nn; ++q) {
                DNode<R>& n = nodes[q];
                R& H0 = H(n.i, n.j, n.k);
                C8* Jn = &d.J[c][q * np];
                for (int p = 0; p < np; ++p) {
                    double re = d.g3[p].re * Jn[p].re - d.g3[p].im * Jn[p].im;
                    H0 = (R)((double)H0 - re);
                }
                R diff = H0 - n.prev;
                for (int p = 0; p < np; ++p) {
                    C8 kj = cmul(d.kappa[p], Jn[p]);
                    C8 bd{d.beta[p].re / dt, d.beta[p].im / dt};
                    bd.re = bd.re * (double)diff;
                    bd.im = bd.im * (double)diff;
                    Jn[p] = C8{kj.re + bd.re, kj.im + bd.im};
                }
                n.prev = H0;
            }
        }
    }
}

// AdvancePlaneWaveE, planewaves.F90:878-1174, called only while
// still_planewave_time holds (timestepping.F90:1423-1427); the routine lowers
// the switch before its face loops (planewaves.F90:904).
template <class R> void advance_pw_e(Sim<R>& s, int n) {
    if (s.pws.empty() || !s.still_planewave_time) return;
    s.still_planewave_time = false;
    R timei = (R)s.time(n);
    R G2_1 = s.G2[1];
    A3<R>&Ex = s.F[iEx], &Ey = s.F[iEy], &Ez = s.F[iEz];
    for (const PlaneWave<R>& pw : s.pws) {
        const PWFaces& F = pw.f;
        if (F.tr) {
            int i = F.trfr_i_tra[iEz];
            R Id = s.Idxh(i);
            for (int k = F.trfr_k_com[iEz]; k <= F.trfr_k_fin[iEz]; ++k)
                for (int j = F.trfr_j_com[iEz]; j <= F.trfr_j_fin[iEz]; ++j)
                    Ez(i, j, k) = Ez(i, j, k) - G2_1 * incid(s, pw, iHy, timei, i - 1, j, k) * Id;
            i = F.trfr_i_tra[iEy];
            Id = s.Idxh(i);
            for (int k = F.trfr_k_com[iEy]; k <= F.trfr_k_fin[iEy]; ++k)
                for (int j = F.trfr_j_com[iEy]; j <= F.trfr_j_fin[iEy]; ++j)
                    Ey(i, j, k) = Ey(i, j, k) + G2_1 * incid(s, pw, iHz, timei, i - 1, j, k) * Id;
        }
        if (F.fr) {
            int i = F.trfr_i_fro[iEz];
            R Id = s.Idxh(i);
            for (int k = F.trfr_k_com[iEz]; k <= F.trfr_k_fin[iEz]; ++k)
                for (int j = F.trfr_j_com[iEz]; j <= F.trfr_j_fin[iEz]; ++j)
                    Ez(i, j, k) = Ez(i, j, k) + G2_1 * incid(s, pw, iHy, timei, i, j, k) * Id;
            i = F.trfr_i_fro[iEy];
            Id = s.Idxh(i);
            for (int k = F.trfr_k_com[iEy]; k <= F.trfr_k_fin[iEy]; ++k)
                for (int j = F.trfr_j_com[iEy]; j <= F.trfr_j_fin[iEy]; ++j)
                    Ey(i, j, k) = Ey(i, j, k) - G2_1 * incid(s, pw, iHz, timei, i, j, k) * Id;
        }
        if (F.iz) {
            int j = F.izde_j_izq[iEx];
            R Id = s.Idyh(j);
            for (int k = F.izde_k_com[iEx]; k <= F.izde_k_fin[iEx]; ++k)
                for (int i = F.izde_i_com[iEx]; i <= F.izde_i_fin[iEx]; ++i)
                    Ex(i, j, k) = Ex(i, j, k) - G2_1 * incid(s, pw, iHz, timei, i, j - 1, k) * Id;
            j = F.izde_j_izq[iEz];
            Id = s.Idyh(j);
            for (int k = F.izde_k_com[iEz]; k <= F.izde_k_fin[iEz]; ++k)
                for (int i = F.izde_i_com[iEz]; i <= F.izde_i_fin[iEz]; ++i)
                    Ez(i, j, k) = Ez(i, j, k) + G2_1 * incid(s, pw, iHx, timei, i, j - 1, k) * Id;
        }
        if (F.de) {
            int j = F.izde_j_der[iEz];
            R Id = s.Idyh(j);
            for (int k = F.izde_k_com[iEz]; k <= F.izde_k_fin[iEz]; ++k)
                for (int i = F.izde_i_com[iEz]; i <= F.izde_i_fin[iEz]; ++i)
                    Ez(i, j, k) = Ez(i, j, k) - G2_1 * incid(s, pw, iHx, timei, i, j, k) * Id;
            j = F.izde_j_der[iEx];
            Id = s.Idyh(j);
            for (int k = F.izde_k_com[iEx]; k <= F.izde_k_fin[iEx]; ++k)
                for (int i = F.izde_i_com[iEx]; i <= F.izde_i_fin[iEx]; ++i)
                    Ex(i, j, k) = Ex(i, j, k) + G2_1 * incid(s, pw, iHz, timei, i, j, k) * Id;
        }
        if (F.ab) {
            int k = F.abar_k_aba[iEx];
            R Id = s.Idzh(k);
            for (int j = F.abar_j_com[iEx]; j <= F.abar_j_fin[iEx]; ++j)
                for (int i = F.abar_i_com[iEx]; i <= F.abar_i_fin[iEx]; ++i)
                    Ex(i, j, k) = Ex(i, j, k) + G2_1 * incid(s, pw, iHy, timei, i, j, k - 1) * Id;
            k = F.abar_k_aba[iEy];
            Id = s.Idzh(k);
            for (int j = F.abar_j_com[iEy]; j <= F.abar_j_fin[iEy]; ++j)
                for (int i = F.abar_i_com[iEy]; i <= F.abar_i_fin[iEy]; ++i)
                    Ey(i, j, k) = Ey(i, j, k) - G2_1 * incid(s, pw, iHx, timei, i, j, k - 1) * Id;
        }
        if (F.ar) {
            int k = F.abar_k_arr[iEx];
            R Id = s.Idzh(k);
            for (int j = F.abar_j_com[iEx]; j <= F.abar_j_fin[iEx]; ++j)
                for (int i = F.abar_i_com[iEx]; i <= F.abar_i_fin[iEx]; ++i)
                    Ex(i, j, k) = Ex(i, j, k) - G2_1 * incid(s, pw, iHy, timei, i, j, k) * Id;
            k = F.abar_k_arr[iEy];
            Id = s.Idzh(k);
            for (int j = F.abar_j_com[iEy]; j <= F.abar_j_fin[iEy]; ++j)
                for (int i = F.abar_i_com[iEy]; i <= F.abar_i_fin[iEy]; ++i)
                    Ey(i, j, k) = Ey(i, j, k) + G2_1 * incid(s, pw, iHx, timei, i, j, k) * Id;
        }
    }
}

// AdvancePlaneWaveH, planewaves.F90:1180-1475, under the same switch
// (timestepping.F90:1596-1600, planewaves.F90:1206).
template <class R> void advance_pw_h(Sim<R>& s, int n) {
    if (s.pws.empty() || !s.still_planewave_time) return;
    s.still_planewave_time = false;
    R timei = (R)(s.time(n) + (double)(R)0.5 * s.dt);
    R Gm2_1 = s.GM2[1];
    A3<R>&Hx = s.F[iHx], &Hy = s.F[iHy], &Hz = s.F[iHz];
    for (const PlaneWave<R>& pw : s.pws) {
        const PWFaces& F = pw.f;
        if (F.tr) {
            int i = F.trfr_i_tra[iHz];
            R Id = s.Idxe(i);
            for (int k = F.trfr_k_com[iHz]; k <= F.trfr_k_fin[iHz]; ++k)
                for (int j = F.trfr_j_com[iHz]; j <= F.trfr_j_fin[iHz]; ++j)
                    Hz(i, j, k) = Hz(i, j, k) + Gm2_1 * incid(s, pw, iEy, timei, i + 1, j, k) * Id;
            i = F.trfr_i_tra[iHy];
            Id = s.Idxe(i);
            for (int k = F.trfr_k_com[iHy]; k <= F.trfr_k_fin[iHy]; ++k)
                for (int j = F.trfr_j_com[iHy]; j <= F.trfr_j_fin[iHy]; ++j)
                    Hy(i, j, k) = Hy(i, j, k) - Gm2_1 * incid(s, pw, iEz, timei, i + 1, j, k) * Id;
        }
        if (F.fr) {
            int i = F.trfr_i_fro[iHz];
            R Id = s.Idxe(i);
            for (int k = F.trfr_k_com[iHz]; k <= F.trfr_k_fin[iHz]; ++k)
                for (int j = F.trfr_j_com[iHz]; j <= F.trfr_j_fin[iHz]; ++j)
                    Hz(i, j, k) = Hz(i, j, k) - Gm2_1 * incid(s, pw, iEy, timei, i, j, k) * Id;
            i = F.trfr_i_fro[iHy];
            Id = s.Idxe(i);
            for (int k = F.trfr_k_com[iHy]; k <= F.trfr_k_fin[iHy]; ++k)
                for (int j = F.trfr_j_com[iHy]; j <= F.trfr_j_fin[iHy]; ++j)
                    Hy(i, j, k) = Hy(i, j, k) + Gm2_1 * incid(s, pw, iEz, timei, i, j, k) * Id;
        }
        if (F.iz) {
            int j = F.izde_j_izq[iHx];
            R Id = s.Idye(j);
            for (int k = F.izde_k_com[iHx]; k <= F.izde_k_fin[iHx]; ++k)
                for (int i = F.izde_i_com[iHx]; i <= F.izde_i_fin[iHx]; ++i)
                    Hx(i, j, k) = Hx(i, j, k) + Gm2_1 * incid(s, pw, iEz, timei, i, j + 1, k) * Id;
            j = F.izde_j_izq[iHz];
            Id = s.Idye(j);
            for (int k = F.izde_k_com[iHz]; k <= F.izde_k_fin[iHz]; ++k)
                for (int i = F.izde_i_com[iHz]; i <= F.izde_i_fin[iHz]; ++i)
                    Hz(i, j, k) = Hz(i, j, k) - Gm2_1 * incid(s, pw, iEx, timei, i, j + 1, k) * Id;
        }
        if (F.de) {
            int j = F.izde_j_der[iHx];
            R Id = s.Idye(j);
            for (int k = F.izde_k_com[iHx]; k <= F.izde_k_fin[iHx]; ++k)
                for (int i = F.izde_i_com[iHx]; i <= F.izde_i_fin[iHx]; ++i)
                    Hx(i, j, k) = Hx(i, j, k) - Gm2_1 * incid(s, pw, iEz, timei, i, j, k) * Id;
            j = F.izde_j_der[iHz];
            Id = s.Idye(j);
            for (int k = F.izde_k_com[iHz]; k <= F.izde_k_fin[iHz]; ++k)
                for (int i = F.izde_i_com[iHz]; i <= F.izde_i_fin[iHz]; ++i)
                    Hz(i, j, k) = Hz(i, j, k) + Gm2_1 * incid(s, pw, iEx, timei, i, j, k) * Id;
        }
        if (F.ab) {
            int k = F.abar_k_aba[iHx];
            R Id = s.Idze(k);
            for (int j = F.abar_j_com[iHx]; j <= F.abar_j_fin[iHx]; ++j)
                for (int i = F.abar_i_com[iHx]; i <= F.abar_i_fin[iHx]; ++i)
                    Hx(i, j, k) = Hx(i, j, k) - Gm2_1 * incid(s, pw, iEy, timei, i, j, k + 1) * Id;
            k = F.abar_k_aba[iHy];
            Id = s.Idze(k);
            for (int j = F.abar_j_com[iHy]; j <= F.abar_j_fin[iHy]; ++j)
                for (int i = F.abar_i_com[iHy]; i <= F.abar_i_fin[iHy]; ++i)
                    Hy(i, j, k) = Hy(i, j, k) + Gm2_1 * incid(s, pw, iEx, timei, i, j, k + 1) * Id;
        }
        if (F.ar) {
            int k = F.abar_k_arr[iHx];
            R Id = s.Idze(k);
            for (int j = F.abar_j_com[iHx]; j <= F.abar_j_fin[iHx]; ++j)
                for (int i = F.abar_i_com[iHx]; i <= F.abar_i_fin[iHx]; ++i)
                    Hx(i, j, k) = Hx(i, j, k) + Gm2_1 * incid(s, pw, iEy, timei, i, j, k) * Id;
            k = F.abar_k_arr[iHy];
            Id = s.Idze(k);
            for (int j = F.abar_j_com[iHy]; j <= F.abar_j_fin[iHy]; ++j)
                for (int i = F.abar_i_com[iHy]; i <= F.abar_i_fin[iHy]; ++i)
                    Hy(i, j, k) = Hy(i, j, k) - Gm2_1 * incid(s, pw, iEx, timei, i, j, k) * Id;
        }
    }
}

// AdvancenodalE / AdvancenodalH, nodalsources.F90:396-777.  Soft sources
// scale by the two transverse inverse steps of the component.
template <class R> void advance_nodal(Sim<R>& s, int n, bool elec) {
    R timei = elec ? (R)s.time(n) : (R)(s.time(n) + (double)(R)0.5 * s.dt);
    const R* g2 = elec ? s.G2.data() : s.GM2.data();
    for (int a = 0; a < 3; ++a) {
        int f = (elec ? 0 : 3) + a;
        A3<R>& G = s.F[f];
        for (int hard = 1; hard >= 0; --hard) {
            const NodalSet<R>& set = hard ? s.nodal_hard[f] : s.nodal_soft[f];
            for (const NodalPoint<R>& pt : set.pts) {
                R ev = nodal_evol(set, timei);
                for (int k = pt.p.ZI; k <= pt.p.ZE; ++k)
                    for (int j = pt.p.YI; j <= pt.p.YE; ++j)
                        for (int i = pt.p.XI; i <= pt.p.XE; ++i) {
                            int m = s.mi[f](i, j, k);
                            if (elec && s.med[m].pec) continue;
                            if (hard) {
                                G(i, j, k) = pt.amp * ev;
                            } else {
                                R I1, I2;
                                if (elec) {
                                    I1 = a == 0 ? s.Idyh(j) : s.Idxh(i);
                                    I2 = a == 2 ? s.Idyh(j) : s.Idzh(k);
                                } else {
                                    I1 = a == 0 ? s.Idye(j) : s.Idxe(i);
                                    I2 = a == 2 ? s.Idye(j) : s.Idze(k);
                                }
                                G(i, j, k) = G(i, j, k) - g2[m] * I1 * I2 * pt.amp * ev;
                            }
                        }
            }
        }
    }
}

// One whole-plane assignment F(plane dst) = +-F(plane src) along `axis`,
// over the full Alloc extent of the other two axes.
template <class R> void plane_copy(A3<R>& F, int axis, int dst, int src, bool negate) {
    const Lim& b = F.b;
    int lo[3] = {b.XI, b.YI, b.ZI}, hi[3] = {b.XE, b.YE, b.ZE};
    lo[axis] = hi[axis] = dst;
    const int sh = src - dst;
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                const R v = F(i + (axis == 0 ? sh : 0), j + (axis == 1 ? sh : 0), k + (axis == 2 ? sh : 0));
                F(i, j, k) = negate ? -v : v;
            }
}

// The twelve (component, face) assignments of MinusCloneMagneticPMC and
// CloneMagneticPeriodic in their order: Hx down/up/left/right, Hy back/front/
// down/up, Hz back/front/left/right (bordersother.F90:82-135, 157-189).
const int kCloneOps[12][3] = {{iHx, 2, 0}, {iHx, 2, 1}, {iHx, 1, 0}, {iHx, 1, 1}, {iHy, 0, 0}, {iHy, 0, 1},
                              {iHy, 2, 0}, {iHy, 2, 1}, {iHz, 0, 0}, {iHz, 0, 1}, {iHz, 1, 0}, {iHz, 1, 1}};

// MinusCloneMagneticPMC, bordersother.F90:65-140: the H outside a PMC face
// is minus the first swept H (image theory); one layout, so the z faces
// always apply.
template <class R> void clone_pmc(Sim<R>& s) {
    for (const auto& op : kCloneOps) {
        const int f = op[0], a = op[1], sd = op[2];
        if (!s.isPMC[a][sd]) continue;
        const Lim& c = s.Sweep[f];
        const int lo = a == 0 ? c.XI : (a == 1 ? c.YI : c.ZI), hi = a == 0 ? c.XE : (a == 1 ? c.YE : c.ZE);
        if (sd == 0) plane_copy(s.F[f], a, lo - 1, lo, true);
        else plane_copy(s.F[f], a, hi + 1, hi, true);
    }
}

// CloneMagneticPeriodic, bordersother.F90:146-190: the H outside a periodic
// face is the swept H at the opposite end.
template <class R> void clone_periodic(Sim<R>& s) {
    for (const auto& op : kCloneOps) {
        const int f = op[0], a = op[1], sd = op[2];
        if (!s.isPer[a][sd]) continue;
        const Lim& c = s.Sweep[f];
        const int lo = a == 0 ? c.XI : (a == 1 ? c.YI : c.ZI), hi = a == 0 ? c.XE : (a == 1 ? c.YE : c.ZE);
        if (sd == 0) plane_copy(s.F[f], a, lo - 1, hi, false);
        else plane_copy(s.F[f], a, hi + 1, lo, false);
    }
}

// AdvanceMagneticMUR, first order (bordersmur.F90:1129-1383), then the
// storage of the Past_ layers (:1396-1650):
//   H(outer) = Past(inner) + CAB1(medium of the inner node) * (H(inner) - Past(outer))
template <class R> void advance_mur(Sim<R>& s) {
    if (!s.anyMur) return;
    struct Part { int reg, comp; A3<R>* past; };
    const Part parts[12] = {{Left, iHx, &s.pastLR[0][0]},  {Left, iHz, &s.pastLR[0][1]},  {Right, iHx, &s.pastLR[1][0]},
                            {Right, iHz, &s.pastLR[1][1]}, {Down, iHy, &s.pastDU[0][0]},  {Down, iHx, &s.pastDU[0][1]},
                            {Up, iHy, &s.pastDU[1][0]},    {Up, iHx, &s.pastDU[1][1]},    {Back, iHz, &s.pastBF[0][0]},
                            {Back, iHy, &s.pastBF[0][1]},  {Front, iHz, &s.pastBF[1][0]}, {Front, iHy, &s.pastBF[1][1]}};
    for (const Part& p : parts) {
        const int a = kRegAxis[p.reg], side = kRegSide[p.reg];
        if (!s.isMur[a][side]) continue;
        const Lim& b = s.MURc[p.comp][p.reg];
        int lo[3] = {b.XI, b.YI, b.ZI}, hi[3] = {b.XE, b.YE, b.ZE};
        const int outer = side == 0 ? lo[a] : hi[a], d = side == 0 ? 1 : -1;
        lo[a] = hi[a] = outer;
        A3<R>& H = s.F[p.comp];
        A3<R>& P = *p.past;
        const std::vector<R>& cab = s.CAB1[p.reg];
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i) {
                    const int ii = i + (a == 0 ? d : 0), jj = j + (a == 1 ? d : 0), kk = k + (a == 2 ? d : 0);
                    const int medio = s.mi[p.comp](ii, jj, kk);
                    H(i, j, k) = P(ii, jj, kk) + cab[medio] * (H(ii, jj, kk) - P(i, j, k));
                }
    }
    for (const Part& p : parts) {
        if (!s.isMur[kRegAxis[p.reg]][kRegSide[p.reg]]) continue;
        const Lim& b = s.MURc[p.comp][p.reg];
        for (int k = b.ZI; k <= b.ZE; ++k)
            for (int j = b.YI; j <= b.YE; ++j)
                for (int i = b.XI; i <= b.XE; ++i) (*p.past)(i, j, k) = s.F[p.comp](i, j, k);
    }
}

// The loop body of timestepping.F90:1286-1712 for the routines of this path.
template <class R> void one_step(Sim<R>& s, int n) {
    advance_e(s);
    advance_cpml_e(s);
    advance_edisp(s);
    advance_pw_e(s, n);
    advance_nodal(s, n, true);
    advance_h(s);
    advance_cpml_h(s);
    clone_pmc(s);
    clone_periodic(s);
    advance_mdisp(s);
    advance_pw_h(s, n);
    advance_nodal(s, n, false);
    clone_pmc(s);
    clone_periodic(s);
    advance_mur(s);
}

template <class R> int create(const orc_problem* p, Sim<R>** out) {
    Sim<R>* s = new (std::nothrow) Sim<R>();
    if (!s) return 2;
    for (int f = 0; f < 6; ++f) {
        const int kind = p->border[f] == 0 ? 9 : p->border[f];
        if (kind != 1 && kind != 2 && kind != 4 && kind != 7 && kind != 9) { delete s; return 3; }
        if (kind == 9 && p->pml_layers[f] < 1) { delete s; return 3; }
    }
    setup_grid(*s, p);
    setup_dt(*s, p);
    setup_media(*s, p);
    calc_g(*s);
    for (int f = 0; f < 6; ++f) s->F[f].alloc(s->Alloc[f], (R)0);
    setup_metrics(*s);
    setup_cpml(*s);
    setup_mur(*s);
    setup_disp(*s, p, false);
    setup_disp(*s, p, true);
    setup_planewave(*s, p);
    setup_nodal(*s, p);
    s->probes.assign(p->probes, p->probes + 4 * p->nprobes);
    *out = s;
    return 0;
}

struct Handle {
    int fp64;
    Sim<float>* sf = nullptr;
    Sim<double>* sd = nullptr;
    int nthreads;
};

// UpdateObservation for a frequency-domain volume probe after step n
// (observation.F90:3527-3600): auxExp_E = dt*(1,0)*Exp(mcPI2*Freq*at),
// auxExp_H = auxExp_E*Exp(mcPI2*Freq*dt*0.5), mcPI2 = -(0,1)*2*pi in real(4)
// constants (fdetypes.F90:190), then V = V + auxExp*F for the three
// components at every sampled node.  Complex times real multiplies both parts.
template <class R> void update_freq_probe(Sim<R>& s, typename Sim<R>::FreqProbe& p, int n) {
    const double at = s.time(n);
    const std::complex<double> mcpi2(-0.0, -(double)(2.0f * 3.14159265358979323846f));
    const int c0 = p.mag ? 3 : 0;
    const long nodes = (long)p.ni * p.nj * p.nk;
    for (size_t f = 0; f < p.freq.size(); ++f) {
        const std::complex<double> z = mcpi2 * (double)p.freq[f];
        std::complex<double> w = s.dt * std::exp(z * at);
        if (p.mag) w = w * std::exp(z * s.dt * 0.5);
        for (int c = 0; c < 3; ++c)
            for (int kk = 0; kk < p.nk; ++kk)
                for (int jj = 0; jj < p.nj; ++jj)
                    for (int ii = 0; ii < p.ni; ++ii) {
                        const double v = (double)s.F[c0 + c]((p.i0 + ii) * p.tr[0], (p.j0 + jj) * p.tr[1], (p.k0 + kk) * p.tr[2]);
                        std::complex<double>& a = p.V[((f * 3 + c) * nodes) + ((long)kk * p.nj + jj) * p.ni + ii];
                        a = a + w * v;
                    }
    }
}

// Restart records (resuming.F90:213-496 and the Init* resume branches):
// Fortran sequential unformatted, each record framed by its byte length.
struct RecIO {
    FILE* f = nullptr;
    bool write = false, ok = true;
    void rec(void* p, size_t n) {
        if (!ok) return;
        int32_t m = (int32_t)n, b = -1;
        if (write) {
            ok = fwrite(&m, 4, 1, f) == 1 && (!n || fwrite(p, 1, n, f) == n) && fwrite(&m, 4, 1, f) == 1;
        } else {
            ok = fread(&b, 4, 1, f) == 1 && b == m && (!n || fread(p, 1, n, f) == n) && fread(&b, 4, 1, f) == 1 && b == m;
        }
    }
};

template <class R> void resume_body(Sim<R>& s, RecIO& r) {
    // StoreFields / ReadFields: rows of BLOCK_SIZE = 1024 values and a remainder
    for (int f = 0; f < 6; ++f) {
        A3<R>& a = s.F[f];
        for (int k = a.b.ZI; k <= a.b.ZE; ++k)
            for (int j = a.b.YI; j <= a.b.YE; ++j) {
                R* row = &a(a.b.XI, j, k);
                long i = 0;
                for (; i + 1024 <= a.sx; i += 1024) r.rec(row + i, 1024 * sizeof(R));
                r.rec(row + i, (a.sx - i) * sizeof(R));
            }
    }
    auto rows = [&](A3<R>& a, bool zeros) {
        std::vector<R> z(std::max(0L, a.sx), (R)0);
        for (int k = a.b.ZI; k <= a.b.ZE; ++k)
            for (int j = a.b.YI; j <= a.b.YE; ++j) {
                if (zeros) {
                    r.rec(z.data(), a.sx * sizeof(R));
                    if (!r.write) std::fill(z.begin(), z.end(), (R)0);
                } else {
                    r.rec(&a(a.b.XI, j, k), a.sx * sizeof(R));
                }
            }
    };
    // StoreFieldsCPMLBorders (borderscpml.F90:481-558)
    bool anyPML = false;
    for (int a = 0; a < 3; ++a)
        for (int sd = 0; sd < 2; ++sd) anyPML = anyPML || s.isPML[a][sd];
    if (anyPML) {
        for (int q = 0; q < 2; ++q)
            for (int w = 0; w < 4; ++w) rows(s.psiLR[q][w], false);
        for (int q = 0; q < 2; ++q)
            for (int w = 0; w < 4; ++w) rows(s.psiDU[q][w], false);
        for (int q = 0; q < 2; ++q)
            for (int w = 0; w < 4; ++w) rows(s.psiBF[q][w], false);
    }
    // StoreFieldsMURBorders (bordersmur.F90:369-454): Past_, then PastPast_
    // (never updated by the first-order branch: zeros of the same boxes)
    if (s.anyMur)
        for (int pass = 0; pass < 2; ++pass) {
            for (int q = 0; q < 2; ++q)
                for (int w = 0; w < 2; ++w) rows(s.pastLR[q][w], pass == 1);
            for (int q = 0; q < 2; ++q)
                for (int w = 0; w < 2; ++w) rows(s.pastDU[q][w], pass == 1);
            for (int q = 0; q < 2; ++q)
                for (int w = 0; w < 2; ++w) rows(s.pastBF[q][w], pass == 1);
        }
    // StoreFieldsEDispersives / StoreFieldsMDispersives
    for (auto* list : {&s.dut, &s.mdut})
        for (auto& m : *list)
            for (int c = 0; c < 3; ++c)
                for (size_t q = 0; q < m.nodes[c].size(); ++q) {
                    r.rec(&m.nodes[c][q].prev, sizeof(R));
                    for (int p = 0; p < m.np; ++p) {
                        C8& j = m.J[c][q * m.np + p];
                        double v[2] = {j.re, j.im};
                        r.rec(v, sizeof(v));
                        j = C8{v[0], v[1]};
                    }
                }
}

template <class R> int resume_io(Sim<R>& s, const char* path, bool write, int* n) {
    RecIO r;
    r.write = write;
    r.f = fopen(path, write ? "wb" : "rb");
    if (!r.f) return 2;
    // header: n, tiempo(n), dt, eps0, mu0 in one record
    unsigned char hd[4 + 8 + 8 + 2 * sizeof(R)];
    if (write) {
        const int32_t nn = *n;
        const double t = s.time(*n), dt = s.dt;
        std::memcpy(hd, &nn, 4);
        std::memcpy(hd + 4, &t, 8);
        std::memcpy(hd + 12, &dt, 8);
        std::memcpy(hd + 20, &s.eps0, sizeof(R));
        std::memcpy(hd + 20 + sizeof(R), &s.mu0, sizeof(R));
    }
    r.rec(hd, sizeof(hd));
    if (!write && r.ok) {
        int32_t nn;
        double dt;
        std::memcpy(&nn, hd, 4);
        std::memcpy(&dt, hd + 12, 8);
        *n = nn;
        if (dt != s.dt) r.ok = false;
    }
    if (r.ok) resume_body(s, r);
    if (!write && r.ok && fgetc(r.f) != EOF) r.ok = false;
    // a resumed run starts with the plane-wave switch up (timestepping.F90:1219)
    if (!write && r.ok) s.still_planewave_time = true;
    fclose(r.f);
    return r.ok ? 0 : 1;
}

// UpdateFarField, farfield.F90:1163-1733.
template <class R> void update_farfield(Sim<R>& s, typename Sim<R>::FarOrc& ff, int ntime) {
    if ((ntime - 1) % ff.ndecim != 0) return;
    const int nf = (int)ff.freq.size();
    for (int fc = 0; fc < 6; ++fc) {
        if (!ff.on[fc]) continue;
        const int axis = fc / 2;
        for (int k = 0; k < 6; ++k) {
            auto& A = ff.arr[fc][k];
            const int n1 = A.hi1 - A.lo1 + 1, n2 = A.hi2 - A.lo2 + 1;
            if (n1 <= 0 || n2 <= 0) continue;
            const auto& aux = A.comp >= 3 ? ff.auxH : ff.auxE;
            for (int o = A.lo1; o <= A.hi1; ++o)
                for (int u = A.lo2; u <= A.hi2; ++u) {
                    int i, j, kk;
                    if (axis == 0) { i = A.plane; j = u; kk = o; }
                    else if (axis == 1) { i = u; j = A.plane; kk = o; }
                    else { i = u; j = o; kk = A.plane; }
                    const double v = (double)s.F[A.comp](i, j, kk);
                    for (int f = 0; f < nf; ++f) {
                        std::complex<double>& x = A.v[((size_t)f * n1 + (o - A.lo1)) * n2 + (u - A.lo2)];
                        x = std::complex<double>(x.real() + aux[f].real() * v, x.imag() + aux[f].imag() * v);
                    }
                }
        }
    }
    for (int f = 0; f < nf; ++f) {
        const std::complex<double> a = ff.auxE[f], b = ff.auxH[f], e = ff.expIwdt[f];
        ff.auxE[f] = {a.real() * e.real() - a.imag() * e.imag(), a.real() * e.imag() + a.imag() * e.real()};
        ff.auxH[f] = {b.real() * e.real() - b.imag() * e.imag(), b.real() * e.imag() + b.imag() * e.real()};
    }
}

// InitFarField, farfield.F90:118-1158, for one layout.
template <class R> int add_farfield(Sim<R>& s, const int* box, const int* faces, float fi_, float ff_, float fs_, int logf,
                                    int decimate) {
    typename Sim<R>::FarOrc F;
    const Lim &HX = s.SINPML[3], &HY = s.SINPML[4], &HZ = s.SINPML[5];
    int e[6] = {std::max(box[0], HX.XI), std::min(box[1], HX.XE), std::max(box[2], HY.YI),
                std::min(box[3], HY.YE), std::max(box[4], HZ.ZI), std::min(box[5], HZ.ZE)};
    const Lim &WX = s.SINPMLSweep[3], &WY = s.SINPMLSweep[4], &WZ = s.SINPMLSweep[5];
    const bool in[6] = {e[0] > WX.XI && e[0] <= WX.XE, e[1] < WX.XE && e[1] >= WX.XI, e[2] > WY.YI && e[2] <= WY.YE,
                        e[3] < WY.YE && e[3] >= WY.YI, e[4] > WZ.ZI && e[4] <= WZ.ZE, e[5] < WZ.ZE && e[5] >= WZ.ZI};
    const bool edge[6] = {e[0] <= HX.XI, e[1] >= HX.XE, e[2] <= HY.YI, e[3] >= HY.YE, e[4] <= HZ.ZI, e[5] >= HZ.ZE};
    for (int f = 0; f < 6; ++f) {
        const bool image = s.isPEC[f / 2][f % 2] || s.isPMC[f / 2][f % 2];
        if (!edge[f] || !image) continue;
        for (int g = 0; g < 6; ++g)
            if (g != f && in[g]) return -2;  // NF2FF STILL UNSUPPORTED
    }
    for (int f = 0; f < 6; ++f) F.on[f] = in[f] && faces[f];
    const Lim &Sx = s.SINPMLSweep[0], &Sy = s.SINPMLSweep[1], &Sz = s.SINPMLSweep[2];
    for (int sd = 0; sd < 2; ++sd) {
        const bool lo = sd == 0;
        int* L = F.lim[sd][0];  // TrFr Ez
        L[0] = lo ? std::max(Sz.XI, e[0]) : std::min(Sz.XE, e[1]);
        L[1] = std::max(Sz.ZI, e[4]); L[2] = std::min(Sz.ZE, e[5] - 1); L[3] = std::max(Sz.YI, e[2]); L[4] = std::min(Sz.YE, e[3]);
        L = F.lim[sd][1];  // TrFr Ey
        L[0] = lo ? std::max(Sy.XI, e[0]) : std::min(Sy.XE, e[1]);
        L[1] = std::max(Sy.ZI, e[4]); L[2] = std::min(Sy.ZE - 1, e[5]); L[3] = std::max(Sy.YI, e[2]); L[4] = std::min(Sy.YE, e[3] - 1);
        L = F.lim[2 + sd][0];  // IzDe Ez
        L[0] = lo ? std::max(Sz.YI, e[2]) : std::min(Sz.YE, e[3]);
        L[1] = std::max(Sz.ZI, e[4]); L[2] = std::min(Sz.ZE, e[5] - 1); L[3] = std::max(Sz.XI, e[0]); L[4] = std::min(Sz.XE, e[1]);
        L = F.lim[2 + sd][1];  // IzDe Ex
        L[0] = lo ? std::max(Sx.YI, e[2]) : std::min(Sx.YE, e[3]);
        L[1] = std::max(Sx.ZI, e[4]); L[2] = std::min(Sx.ZE - 1, e[5]); L[3] = std::max(Sx.XI, e[0]); L[4] = std::min(Sx.XE, e[1] - 1);
        L = F.lim[4 + sd][0];  // AbAr Ey
        L[0] = lo ? std::max(Sy.ZI, e[4]) : std::min(Sy.ZE, e[5]);
        L[1] = std::max(Sy.YI, e[2]); L[2] = std::min(Sy.YE, e[3] - 1); L[3] = std::max(Sy.XI, e[0]); L[4] = std::min(Sy.XE, e[1]);
        L = F.lim[4 + sd][1];  // AbAr Ex
        L[0] = lo ? std::max(Sx.ZI, e[4]) : std::min(Sx.ZE, e[5]);
        L[1] = std::max(Sx.YI, e[2]); L[2] = std::min(Sx.YE, e[3]); L[3] = std::max(Sx.XI, e[0]); L[4] = std::min(Sx.XE, e[1] - 1);
    }
    const R fi = (R)fi_, ffin = (R)ff_, fs = (R)fs_;
    const int nf = fs != (R)0 ? (int)(std::fabs(fi - ffin) / fs) + 1 : 1;
    if (nf < 1 || nf > 100000) return -1;
    R init = fi, step = fs;
    if (logf) {
        init = std::log10(fi);
        step = std::fabs(init - std::log10(ffin)) / (R)nf;
    }
    for (int q = 0; q < nf; ++q) {
        const R x = init + (R)q * step;
        F.freq.push_back(logf ? (R)std::pow((R)10, x) : x);
    }
    F.ndecim = decimate ? std::max((int)((double)((R)0.5 / ffin) / s.dt) - 1, 1) : 1;
    F.dtDecim = (R)((double)F.ndecim * s.dt);
    const R pi = (R)3.14159265358979323846;
    for (int q = 0; q < nf; ++q) {
        // Exp(-(0,1) * 2 * pi * freq * dtDecim) in complex(RKIND)
        const std::complex<R> z4(-(R)0, ((-((R)2 * pi)) * F.freq[q]) * F.dtDecim);
        const std::complex<R> e4 = std::exp(z4);
        F.expIwdt.push_back(std::complex<double>((double)e4.real(), (double)e4.imag()));
        F.auxE.push_back(std::complex<double>((double)F.dtDecim, 0.0));
        // the half-step factor is a complex(8) exponential (sgg%dt is real(8))
        const double x = s.dt * 0.5;
        const std::complex<double> eh = std::exp(std::complex<double>(-0.0 * x, (double)((-((R)2 * pi)) * F.freq[q]) * x));
        F.auxH.push_back(std::complex<double>((double)F.dtDecim * eh.real(), (double)F.dtDecim * eh.imag()));
    }
    const int tan[3][2] = {{2, 1}, {2, 0}, {1, 0}};
    for (int fc = 0; fc < 6; ++fc) {
        if (!F.on[fc]) continue;
        const int axis = fc / 2;
        for (int t = 0; t < 2; ++t) {
            const int* L = F.lim[fc][t];
            const int c = tan[axis][t], hc = 3 + (3 - axis - c);
            const int hp = fc % 2 == 0 ? L[0] - 1 : L[0];  // TrFr%I%tra%Hy = tra%Ez - 1, fro%Hy = fro%Ez
            const int comp[3] = {c, hc, hc}, plane[3] = {L[0], hp, hp + 1}, slot[3] = {t, 2 + 2 * t, 3 + 2 * t};
            for (int q = 0; q < 3; ++q) {
                auto& A = F.arr[fc][slot[q]];
                A.comp = comp[q];
                A.plane = plane[q];
                A.lo1 = L[1]; A.hi1 = L[2]; A.lo2 = L[3]; A.hi2 = L[4];
                const long n1 = std::max(0, L[2] - L[1] + 1), n2 = std::max(0, L[4] - L[3] + 1);
                A.v.assign((size_t)nf * n1 * n2, std::complex<double>(0.0, 0.0));
            }
        }
    }
    s.farfields.push_back(std::move(F));
    return (int)s.farfields.size() - 1;
}

// update_LN, farfield.F90:3426-3449.
struct LN {
    std::complex<double> Lt, Lp, Nt, Np;
};
template <class R> void update_ln(std::complex<double> comun, const R co[6][3], const R* t, const std::complex<double>* MJ,
                                  LN& ln) {
    // t: sintheta_cosphi, sintheta_sinphi, costheta, costheta_cosphi, costheta_sinphi, sintheta, sinphi, cosphi
    std::complex<double> cm[6];
    for (int k = 0; k < 6; ++k) {
        const R d = co[k][0] * t[0] + co[k][1] * t[1] + co[k][2] * t[2];
        const std::complex<double> z(comun.real() * (double)d, comun.imag() * (double)d);
        cm[k] = std::exp(z);
    }
    auto sc = [](std::complex<double> a, R r) { return std::complex<double>(a.real() * (double)r, a.imag() * (double)r); };
    ln.Lt = ln.Lt + (sc(MJ[0], t[3]) * cm[0] + sc(MJ[1], t[4]) * cm[1] - sc(MJ[2], t[5]) * cm[2]);
    ln.Lp = ln.Lp + (sc(-MJ[0], t[6]) * cm[0] + sc(MJ[1], t[7]) * cm[1]);
    ln.Nt = ln.Nt + (sc(MJ[3], t[3]) * cm[3] + sc(MJ[4], t[4]) * cm[4] - sc(MJ[5], t[5]) * cm[5]);
    ln.Np = ln.Np + (sc(-MJ[3], t[6]) * cm[3] + sc(MJ[4], t[7]) * cm[4]);
}

// average(), farfield.F90:3553-3579.
template <class R> std::complex<double> ff_average(int pasadas, std::complex<double> z1, std::complex<double> z2) {
    const R pi = (R)3.14159265358979323846;
    if (pasadas == 2) {
        const R phi1 = (R)std::atan2(z1.imag(), z1.real()), phi2 = (R)std::atan2(z2.imag(), z2.real());
        R n1 = phi1, n2 = phi2;
        if (phi1 < -pi / (R)2 && phi2 > pi / (R)2) n1 = phi1 - (R)2 * pi;
        if (phi2 < -pi / (R)2 && phi1 > pi / (R)2) n2 = phi2 - (R)2 * pi;
        const std::complex<R> e = std::exp(std::complex<R>((R)0, (n1 + n2) / (R)2));
        const std::complex<double> p(z1.real() * z2.real() - z1.imag() * z2.imag(), z1.real() * z2.imag() + z1.imag() * z2.real());
        const double r = std::sqrt(std::abs(p));
        return {r * (double)e.real(), r * (double)e.imag()};
    }
    return {(z1.real() + z2.real()) / 2.0, (z1.imag() + z2.imag()) / 2.0};
}

// FlushFarfield, farfield.F90:2408-3423 (one layout, no image faces): rows of
// freq, theta, phi, |Etheta|, arg Etheta, |Ephi|, arg Ephi, RCS(arit), RCS(geom).
template <class R> int farfield_transform(Sim<R>& s, int id, const float* ang, const float* inc, int ninc, double* out,
                                          int max_rows, int* rows) {
    if (id < 0 || id >= (int)s.farfields.size()) return 1;
    auto& F = s.farfields[id];
    const R pi = (R)3.14159265358979323846;
    const R ts = (R)ang[0], tstop = (R)ang[1], tstep = (R)ang[2], ps = (R)ang[3], pstop = (R)ang[4], pstep = (R)ang[5];
    if (!(tstep > 0) || !(pstep > 0)) return 1;
    std::vector<R> dirs;
    for (R theta = ts - tstep; theta < tstop;) {
        theta = std::min(theta + tstep, tstop);
        for (R phi = ps - pstep; phi < pstop;) {
            phi = std::min(phi + pstep, pstop);
            dirs.push_back(theta);
            dirs.push_back(phi);
        }
    }
    const int nd = (int)dirs.size() / 2, nf = (int)F.freq.size();
    *rows = nd * nf;
    if (!out) return 0;
    if (max_rows < nd * nf || ninc < 2) return 1;
    // dftEntrada, :1021-1070
    std::vector<std::complex<double>> dft(nf);
    {
        const R dtevol = (R)inc[2] - (R)inc[0];
        const std::complex<double> mcpi2(-0.0, -(double)((R)2 * pi));
        for (int q = 0; q < nf; ++q) {
            const std::complex<double> z = std::complex<double>(mcpi2.real() * (double)F.freq[q], mcpi2.imag() * (double)F.freq[q]);
            const std::complex<double> ex = std::exp(std::complex<double>(z.real() * (double)dtevol, z.imag() * (double)dtevol));
            std::complex<double> aux((double)dtevol, 0.0), acc(0.0, 0.0);
            for (int m = 1; m < ninc; ++m) {
                const double v = (double)(R)inc[2 * m + 1];
                acc = std::complex<double>(acc.real() + v * aux.real(), acc.imag() + v * aux.imag());
                aux = std::complex<double>(aux.real() * ex.real() - aux.imag() * ex.imag(), aux.real() * ex.imag() + aux.imag() * ex.real());
            }
            dft[q] = acc;
        }
    }
    auto cell = [&](const A1<R>& a, int i) { return a(i); };
    auto val = [&](const typename Sim<R>::FarArr& A, int f, int o, int u) -> std::complex<double> {
        if (o < A.lo1 || o > A.hi1 || u < A.lo2 || u > A.hi2) return {0.0, 0.0};
        const int n1 = A.hi1 - A.lo1 + 1, n2 = A.hi2 - A.lo2 + 1;
        return A.v[((size_t)f * n1 + (o - A.lo1)) * n2 + (u - A.lo2)];
    };
    auto sc = [](std::complex<double> a, R r) { return std::complex<double>(a.real() * (double)r, a.imag() * (double)r); };
    int row = 0;
    for (int ii = 0; ii < nf; ++ii) {
        const R freq = F.freq[ii];
        const std::complex<R> c4 = std::complex<R>((R)0, (((R)2 * pi) * freq) / s.cluz);
        const std::complex<double> comun((double)c4.real(), (double)c4.imag());
        for (int d = 0; d < nd; ++d) {
            const R theta = dirs[2 * d], phi = dirs[2 * d + 1];
            double Et[3][2] = {}, Ep[3][2] = {};
            R rcs[3] = {};
            for (int pasadas = 2; pasadas >= 1; --pasadas) {
                const R t[8] = {std::sin(theta) * std::cos(phi), std::sin(theta) * std::sin(phi), std::cos(theta),
                                std::cos(theta) * std::cos(phi), std::cos(theta) * std::sin(phi), std::sin(theta),
                                std::sin(phi), std::cos(phi)};
                LN fin{};
                for (int fc = 0; fc < 6; ++fc) {
                    if (!F.on[fc]) continue;
                    const int axis = fc / 2;
                    const R normal = fc % 2 == 0 ? (R)-1 : (R)1;
                    const auto* A = F.arr[fc];
                    const int(*L)[5] = F.lim[fc];
                    LN ln{};
                    // co rows: Mx, My, Mz, Jx, Jy, Jz; MJ the same order
                    if (axis == 0) {
                        const int i = L[0][0];
                        for (int k = L[0][1]; k <= L[1][2]; ++k)
                            for (int j = L[0][3]; j <= L[0][4]; ++j) {
                                std::complex<double> MJ[6] = {};
                                if (k <= L[0][2]) MJ[1] = sc(sc(sc(-val(A[0], ii, k, j), cell(s.dyh, j)), cell(s.dze, k)), normal);
                                if (j <= L[1][4]) MJ[2] = sc(sc(sc(val(A[1], ii, k, j), cell(s.dye, j)), cell(s.dzh, k)), normal);
                                if (k <= L[1][2]) MJ[4] = sc(sc(sc(ff_average<R>(pasadas, val(A[4], ii, k, j), val(A[5], ii, k, j)), cell(s.dye, j)), cell(s.dzh, k)), normal);
                                if (j <= L[0][4]) MJ[5] = sc(sc(sc(-ff_average<R>(pasadas, val(A[2], ii, k, j), val(A[3], ii, k, j)), cell(s.dyh, j)), cell(s.dze, k)), normal);
                                R co[6][3] = {};
                                const R pz[3] = {s.physc(2, 0, i), s.physc(2, 1, j), s.physc(2, 2, k)};
                                const R py[3] = {s.physc(1, 0, i), s.physc(1, 1, j), s.physc(1, 2, k)};
                                for (int a = 0; a < 3; ++a) { co[1][a] = pz[a]; co[2][a] = py[a]; co[4][a] = py[a]; co[5][a] = pz[a]; }
                                update_ln<R>(comun, co, t, MJ, ln);
                            }
                    } else if (axis == 1) {
                        const int j = L[1][0];
                        for (int k = L[1][1]; k <= L[1][2]; ++k)
                            for (int i = L[1][3]; i <= L[0][4]; ++i) {
                                std::complex<double> MJ[6] = {};
                                if (k <= L[0][2]) MJ[0] = sc(sc(sc(val(A[0], ii, k, i), cell(s.dxh, i)), cell(s.dze, k)), normal);
                                if (i <= L[1][4]) MJ[2] = sc(sc(sc(-val(A[1], ii, k, i), cell(s.dxe, i)), cell(s.dzh, k)), normal);
                                if (k <= L[1][2]) MJ[3] = sc(sc(sc(-ff_average<R>(pasadas, val(A[4], ii, k, i), val(A[5], ii, k, i)), cell(s.dxe, i)), cell(s.dzh, k)), normal);
                                if (i <= L[0][4]) MJ[5] = sc(sc(sc(ff_average<R>(pasadas, val(A[2], ii, k, i), val(A[3], ii, k, i)), cell(s.dxh, i)), cell(s.dze, k)), normal);
                                R co[6][3] = {};
                                const R pz[3] = {s.physc(2, 0, i), s.physc(2, 1, j), s.physc(2, 2, k)};
                                const R px[3] = {s.physc(0, 0, i), s.physc(0, 1, j), s.physc(0, 2, k)};
                                for (int a = 0; a < 3; ++a) { co[0][a] = pz[a]; co[2][a] = px[a]; co[5][a] = pz[a]; co[3][a] = px[a]; }
                                update_ln<R>(comun, co, t, MJ, ln);
                            }
                    } else {
                        const int k = L[0][0];
                        for (int j = L[0][1]; j <= L[1][2]; ++j)
                            for (int i = L[0][3]; i <= L[0][4]; ++i) {
                                std::complex<double> MJ[6] = {};
                                if (j <= L[0][2]) MJ[0] = sc(sc(sc(-val(A[0], ii, j, i), cell(s.dxh, i)), cell(s.dye, j)), normal);
                                if (i <= L[1][4]) MJ[1] = sc(sc(sc(val(A[1], ii, j, i), cell(s.dxe, i)), cell(s.dyh, j)), normal);
                                if (j <= L[1][2]) MJ[3] = sc(sc(sc(ff_average<R>(pasadas, val(A[4], ii, j, i), val(A[5], ii, j, i)), cell(s.dxe, i)), cell(s.dyh, j)), normal);
                                if (i <= L[0][4]) MJ[4] = sc(sc(sc(-ff_average<R>(pasadas, val(A[2], ii, j, i), val(A[3], ii, j, i)), cell(s.dxh, i)), cell(s.dye, j)), normal);
                                R co[6][3] = {};
                                const R py[3] = {s.physc(1, 0, i), s.physc(1, 1, j), s.physc(1, 2, k)};
                                const R px[3] = {s.physc(0, 0, i), s.physc(0, 1, j), s.physc(0, 2, k)};
                                for (int a = 0; a < 3; ++a) { co[0][a] = py[a]; co[1][a] = px[a]; co[3][a] = px[a]; co[4][a] = py[a]; }
                                update_ln<R>(comun, co, t, MJ, ln);
                            }
                    }
                    fin.Lt += ln.Lt; fin.Lp += ln.Lp; fin.Nt += ln.Nt; fin.Np += ln.Np;
                }
                const R be = -freq / ((R)2 * s.cluz), bp = freq / ((R)2 * s.cluz);
                const std::complex<double> X = fin.Lp + sc(fin.Nt, s.zvac), Y = fin.Lt - sc(fin.Np, s.zvac);
                Et[pasadas][0] = -((double)be * X.imag()); Et[pasadas][1] = (double)be * X.real();
                Ep[pasadas][0] = -((double)bp * Y.imag()); Ep[pasadas][1] = (double)bp * Y.real();
                const R q = (((R)2 * pi) * freq) / s.cluz;
                const double hd = std::abs(dft[ii]), hx = std::abs(X), hy = std::abs(Y);
                rcs[pasadas] = (R)((double)(q * q) / ((double)((R)4 * pi) * (hd * hd)) * (hx * hx + hy * hy));
            }
            double* r = out + (size_t)row * 9;
            r[0] = (double)freq; r[1] = (double)theta; r[2] = (double)phi;
            r[3] = std::hypot(Et[2][0], Et[2][1]); r[4] = std::atan2(Et[2][1], Et[2][0]);
            r[5] = std::hypot(Ep[2][0], Ep[2][1]); r[6] = std::atan2(Ep[2][1], Ep[2][0]);
            r[7] = (double)rcs[1]; r[8] = (double)rcs[2];
            ++row;
        }
    }
    return 0;
}

template <class R> int run(Sim<R>& s, int n0, int n1, float* out) {
    const int np = (int)s.probes.size() / 4;
    for (int n = n0; n < n1; ++n) {
        one_step(s, n);
        if (out) {
            // UpdateObservation point probes, observation.F90:2633-2668
            for (int q = 0; q < np; ++q) {
                const int* pr = &s.probes[4 * q];
                out[(long)(n - n0) * np + q] = (float)s.F[pr[0]](pr[1], pr[2], pr[3]);
            }
        }
        for (auto& p : s.fprobes) update_freq_probe(s, p, n);
        for (auto& ff : s.farfields) update_farfield(s, ff, n);
    }
    return 0;
}

// XItrancos / XEtrancos of observation.F90:318-331 (truncating division and
// MOD, as Fortran's INT and MOD).
inline bool trancos(int lo, int hi, int tr, int* first, int* count) {
    if (tr < 1 || hi < lo) return false;
    int a = lo / tr;
    const int b = hi / tr;
    if (lo % tr != 0) a += 1;
    *first = a;
    *count = b - a + 1;
    return *count > 0;
}

template <class R> int add_freq_probe(Sim<R>& s, int mag, const int* box, const int* stride, int nfreq, const float* freq) {
    typename Sim<R>::FreqProbe p;
    p.mag = mag;
    if (!trancos(box[0], box[1], stride[0], &p.i0, &p.ni) || !trancos(box[2], box[3], stride[1], &p.j0, &p.nj) ||
        !trancos(box[4], box[5], stride[2], &p.k0, &p.nk) || nfreq < 1)
        return -1;
    for (int a = 0; a < 3; ++a) p.tr[a] = stride[a];
    p.freq.assign(freq, freq + nfreq);
    p.V.assign((size_t)nfreq * 3 * p.ni * p.nj * p.nk, std::complex<double>(0.0, 0.0));
    s.fprobes.push_back(std::move(p));
    return (int)s.fprobes.size() - 1;
}

template <class R> const A1<R>* metric(Sim<R>& s, int which) {
    const A1<R>* t[18] = {&s.Idxe, &s.Idye, &s.Idze, &s.Idxh, &s.Idyh, &s.Idzh, &s.P_be_x, &s.P_be_y, &s.P_be_z,
                          &s.P_ce_x, &s.P_ce_y, &s.P_ce_z, &s.P_bm_x, &s.P_bm_y, &s.P_bm_z, &s.P_cm_x, &s.P_cm_y, &s.P_cm_z};
    if (which < 0 || which >= 18) return nullptr;
    return t[which];
}

}  // namespace

extern "C" {

int orc_create(const orc_problem* p, int fp64, int nthreads, void** handle) {
    if (!p || !handle) return 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    Handle* h = new Handle();
    h->fp64 = fp64;
    h->nthreads = nthreads;
    int rc = fp64 ? create<double>(p, &h->sd) : create<float>(p, &h->sf);
    if (rc) { delete h; return rc; }
    *handle = h;
    return 0;
}

void orc_destroy(void* hv) {
    Handle* h = (Handle*)hv;
    if (!h) return;
    delete h->sf;
    delete h->sd;
    delete h;
}

int orc_add_freq_probe(void* hv, int magnetic, const int* box, const int* stride, int nfreq, const float* freq) {
    Handle* h = (Handle*)hv;
    if (!h || !box || !stride || !freq || (magnetic != 0 && magnetic != 1)) return -1;
    return h->fp64 ? add_freq_probe(*h->sd, magnetic, box, stride, nfreq, freq)
                   : add_freq_probe(*h->sf, magnetic, box, stride, nfreq, freq);
}

int orc_read_freq_probe(void* hv, int id, int* shape4, double* out) {
    Handle* h = (Handle*)hv;
    auto rd = [&](auto& s) -> int {
        if (id < 0 || id >= (int)s.fprobes.size()) return 1;
        const auto& p = s.fprobes[id];
        if (shape4) {
            shape4[0] = (int)p.freq.size();
            shape4[1] = p.nk;
            shape4[2] = p.nj;
            shape4[3] = p.ni;
        }
        if (out)
            for (size_t q = 0; q < p.V.size(); ++q) {
                out[2 * q] = p.V[q].real();
                out[2 * q + 1] = p.V[q].imag();
            }
        return 0;
    };
    return h->fp64 ? rd(*h->sd) : rd(*h->sf);
}

int orc_add_farfield(void* hv, const int* box, const int* faces, float fi, float ff, float fs, int logarithmic,
                     int decimate) {
    Handle* h = (Handle*)hv;
    if (!h || !box || !faces) return -1;
    return h->fp64 ? add_farfield(*h->sd, box, faces, fi, ff, fs, logarithmic, decimate)
                   : add_farfield(*h->sf, box, faces, fi, ff, fs, logarithmic, decimate);
}

int orc_read_farfield(void* hv, int id, int face, int slot, int* dims, double* out) {
    Handle* h = (Handle*)hv;
    auto rd = [&](auto& s) -> int {
        if (id < 0 || id >= (int)s.farfields.size() || face < 0 || face > 5 || slot < 0 || slot > 5) return 1;
        const auto& F = s.farfields[id];
        if (!F.on[face]) { dims[0] = dims[1] = 0; return 0; }
        const auto& A = F.arr[face][slot];
        dims[0] = std::max(0, A.hi1 - A.lo1 + 1);
        dims[1] = std::max(0, A.hi2 - A.lo2 + 1);
        if (out) std::memcpy(out, A.v.data(), A.v.size() * sizeof(std::complex<double>));
        return 0;
    };
    if (!h || !dims) return 1;
    return h->fp64 ? rd(*h->sd) : rd(*h->sf);
}

int orc_farfield_transform(void* hv, int id, const float* angles, const float* incident, int n_incident, double* out,
                           int max_rows, int* rows) {
    Handle* h = (Handle*)hv;
    if (!h || !angles || !rows) return 1;
    return h->fp64 ? farfield_transform(*h->sd, id, angles, incident, n_incident, out, max_rows, rows)
                   : farfield_transform(*h->sf, id, angles, incident, n_incident, out, max_rows, rows);
}

int orc_store_resume(void* hv, const char* path, int last_step) {
    Handle* h = (Handle*)hv;
    int n = last_step;
    return h->fp64 ? resume_io(*h->sd, path, true, &n) : resume_io(*h->sf, path, true, &n);
}

int orc_load_resume(void* hv, const char* path, int* last_step) {
    Handle* h = (Handle*)hv;
    int n = 0;
    int rc = h->fp64 ? resume_io(*h->sd, path, false, &n) : resume_io(*h->sf, path, false, &n);
    if (!rc && last_step) *last_step = n;
    return rc;
}

void orc_set_threads(void* hv, int nthreads) { ((Handle*)hv)->nthreads = nthreads; }

int orc_run(void* hv, int n0, int n1, float* out) {
    Handle* h = (Handle*)hv;
#ifdef _OPENMP
    if (h->nthreads > 0) omp_set_num_threads(h->nthreads);
#endif
    return h->fp64 ? run(*h->sd, n0, n1, out) : run(*h->sf, n0, n1, out);
}

int orc_get_lims(void* hv, orc_lim* a, orc_lim* w, orc_lim* q) {
    Handle* h = (Handle*)hv;
    for (int f = 0; f < 6; ++f) {
        const Lim& A = h->fp64 ? h->sd->Alloc[f] : h->sf->Alloc[f];
        const Lim& W = h->fp64 ? h->sd->Sweep[f] : h->sf->Sweep[f];
        const Lim& Q = h->fp64 ? h->sd->SINPML[f] : h->sf->SINPML[f];
        a[f] = orc_lim{A.XI, A.XE, A.YI, A.YE, A.ZI, A.ZE};
        w[f] = orc_lim{W.XI, W.XE, W.YI, W.YE, W.ZI, W.ZE};
        q[f] = orc_lim{Q.XI, Q.XE, Q.YI, Q.YE, Q.ZI, Q.ZE};
    }
    return 0;
}

double orc_get_dt(void* hv) {
    Handle* h = (Handle*)hv;
    return h->fp64 ? h->sd->dt : h->sf->dt;
}

double orc_get_time(void* hv, int n) {
    Handle* h = (Handle*)hv;
    return h->fp64 ? h->sd->time(n) : h->sf->time(n);
}

int orc_get_num_media(void* hv) {
    Handle* h = (Handle*)hv;
    return h->fp64 ? h->sd->NumMedia : h->sf->NumMedia;
}

int orc_get_field(void* hv, int comp, float* out) {
    Handle* h = (Handle*)hv;
    if (comp < 0 || comp > 5) return 1;
    if (h->fp64) {
        const auto& v = h->sd->F[comp].v;
        for (size_t i = 0; i < v.size(); ++i) out[i] = (float)v[i];
    } else {
        const auto& v = h->sf->F[comp].v;
        std::memcpy(out, v.data(), v.size() * sizeof(float));
    }
    return 0;
}

int orc_set_field(void* hv, int comp, const float* in) {
    Handle* h = (Handle*)hv;
    if (comp < 0 || comp > 5) return 1;
    if (h->fp64) {
        auto& v = h->sd->F[comp].v;
        for (size_t i = 0; i < v.size(); ++i) v[i] = in[i];
    } else {
        auto& v = h->sf->F[comp].v;
        std::memcpy(v.data(), in, v.size() * sizeof(float));
    }
    return 0;
}

int orc_get_field_f64(void* hv, int comp, double* out) {
    Handle* h = (Handle*)hv;
    if (comp < 0 || comp > 5) return 1;
    if (h->fp64) {
        const auto& v = h->sd->F[comp].v;
        std::memcpy(out, v.data(), v.size() * sizeof(double));
    } else {
        const auto& v = h->sf->F[comp].v;
        for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    }
    return 0;
}

int orc_get_media(void* hv, int comp, short* out) {
    Handle* h = (Handle*)hv;
    if (comp < 0 || comp > 5) return 1;
    const auto& v = h->fp64 ? h->sd->mi[comp].v : h->sf->mi[comp].v;
    std::memcpy(out, v.data(), v.size() * sizeof(short));
    return 0;
}

int orc_get_g(void* hv, float* g1, float* g2, float* gm1, float* gm2) {
    Handle* h = (Handle*)hv;
    int n = orc_get_num_media(hv) + 1;
    for (int i = 0; i < n; ++i) {
        if (h->fp64) {
            g1[i] = (float)h->sd->G1[i]; g2[i] = (float)h->sd->G2[i];
            gm1[i] = (float)h->sd->GM1[i]; gm2[i] = (float)h->sd->GM2[i];
        } else {
            g1[i] = h->sf->G1[i]; g2[i] = h->sf->G2[i];
            gm1[i] = h->sf->GM1[i]; gm2[i] = h->sf->GM2[i];
        }
    }
    return 0;
}

int orc_get_metric_range(void* hv, int which, int* lo, int* hi) {
    Handle* h = (Handle*)hv;
    if (h->fp64) {
        const A1<double>* a = metric(*h->sd, which);
        if (!a) return 1;
        *lo = a->lo; *hi = a->hi;
    } else {
        const A1<float>* a = metric(*h->sf, which);
        if (!a) return 1;
        *lo = a->lo; *hi = a->hi;
    }
    return 0;
}

int orc_get_metric(void* hv, int which, float* out) {
    Handle* h = (Handle*)hv;
    if (h->fp64) {
        const A1<double>* a = metric(*h->sd, which);
        if (!a) return 1;
        for (size_t i = 0; i < a->v.size(); ++i) out[i] = (float)a->v[i];
    } else {
        const A1<float>* a = metric(*h->sf, which);
        if (!a) return 1;
        std::memcpy(out, a->v.data(), a->v.size() * sizeof(float));
    }
    return 0;
}

long orc_check_div_dt(double dt, long n, unsigned long long seed) {
    const double y = 1.0 / dt;
    unsigned long long x = seed ? seed : 0x9E3779B97F4A7C15ull;
    long bad = 0;
    for (long i = 0; i < n; ++i) {
        // xorshift64*: sign, a mantissa and an exponent keeping a/dt normal
        x ^= x >> 12; x ^= x << 25; x ^= x >> 27;
        const unsigned long long r = x * 2685821657736338717ull;
        const int e = (int)((r >> 52) % 1200) - 600;
        double a = std::ldexp(1.0 + (double)(r & ((1ull << 52) - 1)) / 4503599627370496.0, e);
        if (r & (1ull << 63)) a = -a;
        const double q0 = a * y;
        const double rr = std::fma(-q0, dt, a);
        const double q = std::fma(rr, y, q0);
        if (q != a / dt) ++bad;
    }
    return bad;
}

// Incid with calledfromobservation (observation.F90:3826-3875 ->
// planewaves.F90:778-853): the sum over every plane wave of
// fpw(comp) * evolucion at the node's PhysCoor, with a dummy switch.
int orc_incident(void* hv, int comp, int i, int j, int k, int nt, const float* t, float* out) {
    Handle* h = (Handle*)hv;
    if (h->fp64 || comp < 0 || comp > 5) return 1;
    Sim<float>& s = *h->sf;
    const int ijk[3] = {i, j, k};
    for (int a = 0; a < 3; ++a)
        if (!s.pws.empty() && (ijk[a] < s.phys_lo[comp][a] || ijk[a] - s.phys_lo[comp][a] >= (int)s.phys[comp][a].size()))
            return 1;
    for (int q = 0; q < nt; ++q) {
        float ehi = 0.0f;
        for (const PlaneWave<float>& pw : s.pws) {
            const float xf = s.physc(comp, 0, i), yf = s.physc(comp, 1, j), zf = s.physc(comp, 2, k);
            const float d = (xf * pw.px + yf * pw.py + zf * pw.pz) - pw.d0;
            float ev = 0.0f;
            const long long nprev = (long long)((t[q] - d / s.cluz) / pw.deltaevol);
            if (nprev + 1 <= pw.numus && nprev > 0)
                ev = (pw.evol[nprev + 1] - pw.evol[nprev]) / pw.deltaevol * ((t[q] - d / s.cluz) - (float)nprev * pw.deltaevol) +
                     pw.evol[nprev];
            ehi = ehi + pw.fpw[comp] * ev;
        }
        out[q] = ehi;
    }
    return 0;
}

int orc_get_mur_cab1(void* hv, int face, float* out) {
    Handle* h = (Handle*)hv;
    if (face < 0 || face > 5) return 1;
    // face order back, front, left, right, down, up -> region Back..Up
    const int reg[6] = {Back, Front, Left, Right, Down, Up};
    auto get = [&](auto& s) {
        const int r = reg[face];
        if (!s.isMur[kRegAxis[r]][kRegSide[r]]) return 1;
        for (size_t m = 0; m < s.CAB1[r].size(); ++m) out[m] = (float)s.CAB1[r][m];
        return 0;
    };
    return h->fp64 ? get(*h->sd) : get(*h->sf);
}

static int get_disp(void* hv, bool mag, int m, int* medium_index, int* npoles, double* kappa, double* beta, double* g3) {
    Handle* h = (Handle*)hv;
    auto fill = [&](auto& s) {
        auto& list = mag ? s.mdut : s.dut;
        if (m < 0 || m >= (int)list.size()) return 1;
        auto& d = list[m];
        *medium_index = d.indexmed;
        *npoles = d.np;
        for (int q = 0; q < d.np; ++q) {
            if (kappa) { kappa[2 * q] = d.kappa[q].re; kappa[2 * q + 1] = d.kappa[q].im; }
            if (beta) { beta[2 * q] = d.beta[q].re; beta[2 * q + 1] = d.beta[q].im; }
            if (g3) { g3[2 * q] = d.g3[q].re; g3[2 * q + 1] = d.g3[q].im; }
        }
        return 0;
    };
    return h->fp64 ? fill(*h->sd) : fill(*h->sf);
}

int orc_get_edisp(void* hv, int m, int* medium_index, int* npoles, double* kappa, double* beta, double* g3) {
    return get_disp(hv, false, m, medium_index, npoles, kappa, beta, g3);
}

int orc_get_mdisp(void* hv, int m, int* medium_index, int* npoles, double* kappa, double* beta, double* g3) {
    return get_disp(hv, true, m, medium_index, npoles, kappa, beta, g3);
}

}  // extern "C"
