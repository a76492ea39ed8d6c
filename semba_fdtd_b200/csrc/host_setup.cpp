// Level-2 host of libsemba_gpu: builds, from an NFDE-style problem, the arrays
// the reference's set-up produces (grid limits, time step, media table and
// matrices, update coefficients, metrics, CPML, ADE, plane-wave and nodal
// tables), then hands them to the level-1 entry points.  It plays the role
// of semba_fdtd.F90:1197-1300 (NFDE2sgg) and timestepping.F90:305-1014
// (launch_simulation up to the time loop) for callers without the Fortran
// host.  FP32 quantities are float, sgg%dt and the time vector double, the
// ADE coefficients complex(8) computed with gfortran's Fortran-rules complex
// arithmetic (plain product, Smith quotient).  Compiled without FMA
// contraction so each operation rounds where the reference rounds.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "sgpu_internal.h"

namespace {

enum { EX = 0, EY, EZ, HX, HY, HZ };

// semba_fdtd.F90:154-155: default-real literals, i.e. rounded to FP32.
const float kEps0 = 8.8541878176203898505365630317107502606083701665994498081024171524053950954599821142852891607182008932e-12f;
const float kMu0 = 1.2566370614359172953850573533118011536788677597500423283899778369231265625144835994512139301368468271e-6f;
// fdetypes.F90:675-703
const int kPrioBackground = 10, kPrioBody = 20, kPrioDispersive = 40, kPrioPec = 150;

struct Box { int x0, x1, y0, y1, z0, z1; };

// 1-D array with an arbitrary lower bound.
struct Vec {
    int lo = 0;
    std::vector<float> v;
    void init(int l, int h, float x) { lo = l; v.assign(std::max(0, h - l + 1), x); }
    int hi() const { return lo + (int)v.size() - 1; }
    float& operator[](int i) { return v[i - lo]; }
    float operator[](int i) const { return v[i - lo]; }
};

// Planes of an nx x ny box that make about 64 Ki cells: the smallest share
// of a plane loop one set-up thread takes.  Grids under 16 Mi cells are set
// up on the calling thread alone (their plans are usually made many at a
// time, one per thread).
constexpr long long kThreadedCells = 1LL << 24;
long long plane_grain(long long grid_cells, long long nx, long long ny) {
    if (grid_cells < kThreadedCells) return 1LL << 40;
    return std::max(1LL, (1LL << 16) / std::max(1LL, nx * ny));
}

// int16 media matrix over one component's Alloc, column-major (filled with
// medium 1 by several threads on large grids).
struct MediaMat {
    Box b;
    long long nx = 0, ny = 0;
    size_t n = 0;
    std::unique_ptr<int16_t[]> v;
    void init(const Box& bb) {
        b = bb;
        nx = b.x1 - b.x0 + 1;
        ny = b.y1 - b.y0 + 1;
        n = (size_t)nx * ny * (b.z1 - b.z0 + 1);
        v.reset(new int16_t[n]);
        int16_t* p = v.get();
        sgpu::host_parallel((long long)n, [p](long long a, long long e) { std::fill(p + a, p + e, (int16_t)1); }, 1 << 20);
    }
    int16_t& at(int i, int j, int k) { return v[(i - b.x0) + nx * ((j - b.y0) + ny * (long long)(k - b.z0))]; }
    int16_t* data() const { return v.get(); }
    size_t size() const { return n; }
    bool empty() const { return n == 0; }
    void release() {
        v.reset();
        n = 0;
    }
};

struct Med {
    float epr = 1, sigma = 0, mur = 1, sigmam = 0;
    int prio = kPrioBackground;
    bool pec = false, disp = false, mdisp = false, inert = false;
    int region = -1;
};

struct Cx { double r, i; };
Cx cx_mul(Cx a, Cx b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
// Smith's algorithm, the quotient gfortran emits for complex(8) division.
Cx cx_div(Cx a, Cx b) {
    if (std::fabs(b.r) < std::fabs(b.i)) {
        double t = b.r / b.i, den = (b.r * t) + b.i;
        return {((a.r * t) + a.i) / den, ((a.i * t) - a.r) / den};
    }
    double t = b.i / b.r, den = (b.i * t) + b.r;
    return {((a.i * t) + a.r) / den, (a.i - (a.r * t)) / den};
}

struct HostState {
    Box sinpml[6], full[6], alloc[6], sweep[6];
    // border kind per [axis][side] (tipofrontera codes) and the Mur flags
    int kind[3][2];
    bool mur[3][2];
    std::vector<float> cab1[6];  // calc_murconstants, face order back..up
    int layers[3][2];
    float order[3][2], refl[3][2];
    Vec dx, dy, dz, lx, ly, lz;
    float eps0, mu0, cluz, zvac;
    double dt;
    std::vector<Med> med;
    int num_media = 0;
    MediaMat mm[6];
    std::vector<float> g1, g2, gm1, gm2;
    Vec dxe, dye, dze, dxh, dyh, dzh;
    Vec idxe, idye, idze, idxh, idyh, idzh;
    Vec pbe[3], pce[3], pbm[3], pcm[3];
    // descriptors for the level-1 calls (pointers refer to the vectors here)
    sgpu_cpml_desc cd{};
    std::vector<int> didx, dnp, mdidx, mdnp;      // electric / magnetic pole-residue media
    std::vector<double> dK, dB, dG, mdK, mdB, mdG;
    std::vector<uint8_t> pec;
    std::vector<float> phys[6][3];
    int phys_lo[6][3];
    std::vector<std::vector<float>> samples;
    std::vector<sgpu_planewave_desc> pw;
    std::vector<sgpu_nodal_desc> nodal;
    std::vector<int> probes;
    int probe_cap = 1024;
    int max_steps = 0;
    // media matrices built on the device (sgpu_host_create): the regions to
    // paint, in painting order, instead of host matrices
    bool device_media = false;
    struct PaintRegion {
        int idx, prio;
        std::vector<Box> boxes;
    };
    std::vector<PaintRegion> paint_regions;
};

void free_host(void* p) { delete (HostState*)p; }

Box to_box(const sgpu_lim& l) { return Box{l.xi, l.xe, l.yi, l.ye, l.zi, l.ze}; }
sgpu_lim to_lim(const Box& b) { return sgpu_lim{b.x0, b.x1, b.y0, b.y1, b.z0, b.z1}; }

// read_limits_nogeom (preprocess_geom.F90:5266-5737) and the Alloc/Sweep
// rule of NFDE2sgg for a single layout (semba_fdtd.F90:1285-1300).
void limits(HostState& h, const sgpu_problem* p) {
    // reference face order back, front, left, right, down, up; only CPML
    // faces carry layers, order and reflection (sgg%PML starts zeroed,
    // preprocess_geom.F90:5398-5600)
    for (int f = 0; f < 6; ++f) {
        int ax = f / 2, sd = f % 2;
        const int kind = p->border[f] == 0 ? 9 : p->border[f];
        const bool pml = kind == 9;
        h.kind[ax][sd] = kind;
        h.mur[ax][sd] = kind == 7 || (pml && p->mur_after_pml);
        h.layers[ax][sd] = pml ? p->pml_layers[f] : 0;
        float r = pml ? p->pml_refl[f] : 0.0f;
        h.refl[ax][sd] = r >= 1.0f ? (float)0.99999 : r;
        h.order[ax][sd] = pml ? p->pml_order[f] : 0.0f;
    }
    const int N[3] = {p->nx, p->ny, p->nz};
    // components whose SINPML range is one node shorter along an axis
    const int shorter[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 0}};
    for (int f = 0; f < 6; ++f) {
        int hi[3];
        for (int a = 0; a < 3; ++a) hi[a] = N[a] - shorter[f][a];
        h.sinpml[f] = Box{0, hi[0], 0, hi[1], 0, hi[2]};
        h.full[f] = Box{-h.layers[0][0], hi[0] + h.layers[0][1], -h.layers[1][0], hi[1] + h.layers[1][1],
                        -h.layers[2][0], hi[2] + h.layers[2][1]};
        const Box& q = h.full[f];
        h.alloc[f] = Box{q.x0 - 1, q.x1 + 1, q.y0 - 1, q.y1 + 1, q.z0 - 1, q.z1 + 1};
        h.sweep[f] = q;
    }
    const float* des[3] = {p->desx, p->desy, p->desz};
    const float org[3] = {p->originx, p->originy, p->originz};
    Vec* D[3] = {&h.dx, &h.dy, &h.dz};
    Vec* Ln[3] = {&h.lx, &h.ly, &h.lz};
    for (int a = 0; a < 3; ++a) {
        const int n = N[a], L0 = h.layers[a][0], L1 = h.layers[a][1];
        Vec& d = *D[a];
        d.init(-L0 - 2, n + L1 + 2, 0.0f);
        for (int i = 0; i < n; ++i) d[i] = des[a][i];
        for (int i = -1; i >= -L0 - 2; --i) d[i] = d[0];
        for (int i = n; i <= n + L1 + 2; ++i) d[i] = d[n - 1];
        Vec& l = *Ln[a];
        l.init(-L0 - 1, n + L1 + 1, 0.0f);
        l[0] = org[a] + 0.0f * des[a][n > 1 ? 1 : 0];
        for (int i = 0; i < n; ++i) l[i + 1] = des[a][i] + l[i];
        float lo_step = l[1] - l[0];
        for (int i = -1; i >= -L0 - 1; --i) l[i] = l[i + 1] - lo_step;
        float hi_step = l[n] - l[n - 1];
        for (int i = n + 1; i <= n + L1 + 1; ++i) l[i] = l[i - 1] + hi_step;
    }
}

// Time step of NFDE2sgg (semba_fdtd.F90:1208-1257).
void timestep(HostState& h, const sgpu_problem* p) {
    h.eps0 = kEps0;
    h.mu0 = kMu0;
    h.cluz = 1.0f / std::sqrt(h.eps0 * h.mu0);
    h.zvac = std::sqrt(h.mu0 / h.eps0);
    float mins[3];
    const Vec* D[3] = {&h.dx, &h.dy, &h.dz};
    for (int a = 0; a < 3; ++a) mins[a] = *std::min_element(D[a]->v.begin(), D[a]->v.end());
    float r0 = 1.0f / mins[0], r1 = 1.0f / mins[1], r2 = 1.0f / mins[2];
    float courant = 1.0f / (h.cluz * std::sqrt(r0 * r0 + r1 * r1 + r2 * r2));
    double dt = p->dt;
    if (dt < std::fabs((double)(std::numeric_limits<float>::min() * 2.0f)))
        dt = (double)(std::numeric_limits<float>::max() / 2.0f);
    if (p->forcecfl) dt = (double)(courant * p->cfl);
    else if (dt > (double)(courant * 0.8f)) dt = (double)(courant * 0.8f);
    h.dt = dt;
}

// The cells CreateVolumeMM (healer.F90:66-243) paints for cell box pt, per
// component: from the box's lower corner (clipped to the H Alloc ranges) to
// its upper corner, one further on the axes along which the component sits
// on voxel edges or faces (clipped likewise).  Empty boxes have hi < lo.
void paint_ranges(const HostState& h, const Box& pt, Box out[6]) {
    const Box bb{h.alloc[HX].x0, h.alloc[HX].x1, h.alloc[HY].y0, h.alloc[HY].y1, h.alloc[HZ].z0, h.alloc[HZ].z1};
    const int x0 = std::max(pt.x0, bb.x0), y0 = std::max(pt.y0, bb.y0), z0 = std::max(pt.z0, bb.z0);
    const int x1 = std::min(pt.x1, bb.x1 - 1), y1 = std::min(pt.y1, bb.y1 - 1), z1 = std::min(pt.z1, bb.z1 - 1);
    const int X1 = std::min(pt.x1 + 1, bb.x1), Y1 = std::min(pt.y1 + 1, bb.y1), Z1 = std::min(pt.z1 + 1, bb.z1);
    // per component: upper bounds along x, y, z (edge components reach +1)
    const int up[6][3] = {{x1, Y1, Z1}, {X1, y1, Z1}, {X1, Y1, z1}, {X1, y1, z1}, {x1, Y1, z1}, {x1, y1, Z1}};
    for (int f = 0; f < 6; ++f) out[f] = Box{x0, up[f][0], y0, up[f][1], z0, up[f][2]};
}

// CreateVolumeMM (healer.F90:66-243): E nodes on the voxel edges take the
// medium when its priority is higher, H nodes on the faces when it is not
// lower.
void paint(HostState& h, const Box& pt, int idx) {
    Box rg[6];
    paint_ranges(h, pt, rg);
    const int pr = h.med[idx].prio;
    for (int f = 0; f < 6; ++f) {
        MediaMat& m = h.mm[f];
        const bool electric = f < 3;
        const int x0 = rg[f].x0, y0 = rg[f].y0, z0 = rg[f].z0;
        const int up[3] = {rg[f].x1, rg[f].y1, rg[f].z1};
        const int nk = up[2] - z0 + 1;
        if (nk <= 0 || up[1] < y0 || up[0] < x0) continue;
        sgpu::host_parallel(nk, [&](long long a, long long e) {
            for (int k = z0 + (int)a; k < z0 + (int)e; ++k)
                for (int j = y0; j <= up[1]; ++j)
                    for (int i = x0; i <= up[0]; ++i) {
                        int16_t& cell = m.at(i, j, k);
                        const int cur = h.med[cell].prio;
                        if (electric ? pr > cur : pr >= cur) cell = (int16_t)idx;
                    }
        }, plane_grain(h.mm[0].size(), up[0] - x0 + 1, up[1] - y0 + 1));
    }
}

// healer.F90:44-50, as [comp][axis] for the lower (in) and upper (on) side
const int kInLo[6][3] = {{0, 1, 1}, {1, 0, 1}, {1, 1, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
const int kOnHi[6][3] = {{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {0, -1, -1}, {-1, 0, -1}, {-1, -1, 0}};

// The boxes of CreatePMLmatrix: the outer (H Alloc) box, the inner box
// inside the PML, and per component the reach its extrusion covers.
struct PmlGeom {
    Box outer, inner, reach[6];
};
PmlGeom pml_geom(const HostState& h) {
    PmlGeom g;
    g.outer = Box{h.alloc[HX].x0, h.alloc[HX].x1, h.alloc[HY].y0, h.alloc[HY].y1, h.alloc[HZ].z0, h.alloc[HZ].z1};
    const Box& outer = g.outer;
    g.inner = Box{std::max(outer.x0, h.sinpml[HX].x0), std::min(outer.x1, h.sinpml[HX].x1),
                  std::max(outer.y0, h.sinpml[HY].y0), std::min(outer.y1, h.sinpml[HY].y1),
                  std::max(outer.z0, h.sinpml[HZ].z0), std::min(outer.z1, h.sinpml[HZ].z1)};
    for (int f = 0; f < 6; ++f)
        g.reach[f] = Box{std::max(outer.x0, h.full[HX].x0), std::min(outer.x1 + kOnHi[f][0], h.full[HX].x1),
                         std::max(outer.y0, h.full[HY].y0), std::min(outer.y1 + kOnHi[f][1], h.full[HY].y1),
                         std::max(outer.z0, h.full[HZ].z0), std::min(outer.z1 + kOnHi[f][2], h.full[HZ].z1)};
    return g;
}

// Media copies for the PML (the renumbering of CreatePMLmatrix): the media
// whose negated entries the shell holds, ordered by first appearance in the
// sweep (components in order, then k, j, i), become media num_media+1, ...;
// copy_of maps a medium to its copy.  first[v] < 0: v does not appear.
void pml_copies(HostState& h, const std::vector<long long>& first, std::vector<int>& copy_of) {
    std::vector<int> order;
    for (int v = 1; v <= h.num_media; ++v)
        if (first[v] >= 0) order.push_back(v);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return first[a] < first[b]; });
    copy_of.assign(h.num_media + 1, 0);
    int next = h.num_media;
    h.med.resize(h.num_media + 1 + order.size());
    for (int v : order) {
        copy_of[v] = ++next;
        h.med[next] = h.med[v];
    }
    h.num_media = next;
}

// PEC borders (healer.F90:1442-1617): medium 0 on the boundary plane of the
// E components tangential to a PEC face and the H component normal to it;
// fn(component, plane box) for each.
template <class Fn> void pec_planes(const HostState& h, const PmlGeom& g, Fn&& fn) {
    for (int f = 0; f < 6; ++f) {
        const bool elec = f < 3;
        const int own = f % 3;
        for (int a = 0; a < 3; ++a)
            for (int sd = 0; sd < 2; ++sd) {
                if (h.kind[a][sd] != 1 || (elec ? a == own : a != own)) continue;
                const Box& r = g.reach[f];
                int lo[3] = {r.x0, r.y0, r.z0}, hi[3] = {r.x1, r.y1, r.z1};
                lo[a] = hi[a] = sd == 0 ? lo[a] : hi[a];
                fn(f, Box{lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]});
            }
    }
}

// CreatePMLmatrix (healer.F90:961-1420): media reaching the PML interface
// are extruded across the PML and renumbered as new copies.
void pml_media(HostState& h) {
    const int (&in_lo)[6][3] = kInLo;
    const PmlGeom geom = pml_geom(h);
    const Box& outer = geom.outer;
    const Box& inner = geom.inner;
    const Box* reach = geom.reach;
    auto neg = [](int16_t v) { return (int16_t)(-std::abs((int)v)); };
    // the three extrusions in order; within each, planes are independent
    for (int f = 0; f < 6; ++f) {
        MediaMat& m = h.mm[f];
        const Box& r = reach[f];
        const int lo_src[3] = {inner.x0, inner.y0, inner.z0};
        const int hi_src[3] = {inner.x1 + in_lo[f][0] - 1, inner.y1 + in_lo[f][1] - 1, inner.z1 + in_lo[f][2] - 1};
        const long long grain = plane_grain(h.mm[0].size(), r.x1 - r.x0 + 1, r.y1 - r.y0 + 1);
        auto planes = [&](int k0, int k1, auto&& fn) {
            if (k1 >= k0) sgpu::host_parallel(k1 - k0 + 1, [&](long long a, long long e) {
                for (int k = k0 + (int)a; k < k0 + (int)e; ++k) fn(k);
            }, grain);
        };
        // along x (rows are contiguous: k, then j, then the two i ranges)
        planes(r.z0, r.z1, [&](int k) {
            for (int j = r.y0; j <= r.y1; ++j) {
                int16_t* row = &m.at(r.x0, j, k) - r.x0;  // row[i] is cell (i, j, k)
                const int16_t lo = neg(row[lo_src[0]]), hi = neg(row[hi_src[0]]);
                for (int i = r.x0; i <= inner.x0 - 1; ++i) row[i] = lo;
                for (int i = inner.x1 + in_lo[f][0]; i <= r.x1; ++i) row[i] = hi;
            }
        });
        // along y, over the whole x reach (edges): whole rows copied
        auto copy_row = [&](int16_t* dst, const int16_t* src) {
            for (int i = r.x0; i <= r.x1; ++i) dst[i] = neg(src[i]);
        };
        planes(r.z0, r.z1, [&](int k) {
            const int16_t* slo = &m.at(r.x0, lo_src[1], k) - r.x0;
            const int16_t* shi = &m.at(r.x0, hi_src[1], k) - r.x0;
            for (int j = r.y0; j <= inner.y0 - 1; ++j) copy_row(&m.at(r.x0, j, k) - r.x0, slo);
            for (int j = inner.y1 + in_lo[f][1]; j <= r.y1; ++j) copy_row(&m.at(r.x0, j, k) - r.x0, shi);
        });
        // along z, over the whole x and y reach (corners): whole planes copied
        planes(r.z0, inner.z0 - 1, [&](int k) {
            for (int j = r.y0; j <= r.y1; ++j) copy_row(&m.at(r.x0, j, k) - r.x0, &m.at(r.x0, j, lo_src[2]) - r.x0);
        });
        planes(inner.z1 + in_lo[f][2], r.z1, [&](int k) {
            for (int j = r.y0; j <= r.y1; ++j) copy_row(&m.at(r.x0, j, k) - r.x0, &m.at(r.x0, j, hi_src[2]) - r.x0);
        });
    }
    // Only the extruded shell can hold negative (to be copied) entries.  A
    // full sweep (components in order, then k, j, i) numbers the copies in
    // order of first appearance; here every plane of the shell is scanned
    // in parallel for the first position of each entry, and the copies are
    // numbered by those positions.
    struct Task {
        int f, k;
    };
    std::vector<Task> tasks;
    for (int f = 0; f < 6; ++f)
        for (int k = reach[f].z0; k <= reach[f].z1; ++k) tasks.push_back(Task{f, k});
    auto shell_row_spans = [&](const Task& t, auto&& fn) {
        MediaMat& m = h.mm[t.f];
        const Box& r = reach[t.f];
        const int xa = inner.x0, xb = inner.x1 + in_lo[t.f][0] - 1;
        const int ya = inner.y0, yb = inner.y1 + in_lo[t.f][1] - 1;
        const int za = inner.z0, zb = inner.z1 + in_lo[t.f][2] - 1;
        for (int j = r.y0; j <= r.y1; ++j) {
            int16_t* row = &m.at(r.x0, j, t.k) - r.x0;
            if (t.k < za || t.k > zb || j < ya || j > yb) {
                fn(row, j - r.y0, r.x0, r.x1, r.x0);
            } else {
                fn(row, j - r.y0, r.x0, std::min(r.x1, xa - 1), r.x0);
                fn(row, j - r.y0, std::max(r.x0, xb + 1), r.x1, r.x0);
            }
        }
    };
    const long long kNone = std::numeric_limits<long long>::max();
    std::vector<long long> first(h.num_media + 1, kNone);
    std::mutex mu;
    const long long row_cells = (long long)(outer.x1 - outer.x0 + 1) * (outer.y1 - outer.y0 + 1);
    sgpu::host_parallel((long long)tasks.size(), [&](long long a, long long e) {
        std::vector<long long> mine(h.num_media + 1, kNone);
        for (long long q = a; q < e; ++q)
            shell_row_spans(tasks[q], [&](const int16_t* row, int jr, int i0, int i1, int x0) {
                for (int i = i0; i <= i1; ++i) {
                    const int v = row[i];
                    if (v < 0) {
                        const long long key = (q * (outer.y1 - outer.y0 + 1) + jr) * (outer.x1 - outer.x0 + 1) + (i - x0);
                        if (key < mine[-v]) mine[-v] = key;
                    }
                }
            });
        std::lock_guard<std::mutex> g(mu);
        for (size_t v = 0; v < mine.size(); ++v) first[v] = std::min(first[v], mine[v]);
    }, plane_grain(h.mm[0].size(), row_cells, 1));
    std::vector<long long> firsts(h.num_media + 1, -1);
    for (int v = 1; v <= h.num_media; ++v)
        if (first[v] != kNone) firsts[v] = first[v];
    std::vector<int> copy_of;
    pml_copies(h, firsts, copy_of);
    sgpu::host_parallel((long long)tasks.size(), [&](long long a, long long e) {
        for (long long q = a; q < e; ++q)
            shell_row_spans(tasks[q], [&](int16_t* row, int, int i0, int i1, int) {
                for (int i = i0; i <= i1; ++i)
                    if (row[i] < 0) row[i] = (int16_t)copy_of[-row[i]];
            });
    }, plane_grain(h.mm[0].size(), row_cells, 1));
    pec_planes(h, geom, [&](int f, const Box& b) {
        MediaMat& m = h.mm[f];
        for (int k = b.z0; k <= b.z1; ++k)
            for (int j = b.y0; j <= b.y1; ++j)
                for (int i = b.x0; i <= b.x1; ++i) m.at(i, j, k) = 0;
    });
}

// Media table and matrices of read_geomData (preprocess_geom.F90:421-760,
// 1085-1110): PEC volumes use medium 0, then one medium per dielectric
// region, then one per pole-residue region.
void media(HostState& h, const sgpu_problem* p) {
    h.med.assign(4, Med());
    h.med[0].pec = true;
    h.med[0].prio = kPrioPec;
    h.med[0].sigma = 1.0e29f;
    h.med[0].epr = kEps0 / h.eps0;
    h.med[0].mur = kMu0 / h.mu0;
    h.med[1].epr = kEps0 / h.eps0;
    h.med[1].mur = kMu0 / h.mu0;
    h.med[2].inert = true;  // conformal placeholder
    h.med[3].inert = true;  // split placeholder
    if (!h.device_media)
        for (int f = 0; f < 6; ++f) h.mm[f].init(h.alloc[f]);
    auto regions_of = [&](int kind, auto&& fn) {
        for (int r = 0; r < p->nregions; ++r)
            if (p->regions[r].kind == kind) fn(r, p->regions[r]);
    };
    auto paint_all = [&](const sgpu_region& g, int idx) {
        if (h.device_media) {
            HostState::PaintRegion pr{idx, h.med[idx].prio, {}};
            for (int b = 0; b < g.nboxes; ++b) {
                const int* q = g.boxes + 6 * b;
                pr.boxes.push_back(Box{q[0], q[1], q[2], q[3], q[4], q[5]});
            }
            h.paint_regions.push_back(std::move(pr));
            return;
        }
        for (int b = 0; b < g.nboxes; ++b) {
            const int* q = g.boxes + 6 * b;
            paint(h, Box{q[0], q[1], q[2], q[3], q[4], q[5]}, idx);
        }
    };
    regions_of(0, [&](int, const sgpu_region& g) { paint_all(g, 0); });
    int n = 3;
    regions_of(1, [&](int r, const sgpu_region& g) {
        Med m;
        m.prio = kPrioBody;
        m.epr = g.eps / h.eps0;
        m.sigma = g.sigma;
        m.mur = g.mu / h.mu0;
        m.sigmam = g.sigmam;
        m.region = r;
        h.med.push_back(m);
        paint_all(g, ++n);
    });
    regions_of(2, [&](int r, const sgpu_region& g) {
        Med m;
        m.prio = kPrioDispersive;
        m.epr = g.eps / h.eps0;
        m.sigma = g.sigma;
        m.mur = g.mu / h.mu0;
        m.sigmam = g.sigmam;
        m.disp = g.npoles != 0;
        m.mdisp = g.mpoles != 0;
        m.region = r;
        h.med.push_back(m);
        paint_all(g, ++n);
    });
    h.num_media = n;
    if (!h.device_media) pml_media(h);
}

// calc_G1G2Gm1Gm2 (calc_constants.F90:36-148), branches reachable here.
void coefficients(HostState& h) {
    const int n1 = h.num_media + 1;
    h.g1.assign(n1, 0); h.g2.assign(n1, 0); h.gm1.assign(n1, 0); h.gm2.assign(n1, 0);
    const double dt = h.dt;
    auto lossy = [dt](float sig, float eps, float& a, float& b) {
        double x = ((double)sig * dt) / (double)(2.0f * eps);
        a = (float)((1.0 - x) / (1.0 + x));
        b = (float)((dt / (double)eps) / (1.0 + x));
        if (a < 0.0f) {
            a = (float)std::exp(-(((double)sig * dt) / (double)eps));
            b = (1.0f - a) / sig;
        }
    };
    for (int r = 0; r < n1; ++r) {
        const Med& m = h.med[r];
        const float eps = h.eps0 * m.epr, mu = h.mu0 * m.mur;
        if (m.inert) {
            h.g1[r] = 1; h.g2[r] = 0; h.gm1[r] = 1; h.gm2[r] = 0;
        } else if (m.pec || r == 0) {
            h.g1[r] = h.g2[r] = h.gm1[r] = h.gm2[r] = 0;
        } else if (m.disp && !m.mdisp) {
            lossy(m.sigmam, mu, h.gm1[r], h.gm2[r]);  // G1/G2 come from the electric ADE set-up
        } else if (m.mdisp && !m.disp) {
            lossy(m.sigma, eps, h.g1[r], h.g2[r]);    // GM1/GM2 come from the magnetic ADE set-up
        } else {
            // also a medium with both kinds of poles: both ADE set-ups
            // overwrite these values
            lossy(m.sigma, eps, h.g1[r], h.g2[r]);
            lossy(m.sigmam, mu, h.gm1[r], h.gm2[r]);
        }
    }
}

// Metric arrays (timestepping.F90:314-370).
void metrics(HostState& h) {
    h.dxe.init(h.alloc[HX].x0, h.alloc[HX].x1, -1.0e10f);
    h.dye.init(h.alloc[HY].y0, h.alloc[HY].y1, -1.0e10f);
    h.dze.init(h.alloc[HZ].z0, h.alloc[HZ].z1, -1.0e10f);
    h.dxh.init(h.alloc[EX].x0, h.alloc[EX].x1, -1.0e10f);
    h.dyh.init(h.alloc[EY].y0, h.alloc[EY].y1, -1.0e10f);
    h.dzh.init(h.alloc[EZ].z0, h.alloc[EZ].z1, -1.0e10f);
    Vec* e[3] = {&h.dxe, &h.dye, &h.dze};
    Vec* hh[3] = {&h.dxh, &h.dyh, &h.dzh};
    const Vec* D[3] = {&h.dx, &h.dy, &h.dz};
    Vec* ie[3] = {&h.idxe, &h.idye, &h.idze};
    Vec* ih[3] = {&h.idxh, &h.idyh, &h.idzh};
    for (int a = 0; a < 3; ++a) {
        for (int i = e[a]->lo; i <= e[a]->hi(); ++i) (*e[a])[i] = (*D[a])[i];
        for (int i = hh[a]->lo; i <= hh[a]->hi(); ++i) (*hh[a])[i] = ((*D[a])[i] + (*D[a])[i - 1]) / 2.0f;
        ie[a]->init(e[a]->lo, e[a]->hi(), 0.0f);
        ih[a]->init(hh[a]->lo, hh[a]->hi(), 0.0f);
        for (int i = e[a]->lo; i <= e[a]->hi(); ++i) (*ie[a])[i] = 1.0f / (*e[a])[i];
        for (int i = hh[a]->lo; i <= hh[a]->hi(); ++i) (*ih[a])[i] = 1.0f / (*hh[a])[i];
    }
}

// InitCPMLBorders + calc_cpmlconstants (borderscpml.F90:90-473, 1465-1733).
void cpml(HostState& h, const sgpu_problem* p, sgpu_cpml_desc& d) {
    // slab boxes: Down, Up, Left, Right, Back, Front
    for (int f = 0; f < 6; ++f) {
        const Box& w = h.sweep[f];
        const Box& q = h.sinpml[f];
        Box r[6] = {Box{w.x0, w.x1, w.y0, w.y1, w.z0, std::min(q.z0 - 1, w.z1)},
                    Box{w.x0, w.x1, w.y0, w.y1, std::max(q.z1 + 1, w.z0), w.z1},
                    Box{w.x0, w.x1, w.y0, std::min(q.y0 - 1, w.y1), w.z0, w.z1},
                    Box{w.x0, w.x1, std::max(q.y1 + 1, w.y0), w.y1, w.z0, w.z1},
                    Box{w.x0, std::min(q.x0 - 1, w.x1), w.y0, w.y1, w.z0, w.z1},
                    Box{std::max(q.x1 + 1, w.x0), w.x1, w.y0, w.y1, w.z0, w.z1}};
        const int face_axis[6] = {2, 2, 1, 1, 0, 0}, face_side[6] = {0, 1, 0, 1, 0, 1};
        for (int reg = 0; reg < 6; ++reg) {
            if (h.layers[face_axis[reg]][face_side[reg]] == 0) r[reg].z0 = r[reg].z1 + 100;
            d.pmlc[f][reg] = to_lim(r[reg]);
        }
    }
    const float amax = p->alphamax, aord = p->alphaorder, kmax = p->kappamax;
    float smax[3][2], apmax[3][2], kpmax[3][2];
    const float del[3][2] = {{h.dxe[h.alloc[EX].x0], h.dxe[h.alloc[EX].x1]},
                             {h.dye[h.alloc[EY].y0], h.dye[h.alloc[EY].y1]},
                             {h.dze[h.alloc[EZ].z0], h.dze[h.alloc[EZ].z1]}};
    for (int a = 0; a < 3; ++a)
        for (int s = 0; s < 2; ++s) {
            const int L = h.layers[a][s];
            if (L == 0) {
                smax[a][s] = 1.0e29f;
                apmax[a][s] = 0.0f;
                kpmax[a][s] = 1.0f;
                continue;
            }
            if (L == 10 || L == 5)  // borderscpml.F90:1494-1497: R is not used
                smax[a][s] = 0.8f * (h.order[a][s] + 1.0f) / (std::sqrt(h.mu0 / h.eps0) * del[a][s]);
            else
                smax[a][s] = -((std::log(h.refl[a][s]) * (h.order[a][s] + 1.0f)) /
                               (2.0f * std::sqrt(h.mu0 / h.eps0) * (float)L * del[a][s]));
            apmax[a][s] = amax * smax[a][s];
            kpmax[a][s] = kmax;
        }
    // normalised depths inside the PML, electric nodes (ce) and magnetic half
    // nodes (cm), borderscpml.F90:229-300
    const Box* AH[3] = {&h.alloc[HX], &h.alloc[HY], &h.alloc[HZ]};
    const Box* AE[3] = {&h.alloc[EX], &h.alloc[EY], &h.alloc[EZ]};
    const Box* SH[3] = {&h.sinpml[HX], &h.sinpml[HY], &h.sinpml[HZ]};
    const Vec* dhv[3] = {&h.dxh, &h.dyh, &h.dzh};
    const Vec* dev[3] = {&h.dxe, &h.dye, &h.dze};
    Vec* ihv[3] = {&h.idxh, &h.idyh, &h.idzh};
    Vec* iev[3] = {&h.idxe, &h.idye, &h.idze};
    const double dt = h.dt;
    auto lohi = [](const Box* b, int a, int& lo, int& hi) {
        lo = a == 0 ? b->x0 : (a == 1 ? b->y0 : b->z0);
        hi = a == 0 ? b->x1 : (a == 1 ? b->y1 : b->z1);
    };
    // without a CPML face InitCPMLBorders returns before calc_cpmlconstants
    // (borderscpml.F90:140-143): the inverse steps stay as they are; faces
    // without CPML keep order 0 and kPar_max 1, which leaves their outer
    // inverse steps unchanged too (their P_b/P_c are never read)
    bool any_pml = false;
    for (int a = 0; a < 3; ++a) any_pml = any_pml || h.layers[a][0] > 0 || h.layers[a][1] > 0;
    for (int a = 0; a < 3; ++a) {
        int lo, hi, alo, ahi, slo, shi;
        lohi(AH[a], a, lo, hi);
        lohi(SH[a], a, slo, shi);
        const int N0 = h.layers[a][0], N1 = h.layers[a][1];
        Vec ce, ice, cm, icm;
        ce.init(lo, hi, 0); ice.init(lo, hi, 0); cm.init(lo, hi, 0); icm.init(lo, hi, 0);
        for (int i = lo; i <= hi; ++i) {
            if (i <= slo) {
                ce[i] = 1.0f * (float)(slo - i) / (float)N0;
                ice[i] = 1.0f * (float)(N0 - (slo - i)) / (float)N0;
            } else if (i >= shi) {
                ce[i] = 1.0f * (float)(i - shi) / (float)N1;
                ice[i] = 1.0f * (float)(N1 - (i - shi)) / (float)N1;
            }
            if (i <= slo - 1) {
                cm[i] = 1.0f * ((float)slo - ((float)i + 0.5f)) / (float)N0;
                icm[i] = 1.0f * ((float)N0 - ((float)slo - ((float)i + 0.5f))) / (float)N0;
            } else if (i >= shi) {
                cm[i] = 1.0f * ((float)(i - shi) + 0.5f) / (float)N1;
                icm[i] = 1.0f * ((float)N1 - ((float)(i - shi) + 0.5f)) / (float)N1;
            }
        }
        h.pbe[a].init(lo, hi, 1.0f); h.pce[a].init(lo, hi, 0.0f);
        h.pbm[a].init(lo, hi, 1.0f); h.pcm[a].init(lo, hi, 0.0f);
        auto coef = [&](int s, float depth, float idepth, float step, float& pb, float& pc, float& inv) {
            float sig, kap;
            if (h.order[a][s] == 0.0f) {
                sig = smax[a][s];
                kap = 1.0f + (kpmax[a][s] - 1.0f);
            } else {
                sig = smax[a][s] * std::pow(depth, h.order[a][s]);
                kap = 1.0f + (kpmax[a][s] - 1.0f) * std::pow(depth, h.order[a][s]);
            }
            float alp = apmax[a][s] * std::pow(idepth, aord);
            pb = (float)std::exp(-((double)(sig / kap + alp) * dt) / (double)h.eps0);
            pc = (sig * (pb - 1.0f) / (sig + kap * alp) / kap) / step;
            inv = 1.0f / (kap * step);
        };
        lohi(AE[a], a, alo, ahi);
        for (int i = alo; i <= ahi && any_pml; ++i) {
            if (i <= slo - 1) coef(0, ce[i], ice[i], (*dhv[a])[i], h.pbe[a][i], h.pce[a][i], (*ihv[a])[i]);
            else if (i >= shi + 1) coef(1, ce[i], ice[i], (*dhv[a])[i], h.pbe[a][i], h.pce[a][i], (*ihv[a])[i]);
        }
        for (int i = lo; i <= hi && any_pml; ++i) {
            if (i <= slo - 1) coef(0, cm[i], icm[i], (*dev[a])[i], h.pbm[a][i], h.pcm[a][i], (*iev[a])[i]);
            else if (i >= shi) coef(1, cm[i], icm[i], (*dev[a])[i], h.pbm[a][i], h.pcm[a][i], (*iev[a])[i]);
        }
        d.p_be[a] = h.pbe[a].v.data();
        d.p_ce[a] = h.pce[a].v.data();
        d.p_bm[a] = h.pbm[a].v.data();
        d.p_cm[a] = h.pcm[a].v.data();
    }
}

// calc_murconstants (bordersmur.F90:316-363) for the Mur faces:
//   cnum = (1/Id(outer node)) / (dt * cluz / sqrt(Epr*Mur)),  CAB1 = (1-cnum)/(1+cnum)
// with FP32 operands, the FP64 dt promoting the denominator and the quotient
// stored in FP32.  Id is taken after calc_cpmlconstants.
void mur_constants(HostState& h) {
    const float idh[6] = {h.idxh[h.alloc[EX].x0], h.idxh[h.alloc[EX].x1], h.idyh[h.alloc[EY].y0],
                          h.idyh[h.alloc[EY].y1], h.idzh[h.alloc[EZ].z0], h.idzh[h.alloc[EZ].z1]};
    for (int f = 0; f < 6; ++f) {
        h.cab1[f].clear();
        if (!h.mur[f / 2][f % 2]) continue;
        h.cab1[f].resize(h.num_media + 1);
        for (int m = 0; m <= h.num_media; ++m) {
            const float den = std::sqrt(h.med[m].epr * h.med[m].mur);
            const float cnum = (float)((double)(1.0f / idh[f]) / ((h.dt * (double)h.cluz) / (double)den));
            h.cab1[f][m] = (1.0f - cnum) / (1.0f + cnum);
        }
    }
}

// InitEDispersives coefficients (electricdispersive.F90:77-149) and, with
// mag, those of InitMdispersives (magneticdispersive.F90:79-142): the same
// construction from the magnetic poles, mu11 and sigmam11, writing GM1/GM2.
void pole_residue(HostState& h, const sgpu_problem* p, bool mag, std::vector<int>& idx, std::vector<int>& np,
                  std::vector<double>& K, std::vector<double>& B, std::vector<double>& G) {
    const double dt = h.dt;
    std::vector<float>& c1 = mag ? h.gm1 : h.g1;
    std::vector<float>& c2 = mag ? h.gm2 : h.g2;
    for (int m = 1; m <= h.num_media; ++m) {
        if (!(mag ? h.med[m].mdisp : h.med[m].disp)) continue;
        const sgpu_region& g = p->regions[h.med[m].region];
        const int npoles = mag ? g.mpoles : g.npoles;
        const float* res = mag ? g.mresidues : g.residues;
        const float* bp = mag ? g.mbpoles : g.bpoles;
        std::vector<Cx> kap, bet;
        float tempo = 0.0f;
        for (int q = 0; q < npoles; ++q) {
            Cx C{(double)res[2 * q], (double)res[2 * q + 1]};
            Cx a{(double)(-bp[2 * q]), (double)(-bp[2 * q + 1])};
            Cx half{(a.r * dt) / 2.0, (a.i * dt) / 2.0};
            Cx den{1.0 - half.r, -half.i};
            kap.push_back(cx_div(Cx{1.0 + half.r, half.i}, den));
            bet.push_back(cx_div(Cx{C.r * dt, C.i * dt}, den));
            tempo = (float)((double)tempo + bet.back().r);
        }
        const float v11 = mag ? g.mu : g.eps, s11 = mag ? g.sigmam : g.sigma;
        const double lo = (double)(2.0f * v11 + tempo);
        const double sd = (double)s11 * dt;
        c1[m] = (float)((lo - sd) / (lo + sd));
        c2[m] = (float)(((double)2.0f * dt) / (lo + sd));
        const double half_g2 = (double)(c2[m] / 2.0f);
        idx.push_back(m);
        np.push_back(npoles);
        for (int q = 0; q < npoles; ++q) {
            K.push_back(kap[q].r); K.push_back(kap[q].i);
            B.push_back(bet[q].r); B.push_back(bet[q].i);
            G.push_back(half_g2 * (1.0 + kap[q].r)); G.push_back(half_g2 * kap[q].i);
        }
    }
}


// Plane-wave descriptors: InitPlaneWave (planewaves.F90:72-770) with the
// pre-processing of preprocess_geom.F90:290-413 and calc_planewaveconstants
// (:1494-1510).
void planewaves(HostState& h, const sgpu_problem* p) {
    const bool half[6][3] = {{true, false, false}, {false, true, false}, {false, false, true},
                             {false, true, true},  {true, false, true}, {true, true, false}};
    const Vec* lines[3] = {&h.lx, &h.ly, &h.lz};
    for (int f = 0; f < 6; ++f) {
        const Box& w = h.sweep[f];
        const int lo[3] = {w.x0 - 1, w.y0 - 1, w.z0 - 1}, hi[3] = {w.x1 + 1, w.y1 + 1, w.z1 + 1};
        for (int a = 0; a < 3; ++a) {
            h.phys_lo[f][a] = lo[a];
            h.phys[f][a].assign(hi[a] - lo[a] + 1, 0.0f);
            for (int i = lo[a]; i <= (half[f][a] ? hi[a] - 1 : hi[a]); ++i)
                h.phys[f][a][i - lo[a]] = half[f][a] ? ((*lines[a])[i] + (*lines[a])[i + 1]) * 0.5f : (*lines[a])[i];
        }
    }
    h.samples.reserve(p->npw + p->nnodal);
    for (int w = 0; w < p->npw; ++w) {
        const sgpu_planewave_src& src = p->pw[w];
        int bx0 = std::min(src.x1, src.x2), bx1 = std::max(src.x1, src.x2);
        int by0 = std::min(src.y1, src.y2), by1 = std::max(src.y1, src.y2);
        int bz0 = std::min(src.z1, src.z2), bz1 = std::max(src.z1, src.z2);
        if (bx0 == h.sinpml[HX].x0) bx0 -= 5;
        if (bx1 == h.sinpml[HX].x1) bx1 += 5;
        if (by0 == h.sinpml[HY].y0) by0 -= 5;
        if (by1 == h.sinpml[HY].y1) by1 += 5;
        if (bz0 == h.sinpml[HZ].z0) bz0 -= 5;
        if (bz1 == h.sinpml[HZ].z1) bz1 += 5;
        const float amp = 1.0f;
        const float ez = amp * std::cos(src.alpha);
        const float ey = amp * std::sin(src.alpha) * std::sin(src.beta);
        const float ex = amp * std::sin(src.alpha) * std::cos(src.beta);
        float pz = std::cos(src.theta), py = std::sin(src.theta) * std::sin(src.phi), px = std::sin(src.theta) * std::cos(src.phi);
        const float mod = std::sqrt(px * px + py * py + pz * pz);
        px = px / mod; py = py / mod; pz = pz / mod;
        sgpu_planewave_desc d{};
        const Box* SS = h.sinpml;  // sgg%SINPMLSweep equals SINPML_fullsize for one layout
        d.active[0] = bx0 >= SS[HX].x0 && bx0 <= SS[HX].x1;
        d.active[1] = bx1 <= SS[HX].x1 && bx1 >= SS[HX].x0;
        d.active[2] = by0 >= SS[HY].y0 && by0 <= SS[HY].y1;
        d.active[3] = by1 <= SS[HY].y1 && by1 >= SS[HY].y0;
        d.active[4] = bz0 >= SS[HZ].z0 && bz0 <= SS[HZ].z1;
        d.active[5] = bz1 <= SS[HZ].z1 && bz1 >= SS[HZ].z0;
        // TrFr / IzDe / AbAr (planewaves.F90:217-301) as {fixed, lo1, hi1, lo2, hi2}
        auto clip = [&](int c, int axis, int lo, int hi, int& a, int& b) {
            const Box& q = SS[c];
            int qlo = axis == 0 ? q.x0 : (axis == 1 ? q.y0 : q.z0), qhi = axis == 0 ? q.x1 : (axis == 1 ? q.y1 : q.z1);
            a = std::max(qlo, lo);
            b = std::min(qhi, hi);
        };
        for (int c : {EZ, EY}) {
            int i0, i1, j0, j1, k0, k1;
            clip(c, 0, bx0, bx1, i0, i1);
            clip(c, 1, by0, c == EY ? by1 - 1 : by1, j0, j1);
            clip(c, 2, bz0, c == EZ ? bz1 - 1 : bz1, k0, k1);
            const int hc = c == EZ ? HY : HZ;
            int* back = d.lim[0][c]; int* front = d.lim[1][c];
            back[0] = i0; front[0] = i1;
            back[1] = front[1] = k0; back[2] = front[2] = k1; back[3] = front[3] = j0; back[4] = front[4] = j1;
            int* hb = d.lim[0][hc]; int* hf = d.lim[1][hc];
            hb[0] = i0 - 1; hf[0] = i1;
            hb[1] = hf[1] = k0; hb[2] = hf[2] = k1; hb[3] = hf[3] = j0; hb[4] = hf[4] = j1;
        }
        for (int c : {EX, EZ}) {
            int i0, i1, j0, j1, k0, k1;
            clip(c, 1, by0, by1, j0, j1);
            clip(c, 0, bx0, c == EX ? bx1 - 1 : bx1, i0, i1);
            clip(c, 2, bz0, c == EZ ? bz1 - 1 : bz1, k0, k1);
            const int hc = c == EX ? HZ : HX;
            int* l = d.lim[2][c]; int* r = d.lim[3][c];
            l[0] = j0; r[0] = j1;
            l[1] = r[1] = k0; l[2] = r[2] = k1; l[3] = r[3] = i0; l[4] = r[4] = i1;
            int* hl = d.lim[2][hc]; int* hr = d.lim[3][hc];
            hl[0] = j0 - 1; hr[0] = j1;
            hl[1] = hr[1] = k0; hl[2] = hr[2] = k1; hl[3] = hr[3] = i0; hl[4] = hr[4] = i1;
        }
        for (int c : {EY, EX}) {
            int i0, i1, j0, j1, k0, k1;
            clip(c, 2, bz0, bz1, k0, k1);
            clip(c, 0, bx0, c == EX ? bx1 - 1 : bx1, i0, i1);
            clip(c, 1, by0, c == EY ? by1 - 1 : by1, j0, j1);
            const int hc = c == EY ? HX : HY;
            int* dn = d.lim[4][c]; int* up = d.lim[5][c];
            dn[0] = k0; up[0] = k1;
            dn[1] = up[1] = j0; dn[2] = up[2] = j1; dn[3] = up[3] = i0; dn[4] = up[4] = i1;
            int* hd = d.lim[4][hc]; int* hu = d.lim[5][hc];
            hd[0] = k0 - 1; hu[0] = k1;
            hd[1] = hu[1] = j0; hd[2] = hu[2] = j1; hd[3] = hu[3] = i0; hd[4] = hu[4] = i1;
        }
        d.px = px; d.py = py; d.pz = pz;
        d.fpw[0] = ex; d.fpw[1] = ey; d.fpw[2] = ez;
        d.fpw[3] = (py * ez - pz * ey) / h.zvac;
        d.fpw[4] = (pz * ex - px * ez) / h.zvac;
        d.fpw[5] = (px * ey - py * ex) / h.zvac;
        // null-phase corner (planewaves.F90:372-411), no uncertainty term
        const int xl = std::max(bx0 - 1, h.sinpml[HX].x0), xh = std::min(bx1 + 1, h.sinpml[HX].x1);
        const int yl = std::max(by0 - 1, h.sinpml[HY].y0), yh = std::min(by1 + 1, h.sinpml[HY].y1);
        const int zl = std::max(bz0 - 1, h.sinpml[HZ].z0), zh = std::min(bz1 + 1, h.sinpml[HZ].z1);
        const float X0 = px >= 0 ? h.lx[xl] : h.lx[xh];
        const float Y0 = py >= 0 ? h.ly[yl] : h.ly[yh];
        const float Z0 = pz >= 0 ? h.lz[zl] : h.lz[zh];
        const float ddx = h.lx[xl] - h.lx[xh], ddy = h.ly[yl] - h.ly[yh], ddz = h.lz[zl] - h.lz[zh];
        const float diag = std::sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
        d.d0 = ((X0 * px + Y0 * py + Z0 * pz)) - 0.0f * diag;
        d.cluz = h.cluz;
        d.numus = src.nsamples - 1;
        d.deltaevol = src.dsamples;
        h.samples.emplace_back(src.samples, src.samples + src.nsamples);
        d.evol = h.samples.back().data();
        for (int f = 0; f < 6; ++f)
            for (int a = 0; a < 3; ++a) {
                d.phys[f][a] = h.phys[f][a].data();
                d.phys_lo[f][a] = h.phys_lo[f][a];
                d.phys_n[f][a] = (int)h.phys[f][a].size();
            }
        h.pw.push_back(d);
    }
}

// Nodal sources (nodalsources.F90:76-300, 396-777): per component the hard
// sources are applied before the soft ones, each in source order.
void nodal(HostState& h, const sgpu_problem* p) {
    for (int pass = 0; pass < 2; ++pass)
        for (int a = 0; a < 3; ++a)
            for (int hardpass = 1; hardpass >= 0; --hardpass)
                for (int q = 0; q < p->nnodal; ++q) {
                    const sgpu_nodal_src& ns = p->nodal[q];
                    if ((ns.is_hard != 0) != (hardpass != 0)) continue;
                    if ((pass == 0) != (ns.is_elec != 0)) continue;
                    for (int pt = 0; pt < ns.npoints; ++pt) {
                        float amp = ns.amp[3 * pt + a];
                        if (amp == 0.0f) continue;
                        const int comp = (ns.is_elec ? 0 : 3) + a;
                        const Box& w = h.sweep[comp];
                        const int* b = ns.boxes + 6 * pt;
                        sgpu_nodal_desc nd{};
                        nd.comp = comp;
                        nd.hard = ns.is_hard;
                        nd.box = sgpu_lim{std::max(b[0], w.x0), std::min(b[1], w.x1), std::max(b[2], w.y0),
                                          std::min(b[3], w.y1), std::max(b[4], w.z0), std::min(b[5], w.z1)};
                        nd.amplitude = amp;
                        nd.numus = ns.nsamples - 1;
                        nd.deltaevol = ns.dsamples;
                        h.samples.emplace_back(ns.samples, ns.samples + ns.nsamples);
                        nd.evol = h.samples.back().data();
                        h.nodal.push_back(nd);
                    }
                }
}

HostState* make_plan(const sgpu_problem* p, int max_steps, sgpu_status* rc, bool device_media = false) {
    *rc = SGPU_OK;
    if (!p || p->nx < 2 || p->ny < 2 || p->nz < 2 || !p->desx || !p->desy || !p->desz || max_steps < 0) {
        *rc = SGPU_ERR_ARG;
        return nullptr;
    }
    for (int f = 0; f < 6; ++f) {
        const int kind = p->border[f] == 0 ? 9 : p->border[f];
        if (kind != 1 && kind != 2 && kind != 4 && kind != 7 && kind != 9) { *rc = SGPU_ERR_ARG; return nullptr; }
        if (kind == 9 && p->pml_layers[f] < 1) { *rc = SGPU_ERR_ARG; return nullptr; }
    }
    for (int r = 0; r < p->nregions; ++r)
        if (p->regions[r].kind < 0 || p->regions[r].kind > 2 || (p->regions[r].nboxes > 0 && !p->regions[r].boxes) ||
            p->regions[r].npoles < 0 || p->regions[r].mpoles < 0 ||
            (p->regions[r].kind == 2 && p->regions[r].npoles > 0 && (!p->regions[r].residues || !p->regions[r].bpoles)) ||
            (p->regions[r].kind == 2 && p->regions[r].mpoles > 0 && (!p->regions[r].mresidues || !p->regions[r].mbpoles))) {
            *rc = SGPU_ERR_ARG;
            return nullptr;
        }
    HostState* h = new (std::nothrow) HostState();
    if (!h) { *rc = SGPU_ERR_OOM; return nullptr; }
    h->device_media = device_media;
    try {
        limits(*h, p);
        timestep(*h, p);
        media(*h, p);
        if (h->num_media > 32767) { delete h; *rc = SGPU_ERR_UNSUPPORTED; return nullptr; }
        coefficients(*h);
        metrics(*h);
        cpml(*h, p, h->cd);
        mur_constants(*h);
        pole_residue(*h, p, false, h->didx, h->dnp, h->dK, h->dB, h->dG);
        pole_residue(*h, p, true, h->mdidx, h->mdnp, h->mdK, h->mdB, h->mdG);
        h->pec.resize(h->num_media + 1);
        for (int m = 0; m <= h->num_media; ++m) h->pec[m] = h->med[m].pec ? 1 : 0;
        planewaves(*h, p);
        nodal(*h, p);
    } catch (const std::bad_alloc&) {
        delete h;
        *rc = SGPU_ERR_OOM;
        return nullptr;
    }
    h->probes.assign(p->probes, p->probes + 4 * p->nprobes);
    h->probe_cap = p->probe_capacity > 0 ? p->probe_capacity : 1024;  // BuffObse, fdetypes.F90:97
    h->max_steps = max_steps;
    return h;
}

// Floats of the psi array sgpu_init_cpml allocates for a slab box: rows
// start at the local x rounded down to a multiple of 4 and are padded to a
// multiple of 4 floats.
uint64_t psi_floats(const HostState& h, const sgpu_lim& l) {
    if (l.xe < l.xi || l.ye < l.yi || l.ze < l.zi) return 0;
    const int x0 = l.xi - h.alloc[0].x0, x1 = l.xe - h.alloc[0].x0;
    const int xb = x0 & ~3, px = (x1 - xb + 1 + 3) & ~3;
    return (uint64_t)px * (l.ye - l.yi + 1) * (l.ze - l.zi + 1);
}

// Device buffers sgpu_init_borders allocates for the Mur faces: the CAB1
// table per face and Past_ (two layers) per (face, tangential H component).
template <class Fn> void mur_buffers(const HostState& h, Fn&& fn) {
    const int comps[6][2] = {{HZ, HY}, {HZ, HY}, {HX, HZ}, {HX, HZ}, {HY, HX}, {HY, HX}};
    for (int f = 0; f < 6; ++f) {
        if (!h.mur[f / 2][f % 2]) continue;
        fn((uint64_t)(h.num_media + 1) * 4);
        const int a = f / 2;
        for (int comp : comps[f]) {
            const Box& w = h.sweep[comp];
            const uint64_t n[3] = {(uint64_t)(w.x1 - w.x0 + 1), (uint64_t)(w.y1 - w.y0 + 1), (uint64_t)(w.z1 - w.z0 + 1)};
            fn(2 * 4 * (a == 0 ? n[1] * n[2] : (a == 1 ? n[0] * n[2] : n[0] * n[1])));
        }
    }
}

// Hand the plan to the level-1 entry points.
// The planes [z0, z1] of a z-slab sub-domain (the reference's MPI
// decomposition along z, mpicomm.F90): every component's Alloc range
// reaches one plane past the owned planes on a cut side (the halo the
// neighbour fills) and keeps the problem's bounds on the outer sides; its
// Sweep is the owned part of the problem's Sweep.
struct ZWindow {
    bool on = false, first = true, last = true;
    int z0 = 0, z1 = 0;
};

// The media matrices of `h` built on the context's device arrays (regions
// painted in order, the PML extrusion, the copies of the media the PML
// needs, the PEC borders), then the tables that depend on the final media
// list (G1..GM2, CAB1, the ADE coefficients, the PEC flags) recomputed and
// handed to the context.
sgpu_status build_media_on_device(HostState* h, const sgpu_problem* p, sgpu_ctx* c) {
    struct Guard {
        sgpu::DevicePainter* p;
        ~Guard() { sgpu::painter_delete(p); }
    } g{sgpu::painter_new(c)};
    sgpu::DevicePainter* dp = g.p;
    std::vector<int> prio(h->num_media + 1);
    for (int m = 0; m <= h->num_media; ++m) prio[m] = h->med[m].prio;
    sgpu_status s = sgpu::painter_start(dp, prio);
    if (s) return s;
    for (const HostState::PaintRegion& r : h->paint_regions) {
        std::vector<int> items;
        for (const Box& b : r.boxes) {
            Box rg[6];
            paint_ranges(*h, b, rg);
            for (int f = 0; f < 6; ++f)
                if (rg[f].x1 >= rg[f].x0 && rg[f].y1 >= rg[f].y0 && rg[f].z1 >= rg[f].z0)
                    items.insert(items.end(), {f, rg[f].x0, rg[f].x1, rg[f].y0, rg[f].y1, rg[f].z0, rg[f].z1});
        }
        if ((s = sgpu::painter_paint(dp, items, r.idx, r.prio))) return s;
    }
    // CreatePMLmatrix: extrusion along x, y, z per component
    const PmlGeom geom = pml_geom(*h);
    const Box& in = geom.inner;
    int r6[6][6], in6[6][6];
    std::vector<long long> task0(6);
    long long tasks = 0;
    for (int f = 0; f < 6; ++f) {
        const Box& r = geom.reach[f];
        const int v[6] = {r.x0, r.x1, r.y0, r.y1, r.z0, r.z1};
        const int w[6] = {in.x0, in.x1 + kInLo[f][0] - 1, in.y0, in.y1 + kInLo[f][1] - 1, in.z0, in.z1 + kInLo[f][2] - 1};
        std::copy(v, v + 6, r6[f]);
        std::copy(w, w + 6, in6[f]);
        task0[f] = tasks;
        tasks += std::max(0, r.z1 - r.z0 + 1);
        const int lo[3] = {in.x0, in.y0, in.z0};
        for (int a = 0; a < 3; ++a)
            if ((s = sgpu::painter_extrude(dp, f, r6[f], a, lo[a], w[2 * a + 1] + 1, lo[a], w[2 * a + 1]))) return s;
    }
    const long long nyo = geom.outer.y1 - geom.outer.y0 + 1, nxo = geom.outer.x1 - geom.outer.x0 + 1;
    std::vector<long long> first;
    if ((s = sgpu::painter_first(dp, task0, r6, in6, nyo, nxo, h->num_media + 1, first))) return s;
    std::vector<int> copy_of;
    const int before = h->num_media;
    pml_copies(*h, first, copy_of);
    if (h->num_media > 32767) return sgpu::set_error(c, SGPU_ERR_UNSUPPORTED, "more than 32767 media");
    std::vector<int16_t> copy16(before + 1);
    for (int v = 0; v <= before; ++v) copy16[v] = (int16_t)copy_of[v];
    if ((s = sgpu::painter_relabel(dp, r6, in6, copy16))) return s;
    pec_planes(*h, geom, [&](int f, const Box& b) {
        const int b6[6] = {b.x0, b.x1, b.y0, b.y1, b.z0, b.z1};
        if (!s) s = sgpu::painter_zero(dp, f, b6);
    });
    if (s || (s = sgpu::painter_finish(dp))) return s;
    // the tables over the final media list
    coefficients(*h);
    mur_constants(*h);
    h->didx.clear(); h->dnp.clear(); h->dK.clear(); h->dB.clear(); h->dG.clear();
    h->mdidx.clear(); h->mdnp.clear(); h->mdK.clear(); h->mdB.clear(); h->mdG.clear();
    pole_residue(*h, p, false, h->didx, h->dnp, h->dK, h->dB, h->dG);
    pole_residue(*h, p, true, h->mdidx, h->mdnp, h->mdK, h->mdB, h->mdG);
    h->pec.resize(h->num_media + 1);
    for (int m = 0; m <= h->num_media; ++m) h->pec[m] = h->med[m].pec ? 1 : 0;
    return sgpu::set_media_tables(c, h->num_media, h->g1.data(), h->g2.data(), h->gm1.data(), h->gm2.data(), h->pec.data());
}

sgpu_status realize(HostState* h, sgpu::Arena* arena, cudaStream_t stream, sgpu_ctx** out, ZWindow zw = ZWindow(),
                    const sgpu_problem* p = nullptr) {
    Box A[6], W[6];
    for (int f = 0; f < 6; ++f) {
        A[f] = h->alloc[f];
        W[f] = h->sweep[f];
        if (!zw.first) {
            A[f].z0 = zw.z0 - 1;
            W[f].z0 = std::max(W[f].z0, zw.z0);
        }
        if (!zw.last) {
            A[f].z1 = zw.z1 + 1;
            W[f].z1 = std::min(W[f].z1, zw.z1);
        }
        if (W[f].z1 < W[f].z0) {
            delete h;
            return SGPU_ERR_ARG;  // a slab must sweep at least one plane of every component
        }
    }
    sgpu_grid_desc g{};
    for (int f = 0; f < 6; ++f) {
        g.alloc[f] = to_lim(A[f]);
        g.sweep[f] = to_lim(W[f]);
    }
    // z-indexed arrays start at the slab's lower Alloc plane
    const long long dzh = A[HZ].z0 - h->alloc[HZ].z0, dze = A[EZ].z0 - h->alloc[EZ].z0;
    g.num_media = h->num_media;
    g.g1 = h->g1.data(); g.g2 = h->g2.data(); g.gm1 = h->gm1.data(); g.gm2 = h->gm2.data();
    g.is_pec = h->pec.data();
    g.idxe = h->idxe.v.data(); g.idye = h->idye.v.data(); g.idze = h->idze.v.data() + dzh;
    g.idxh = h->idxh.v.data(); g.idyh = h->idyh.v.data(); g.idzh = h->idzh.v.data() + dze;
    g.dt = h->dt;
    sgpu_ctx* c = nullptr;
    sgpu_status s = sgpu::create_in(&g, arena, stream, &c);
    *out = c;
    if (s) { delete h; return s; }
    c->host = h;
    c->host_free = free_host;
    c->zslab = zw.on;
    if (h->device_media) {
        if (!p || zw.on) return sgpu::set_error(c, SGPU_ERR_STATE, "device media need the whole problem");
        if ((s = build_media_on_device(h, p, c))) return s;
    } else {
        for (int f = 0; f < 6; ++f) {
            const size_t off = (size_t)(A[f].z0 - h->alloc[f].z0) * h->mm[f].nx * h->mm[f].ny;
            if ((s = sgpu::upload_media(c, f, h->mm[f].data() + off, false))) return s;  // built here: in range
            h->mm[f].release();  // released once on the device
        }
    }
    sgpu_cpml_desc cd = h->cd;
    if (zw.on) {
        for (int f = 0; f < 6; ++f)
            for (int r = 0; r < 6; ++r) {
                sgpu_lim& b = cd.pmlc[f][r];
                if (!zw.first) b.zi = std::max(b.zi, zw.z0);
                if (!zw.last) b.ze = std::min(b.ze, zw.z1);
            }
        for (int w = 0; w < 4; ++w) {
            const float** v[4] = {&cd.p_be[2], &cd.p_ce[2], &cd.p_bm[2], &cd.p_cm[2]};
            if (*v[w]) *v[w] += dzh;
        }
    }
    if ((s = sgpu_init_cpml(c, &cd))) return s;
    sgpu_border_desc bd{};
    bool borders = false;
    for (int f = 0; f < 6; ++f) {
        const int a = f / 2, sd = f % 2;
        // z faces belong to the slabs at the ends of the problem
        const bool here = a != 2 || (sd == 0 ? zw.first : zw.last);
        if (a == 2 && h->kind[a][sd] == 4 && !(zw.first && zw.last))
            return sgpu::set_error(c, SGPU_ERR_UNSUPPORTED, "periodic z faces across z-slab sub-domains");
        bd.pmc[f] = here && h->kind[a][sd] == 2;
        bd.periodic[f] = here && h->kind[a][sd] == 4;
        bd.mur[f] = here && h->mur[a][sd];
        bd.mur_cab1[f] = h->cab1[f].empty() ? nullptr : h->cab1[f].data();
        borders = borders || bd.pmc[f] || bd.periodic[f] || bd.mur[f];
    }
    if (borders && (s = sgpu_init_borders(c, &bd))) return s;
    sgpu_edisp_desc ed{(int)h->didx.size(), h->didx.data(), h->dnp.data(), h->dK.data(), h->dB.data(), h->dG.data()};
    if ((s = sgpu_init_edisp(c, &ed))) return s;
    if (!h->mdidx.empty()) {
        sgpu_edisp_desc md{(int)h->mdidx.size(), h->mdidx.data(), h->mdnp.data(), h->mdK.data(), h->mdB.data(), h->mdG.data()};
        if ((s = sgpu_init_mdisp(c, &md))) return s;
    }
    for (const sgpu_planewave_desc& d : h->pw)
        if ((s = sgpu_add_planewave(c, &d))) return s;
    for (const sgpu_nodal_desc& d : h->nodal)
        if ((s = sgpu_add_nodal(c, &d))) return s;
    // crea_timevector (timestepping.F90:3230-3240): tiempo(i) = tiempo(i-1) + dt
    std::vector<double> t(h->max_steps + 3);
    t[0] = 0.0;
    for (size_t i = 1; i < t.size(); ++i) t[i] = t[i - 1] + h->dt;
    if ((s = sgpu_set_time(c, 0, (int)t.size(), t.data()))) return s;
    // point probes: a slab records those on the planes it owns (the end slabs
    // also those beyond the first and last swept planes)
    std::vector<int> probes;
    for (size_t q = 0; q + 3 < h->probes.size(); q += 4) {
        const int z = h->probes[q + 3];
        if ((zw.first || z >= zw.z0) && (zw.last || z <= zw.z1)) probes.insert(probes.end(), &h->probes[q], &h->probes[q] + 4);
    }
    if (!probes.empty())
        if ((s = sgpu_set_probes(c, (int)probes.size() / 4, probes.data(), h->probe_cap))) return s;
    return SGPU_OK;
}

}  // namespace

extern "C" {

sgpu_status sgpu_host_plan(const sgpu_problem* p, int max_steps, sgpu_ctx** out) {
    if (!out) return SGPU_ERR_ARG;
    *out = nullptr;
    sgpu_status rc;
    HostState* h = make_plan(p, max_steps, &rc);
    if (!h) return rc;
    sgpu_ctx* c = new (std::nothrow) sgpu_ctx();
    if (!c) { delete h; return SGPU_ERR_OOM; }
    c->host = h;
    c->host_free = free_host;
    c->host_only = true;
    for (int f = 0; f < 6; ++f) {
        c->alloc[f] = to_lim(h->alloc[f]);
        c->sweep[f] = to_lim(h->sweep[f]);
    }
    c->num_media = h->num_media;
    c->dt = h->dt;
    *out = c;
    return SGPU_OK;
}

sgpu_status sgpu_host_create(const sgpu_problem* p, int max_steps, sgpu_ctx** out) {
    if (!out) return SGPU_ERR_ARG;
    *out = nullptr;
    sgpu_status rc;
    // a problem set up alone builds its media matrices on the device
    HostState* h = make_plan(p, max_steps, &rc, true);
    if (!h) return rc;
    return realize(h, nullptr, nullptr, out, ZWindow(), p);
}

sgpu_status sgpu_host_create_zslab(const sgpu_problem* p, int max_steps, int z0, int z1, sgpu_ctx** out) {
    if (!out || z1 < z0) return SGPU_ERR_ARG;
    *out = nullptr;
    sgpu_status rc;
    HostState* h = make_plan(p, max_steps, &rc);
    if (!h) return rc;
    int lo = h->sweep[0].z0, hi = h->sweep[0].z1;
    for (int f = 1; f < 6; ++f) {
        lo = std::min(lo, h->sweep[f].z0);
        hi = std::max(hi, h->sweep[f].z1);
    }
    ZWindow zw;
    zw.on = true;
    zw.z0 = z0;
    zw.z1 = z1;
    zw.first = z0 <= lo;
    zw.last = z1 >= hi;
    return realize(h, nullptr, nullptr, out, zw);
}

sgpu_status sgpu_host_footprint(const sgpu_ctx* c, uint64_t* bytes) {
    if (!c || !c->host || !bytes) return SGPU_ERR_ARG;
    const HostState* h = (const HostState*)c->host;
    // padded field and media volume, as sgpu_create lays it out
    long long nxa = 0, nya = 0, nza = 0;
    for (int f = 0; f < 6; ++f) {
        nxa = std::max<long long>(nxa, h->alloc[f].x1 - h->alloc[0].x0 + 1);
        nya = std::max<long long>(nya, h->alloc[f].y1 - h->alloc[0].y0 + 1);
        nza = std::max<long long>(nza, h->alloc[f].z1 - h->alloc[0].z0 + 1);
    }
    const long long vol = (nxa + 31) / 32 * 32 * nya * nza;
    uint64_t b = (uint64_t)vol * 6 * (sizeof(float) + sizeof(int16_t) + sizeof(uint8_t));
    // psi slabs
    for (int f = 0; f < 6; ++f)
        for (int reg = 0; reg < 6; ++reg) b += psi_floats(*h, h->cd.pmlc[f][reg]) * 4;
    // ADE state: swept E (H) nodes of electric (magnetic) pole-residue media
    for (int side = 0; side < 2; ++side) {
        const std::vector<int>& idx = side ? h->mdidx : h->didx;
        const std::vector<int>& np = side ? h->mdnp : h->dnp;
        if (idx.empty()) continue;
        std::vector<char> disp(h->num_media + 1, 0);
        int nu = 0;
        for (size_t m = 0; m < idx.size(); ++m) {
            disp[idx[m]] = 1;
            nu = std::max(nu, np[m]);
        }
        uint64_t nodes = 0;
        bool have = true;
        for (int f = 3 * side; f < 3 * side + 3; ++f) {
            if (h->mm[f].empty()) { have = false; break; }
            const Box& w = h->sweep[f];
            MediaMat& m = const_cast<MediaMat&>(h->mm[f]);
            for (int k = w.z0; k <= w.z1; ++k)
                for (int j = w.y0; j <= w.y1; ++j)
                    for (int i = w.x0; i <= w.x1; ++i) nodes += disp[m.at(i, j, k)];
        }
        if (!have) nodes = (uint64_t)vol * 3;  // upper bound once the host copy is released
        b += nodes * (4 + 1 + 4 + 16 * (uint64_t)nu);
        b += (nodes / 32 + 6) * 16;  // run descriptors of the node groups (one per 32 nodes and component, plus one)
    }
    mur_buffers(*h, [&](uint64_t n) { b += n; });
    b += (uint64_t)h->probes.size() / 4 * h->probe_cap * 4;
    *bytes = b;
    return SGPU_OK;
}

sgpu_status sgpu_batch_footprint(const sgpu_ctx* c, uint64_t* bytes, uint64_t* largest) {
    if (!c || !c->host || !bytes) return SGPU_ERR_ARG;
    const HostState* h = (const HostState*)c->host;
    uint64_t total = 0, big = 0;
    auto buf = [&](uint64_t b) {
        if (!b) return;
        b = (b + 255) / 256 * 256;  // the arena's grain
        total += b;
        big = std::max(big, b);
    };
    long long nxa = 0, nya = 0, nza = 0;
    for (int f = 0; f < 6; ++f) {
        nxa = std::max<long long>(nxa, h->alloc[f].x1 - h->alloc[0].x0 + 1);
        nya = std::max<long long>(nya, h->alloc[f].y1 - h->alloc[0].y0 + 1);
        nza = std::max<long long>(nza, h->alloc[f].z1 - h->alloc[0].z0 + 1);
    }
    const long long pitch = (nxa + 31) / 32 * 32, vol = pitch * nya * nza;
    for (int f = 0; f < 6; ++f) {
        buf((uint64_t)vol * 4);  // field
        buf((uint64_t)vol * 2);  // media
        buf((uint64_t)vol * 1);  // one-byte media copy
    }
    const uint64_t n1 = (uint64_t)h->num_media + 1;
    for (int q = 0; q < 4; ++q) buf(n1 * 4);  // G1 G2 GM1 GM2
    for (long long n : {pitch, nya, nza, pitch, nya, nza}) buf((uint64_t)n * 4);  // metrics
    for (int q = 0; q < 3; ++q) buf(4);  // step, flag and error words
    // CPML: the twelve per-axis vectors and the psi slabs
    for (int a = 0; a < 3; ++a)
        for (const Vec* v : {&h->pbe[a], &h->pce[a], &h->pbm[a], &h->pcm[a]}) buf((uint64_t)v->v.size() * 4 + 64);
    for (int f = 0; f < 6; ++f)
        for (int reg = 0; reg < 6; ++reg) buf(psi_floats(*h, h->cd.pmlc[f][reg]) * 4);
    // ADE: per component node list, slot, previous field and state; the
    // per-row count/offset scratch of the set-up is live at the same time
    for (int side = 0; side < 2; ++side) {
        const std::vector<int>& idx = side ? h->mdidx : h->didx;
        const std::vector<int>& np = side ? h->mdnp : h->dnp;
        if (idx.empty()) continue;
        std::vector<char> disp(h->num_media + 1, 0);
        int nu = 0;
        for (size_t m = 0; m < idx.size(); ++m) {
            disp[idx[m]] = 1;
            nu = std::max(nu, np[m]);
        }
        buf(idx.size() * sizeof(sgpu::DispMedium) + 64);  // medium table
        buf(n1 * 2);                                      // slot of medium
        for (int f = 3 * side; f < 3 * side + 3; ++f) {
            uint64_t nodes = 0;
            const Box& w = h->sweep[f];
            if (h->mm[f].empty()) {
                nodes = (uint64_t)vol;
            } else {
                MediaMat& m = const_cast<MediaMat&>(h->mm[f]);
                for (int k = w.z0; k <= w.z1; ++k)
                    for (int j = w.y0; j <= w.y1; ++j)
                        for (int i = w.x0; i <= w.x1; ++i) nodes += disp[m.at(i, j, k)];
            }
            const uint64_t rows = (uint64_t)(w.y1 - w.y0 + 1) * (w.z1 - w.z0 + 1);
            buf(nodes * 4);
            buf(nodes * 1);
            buf(nodes * 4);
            buf(nodes * 16 * (uint64_t)std::max(1, nu));
            if (nodes) buf(((nodes + 31) / 32 + 1) * 16);  // run descriptors of the node groups
            buf(rows * 8);
            buf(rows * 4);
        }
    }
    // sources: every plane-wave face node and nodal point is at most one row
    uint64_t rows = 0, samples = 0;
    for (const sgpu_planewave_desc& d : h->pw) {
        for (int f = 0; f < 6; ++f)
            for (int comp = 0; comp < 6; ++comp) {
                const int* l = d.lim[f][comp];
                if (l[2] >= l[1] && l[4] >= l[3]) rows += (uint64_t)(l[2] - l[1] + 1) * (l[4] - l[3] + 1);
            }
        samples += (uint64_t)d.numus + 1;
    }
    for (const sgpu_nodal_desc& d : h->nodal) {
        rows += (uint64_t)(d.box.xe - d.box.xi + 1) * (d.box.ye - d.box.yi + 1) * (d.box.ze - d.box.zi + 1);
        samples += (uint64_t)d.numus + 1;
    }
    for (int side = 0; side < 2; ++side) {
        buf(rows * 4);
        buf(rows * 4);
        buf(rows * 4 + 4);
        buf(rows * 24);
        buf((h->pw.size() + h->nodal.size()) * 16);
        buf(samples * 4);
    }
    mur_buffers(*h, buf);
    buf((uint64_t)(h->max_steps + 3) * 8);  // time vector
    const uint64_t np = h->probes.size() / 4;
    buf(np * 4);
    buf(np * 8);
    buf(np * (uint64_t)(h->max_steps + 1) * 4);  // whole traces
    *bytes = total;
    if (largest) *largest = big;
    return SGPU_OK;
}

sgpu_status sgpu_host_info(const sgpu_ctx* c, double* dt, int* num_media, sgpu_lim* alloc6, sgpu_lim* sweep6,
                           sgpu_lim* sinpml6) {
    if (!c || !c->host) return SGPU_ERR_STATE;
    const HostState* h = (const HostState*)c->host;
    if (dt) *dt = h->dt;
    if (num_media) *num_media = h->num_media;
    // the context's own ranges (a z-slab's differ from the problem's)
    for (int f = 0; f < 6; ++f) {
        if (alloc6) alloc6[f] = c->alloc[f];
        if (sweep6) sweep6[f] = c->sweep[f];
        if (sinpml6) sinpml6[f] = to_lim(h->sinpml[f]);
    }
    return SGPU_OK;
}

sgpu_status sgpu_host_get_g(const sgpu_ctx* c, float* g1, float* g2, float* gm1, float* gm2) {
    if (!c || !c->host) return SGPU_ERR_STATE;
    const HostState* h = (const HostState*)c->host;
    const size_t n = h->g1.size();
    std::memcpy(g1, h->g1.data(), n * 4); std::memcpy(g2, h->g2.data(), n * 4);
    std::memcpy(gm1, h->gm1.data(), n * 4); std::memcpy(gm2, h->gm2.data(), n * 4);
    return SGPU_OK;
}

sgpu_status sgpu_host_get_metric(const sgpu_ctx* c, int which, float* out, int* lo, int* hi) {
    if (!c || !c->host || which < 0 || which > 17) return SGPU_ERR_ARG;
    const HostState* h = (const HostState*)c->host;
    const Vec* t[18] = {&h->idxe, &h->idye, &h->idze, &h->idxh, &h->idyh, &h->idzh, &h->pbe[0], &h->pbe[1], &h->pbe[2],
                        &h->pce[0], &h->pce[1], &h->pce[2], &h->pbm[0], &h->pbm[1], &h->pbm[2], &h->pcm[0], &h->pcm[1], &h->pcm[2]};
    const Vec* v = t[which];
    if (lo) *lo = v->lo;
    if (hi) *hi = v->hi();
    if (out) std::memcpy(out, v->v.data(), v->v.size() * 4);
    return SGPU_OK;
}

sgpu_status sgpu_host_get_constants(const sgpu_ctx* c, float* eps0, float* mu0) {
    if (!c || !c->host) return SGPU_ERR_ARG;
    const HostState* h = (const HostState*)c->host;
    if (eps0) *eps0 = h->eps0;
    if (mu0) *mu0 = h->mu0;
    return SGPU_OK;
}

// Incid as FlushObservationFiles calls it for the incident column of a point
// probe file (observation.F90:3826-3875 -> planewaves.F90:778-853 with
// calledfromobservation): EhI = 0, then EhI = EhI + fpw(w, comp) * evolucion
// over every plane wave w, at the node's PhysCoor of component comp; a dummy
// flag takes still_planewave_time's place, so the run's switch is untouched.
sgpu_status sgpu_host_incident(const sgpu_ctx* c, int comp, int i, int j, int k, int nt, const float* t, float* out) {
    if (!c || !c->host || comp < 0 || comp > 5 || nt < 0 || (nt > 0 && (!t || !out))) return SGPU_ERR_ARG;
    const HostState* h = (const HostState*)c->host;
    if (h->pw.empty()) {
        for (int q = 0; q < nt; ++q) out[q] = 0.0f;
        return SGPU_OK;
    }
    const int ijk[3] = {i, j, k};
    float xyz[3];
    for (int a = 0; a < 3; ++a) {
        const int r = ijk[a] - h->phys_lo[comp][a];
        if (r < 0 || r >= (int)h->phys[comp][a].size())
            return sgpu::set_error(const_cast<sgpu_ctx*>(c), SGPU_ERR_ARG, "node outside the PhysCoor range");
        xyz[a] = h->phys[comp][a][r];
    }
    for (int q = 0; q < nt; ++q) {
        float ehi = 0.0f;
        for (const sgpu_planewave_desc& d : h->pw) {
            const float dd = (xyz[0] * d.px + xyz[1] * d.py + xyz[2] * d.pz) - d.d0;
            float ev = 0.0f;
            const long long nprev = (long long)((t[q] - dd / d.cluz) / d.deltaevol);
            if (nprev + 1 <= d.numus && nprev > 0)
                ev = (d.evol[nprev + 1] - d.evol[nprev]) / d.deltaevol * ((t[q] - dd / d.cluz) - (float)nprev * d.deltaevol) +
                     d.evol[nprev];
            ehi = ehi + d.fpw[comp] * ev;
        }
        out[q] = ehi;
    }
    return SGPU_OK;
}

// InitFarField (farfield.F90:118-1158) for the descriptor of
// sgpu_add_farfield.  SINPMLSweep is the SINPML range of one layout.
sgpu_status sgpu_host_add_farfield(sgpu_ctx* c, const sgpu_farfield_spec* s, int* id) {
    if (!c || !s) return SGPU_ERR_ARG;
    if (!c->host) return sgpu::set_error(c, SGPU_ERR_STATE, "far fields need a context from sgpu_host_create");
    if (c->zslab) return sgpu::set_error(c, SGPU_ERR_STATE, "far fields are not split across z-slabs");
    const HostState* h = (const HostState*)c->host;
    const Box& SX = h->sinpml[HX];
    const Box& SY = h->sinpml[HY];
    const Box& SZ = h->sinpml[HZ];
    // :179-184, the box clipped to the non-CPML H ranges
    int e[6] = {std::max(s->box[0], SX.x0), std::min(s->box[1], SX.x1), std::max(s->box[2], SY.y0),
                std::min(s->box[3], SY.y1), std::max(s->box[4], SZ.z0), std::min(s->box[5], SZ.z1)};
    // :284-301, a face is sampled when it lies strictly inside that range
    const bool in[6] = {e[0] > SX.x0 && e[0] <= SX.x1, e[1] < SX.x1 && e[1] >= SX.x0,
                        e[2] > SY.y0 && e[2] <= SY.y1, e[3] < SY.y1 && e[3] >= SY.y0,
                        e[4] > SZ.z0 && e[4] <= SZ.z1, e[5] < SZ.z1 && e[5] >= SZ.z0};
    // :316-510, a side on the edge of the range with a PEC or PMC border would
    // need image faces, which the reference refuses
    const bool edge[6] = {e[0] <= SX.x0, e[1] >= SX.x1, e[2] <= SY.y0, e[3] >= SY.y1, e[4] <= SZ.z0, e[5] >= SZ.z1};
    for (int f = 0; f < 6; ++f) {
        const int kind = h->kind[f / 2][f % 2];
        if (!edge[f] || (kind != 1 && kind != 2)) continue;
        for (int g = 0; g < 6; ++g)
            if (g != f && in[g]) return sgpu::set_error(c, SGPU_ERR_ARG, "NF2FF STILL UNSUPPORTED (a face on a PEC/PMC border)");
    }
    sgpu_farfield_desc d{};
    for (int f = 0; f < 6; ++f) d.active[f] = in[f] && s->faces[f];
    // :512-580 (TrFr, IzDe, AbAr limits)
    const Box& Sx = h->sinpml[EX];
    const Box& Sy = h->sinpml[EY];
    const Box& Sz = h->sinpml[EZ];
    for (int side = 0; side < 2; ++side) {
        const bool lo = side == 0;
        // x faces: Ez, Ey; loops k then j
        int* L = d.lim[side][0];
        L[0] = lo ? std::max(Sz.x0, e[0]) : std::min(Sz.x1, e[1]);
        L[1] = std::max(Sz.z0, e[4]); L[2] = std::min(Sz.z1, e[5] - 1);
        L[3] = std::max(Sz.y0, e[2]); L[4] = std::min(Sz.y1, e[3]);
        L = d.lim[side][1];
        L[0] = lo ? std::max(Sy.x0, e[0]) : std::min(Sy.x1, e[1]);
        L[1] = std::max(Sy.z0, e[4]); L[2] = std::min(Sy.z1 - 1, e[5]);
        L[3] = std::max(Sy.y0, e[2]); L[4] = std::min(Sy.y1, e[3] - 1);
        // y faces: Ez, Ex; loops k then i
        L = d.lim[2 + side][0];
        L[0] = lo ? std::max(Sz.y0, e[2]) : std::min(Sz.y1, e[3]);
        L[1] = std::max(Sz.z0, e[4]); L[2] = std::min(Sz.z1, e[5] - 1);
        L[3] = std::max(Sz.x0, e[0]); L[4] = std::min(Sz.x1, e[1]);
        L = d.lim[2 + side][1];
        L[0] = lo ? std::max(Sx.y0, e[2]) : std::min(Sx.y1, e[3]);
        L[1] = std::max(Sx.z0, e[4]); L[2] = std::min(Sx.z1 - 1, e[5]);
        L[3] = std::max(Sx.x0, e[0]); L[4] = std::min(Sx.x1, e[1] - 1);
        // z faces: Ey, Ex; loops j then i
        L = d.lim[4 + side][0];
        L[0] = lo ? std::max(Sy.z0, e[4]) : std::min(Sy.z1, e[5]);
        L[1] = std::max(Sy.y0, e[2]); L[2] = std::min(Sy.y1, e[3] - 1);
        L[3] = std::max(Sy.x0, e[0]); L[4] = std::min(Sy.x1, e[1]);
        L = d.lim[4 + side][1];
        L[0] = lo ? std::max(Sx.z0, e[4]) : std::min(Sx.z1, e[5]);
        L[1] = std::max(Sx.y0, e[2]); L[2] = std::min(Sx.y1, e[3]);
        L[3] = std::max(Sx.x0, e[0]); L[4] = std::min(Sx.x1, e[1] - 1);
    }
    // :947-1036, the frequency list in real(4)
    const float fi = s->initial_freq, ff = s->final_freq, fs = s->freq_step;
    const int n = fs != 0.0f ? (int)(std::fabs(fi - ff) / fs) + 1 : 1;
    if (n < 1 || n > 100000) return sgpu::set_error(c, SGPU_ERR_ARG, "Freq. range for NF/FF invalid");
    std::vector<float> freq(n);
    if (s->logarithmic) {
        const float li = std::log10(fi), lf = std::log10(ff), step = std::fabs(li - lf) / (float)n;
        for (int q = 0; q < n; ++q) freq[q] = std::pow(10.0f, li + (float)q * step);
    } else {
        for (int q = 0; q < n; ++q) freq[q] = fi + (float)q * fs;
    }
    d.nfreq = n;
    d.freq = freq.data();
    // :194-199
    d.ndecim = s->decimate ? std::max((int)((double)(0.5f / ff) / h->dt) - 1, 1) : 1;
    d.dtdecim = (float)((double)d.ndecim * h->dt);
    d.cluz = h->cluz;
    d.zvac = h->zvac;
    const Vec* cells[6] = {&h->dxe, &h->dye, &h->dze, &h->dxh, &h->dyh, &h->dzh};
    for (int k = 0; k < 6; ++k) {
        d.cell[k] = cells[k]->v.data();
        d.cell_lo[k] = cells[k]->lo;
        d.cell_n[k] = (int)cells[k]->v.size();
    }
    for (int f = 0; f < 3; ++f)
        for (int a = 0; a < 3; ++a) {
            d.phys[f][a] = h->phys[f][a].data();
            d.phys_lo[f][a] = h->phys_lo[f][a];
            d.phys_n[f][a] = (int)h->phys[f][a].size();
        }
    return sgpu_add_farfield(c, &d, id);
}

sgpu_status sgpu_host_get_mur_cab1(const sgpu_ctx* c, int face, float* out) {
    if (!c || !c->host || face < 0 || face > 5 || !out) return SGPU_ERR_ARG;
    const HostState* h = (const HostState*)c->host;
    if (h->cab1[face].empty()) return SGPU_ERR_ARG;
    std::memcpy(out, h->cab1[face].data(), h->cab1[face].size() * sizeof(float));
    return SGPU_OK;
}

sgpu_status sgpu_host_get_media(const sgpu_ctx* c, int comp, int16_t* out) {
    if (!c || comp < 0 || comp > 5 || !out) return SGPU_ERR_ARG;
    sgpu_ctx* cc = const_cast<sgpu_ctx*>(c);
    if (c->host_only) {
        const HostState* h = (const HostState*)c->host;
        std::memcpy(out, h->mm[comp].data(), h->mm[comp].size() * sizeof(int16_t));
        return SGPU_OK;
    }
    const sgpu_lim& a = c->alloc[comp];
    cudaMemcpy3DParms prm{};
    size_t ax = a.xe - a.xi + 1, ay = a.ye - a.yi + 1, az = a.ze - a.zi + 1;
    prm.srcPtr = make_cudaPitchedPtr(c->M[comp], (size_t)c->pitch * 2, (size_t)c->nxa * 2, c->nya);
    prm.dstPtr = make_cudaPitchedPtr(out, ax * 2, ax * 2, ay);
    prm.extent = make_cudaExtent(ax * 2, ay, az);
    prm.kind = cudaMemcpyDeviceToHost;
    cudaError_t e = cudaMemcpy3DAsync(&prm, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return sgpu::set_error(cc, SGPU_ERR_CUDA, cudaGetErrorString(e));
    return SGPU_OK;
}

}  // extern "C"

sgpu_status sgpu::host_create_in(const sgpu_problem* p, sgpu_ctx* plan, int max_steps, Arena* arena, cudaStream_t stream,
                                 sgpu_ctx** out) {
    if (!out) return SGPU_ERR_ARG;
    *out = nullptr;
    HostState* h = nullptr;
    if (plan) {
        if (!plan->host_only || !plan->host) return SGPU_ERR_ARG;
        h = (HostState*)plan->host;
        plan->host = nullptr;  // the realized context owns it now
    } else {
        sgpu_status rc;
        h = make_plan(p, max_steps, &rc);
        if (!h) return rc;
    }
    if (arena) h->probe_cap = h->max_steps + 1;
    return realize(h, arena, stream, out);
}
