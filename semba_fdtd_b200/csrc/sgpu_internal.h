// Internal structures of libsemba_gpu.so (not part of the C ABI).
//
// Device layout: the six field components and the six media matrices share
// one padded box, the union of the components' sgg%Alloc ranges.  Local
// index l = absolute - origin on every axis, where origin is the common
// lower Alloc bound (-layers-1); a component whose Alloc range is one cell
// shorter simply leaves the last slab unused.  Rows are padded to a
// multiple of 32 floats so every row starts on a 128-byte boundary.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <vector>

#include "../../include/semba_gpu.h"

namespace sgpu {

constexpr int kMaxPolesPerMedium = 8;

// A CPML slab in local coordinates with its psi array: x fastest, rows from
// xb (xlo rounded down to a multiple of 4) with a pitch px (a multiple of 4
// floats), so a TMA box of the slab starts on a 16-byte boundary whenever
// the tile's x origin does.
struct Slab {
    int xlo, xhi, ylo, yhi, zlo, zhi;
    float* psi;
    int xb, px;
};

// Kernel view of the grid: fields, media, coefficient tables, metrics and
// the sweep boxes, all in local coordinates.
struct KGrid {
    float* F[6];
    const int16_t* M[6];
    const float *g1, *g2, *gm1, *gm2;
    const float *idxe, *idye, *idze, *idxh, *idyh, *idzh;
    int pitch;
    long long plane;
    int sw[6][6];  // [comp][xlo xhi ylo yhi zlo zhi]
    int nmed1;     // num_media + 1
};

// psi kinds, two per component in the order the reference applies them:
//   Ex: y(+) z(-)   Ey: z(+) x(-)   Ez: y(-) x(+)
//   Hx: y(-) z(+)   Hy: z(-) x(+)   Hz: y(+) x(-)
struct KCpml {
    const float *pbe[3], *pce[3], *pbm[3], *pcm[3];
    Slab s[6][2][2];  // [comp][which of the two][lo side, hi side]
    int on;
};

// Pole-residue media, electric or magnetic (folded conjugate pairs share one
// state).
struct DispMedium {
    int np;                       // poles of the reference
    int nu;                       // unique poles carrying state
    int map[kMaxPolesPerMedium];  // pole -> unique state slot
    double2 kappa[kMaxPolesPerMedium], beta[kMaxPolesPerMedium], g3[kMaxPolesPerMedium];
    double2 beta_dt[kMaxPolesPerMedium];  // Beta / dt, componentwise (the magnetic current's factor)
};

struct KDisp {
    const int* node[3];           // linear local index per node
    const uint8_t* med[3];        // dispersive-medium slot per node
    float* prev[3];
    double2* J[3];                // [node][unique slot], nu_max slots a node
    long long n[3];
    // per 32 consecutive nodes (a warp's worth): the group's nodes as at
    // most two runs of consecutive cells of one medium each -- x: cell of
    // lane 0's run start minus 0, y: cell of the second run's start minus its
    // first lane, z: that first lane (32: one run; negative: more than two
    // runs, read node[] and med[]), w: slot of run 0 | slot of run 1 << 8
    const int4* grp[3];
    const DispMedium* media;
    const int16_t* slot_of_medium;  // media index -> slot (-1 none)
    int nu_max;
    int uniform;  // every medium has nu_max state slots
    double dt;
    double inv_dt;  // RN(1/dt), for the corrected quotient by dt
};

// One source contribution applied after the curl/CPML/ADE work of a half
// step, in the reference's order (plane-wave faces, then nodal sources).
enum { kSrcPlaneWave = 0, kSrcNodalSoft = 1, kSrcNodalHard = 2 };
struct SrcEntry {
    int comp;
    int type;
    int table;
    float a, b, c;  // plane wave: a = d/c, b = fpw, c = +-Id ; soft: a = G2*I1*I2*amp ; hard: a = amp
};
struct SrcTable {
    int numus;
    float delta;
    int offset;  // into the concatenated samples
    int is_pw;
    // plane waves: per side (E, H), whether the wave has face nodes there and
    // the largest d/c over them, taken over the whole problem (a z slab keeps
    // only its own entries but switches off with the whole domain)
    int has[2];
    float amax[2];
};
struct KSrc {
    int nrows;
    const int* row_node;   // local linear index of each node
    const int* row_comp;
    const int* row_ptr;    // nrows + 1
    const SrcEntry* e;
    const SrcTable* tab;
    const float* samples;
    int ntab;
    int h_first;           // first half step 2n + side run since the start (or a resume)
    int pw_only;           // every contribution is a plane wave's: rows change nothing once the switch is down
};

// Borders of the H field outside the swept box (local coordinates).
// One Mur part is one (face, tangential H component) pair: its outer layer
// and first swept layer, over the component's sweep range of the other two
// axes (u the lower axis, v the higher), with Past_ of both layers.
struct MurPart {
    int comp;              // 3..5
    int axis;              // face normal
    int outer, inner;      // layer indices along the normal
    int u0, nu, v0, nv;
    float* past;           // [2][nv][nu]: outer layer, then inner layer
    const float* cab1;     // num_media + 1
    long long first;       // first cell in the flattened list
};
// One clone part is one (tangential H component, PMC or periodic face): the
// plane outside the face over the component's whole Alloc extent.
struct ClonePart {
    int comp;              // 0..2 for Hx..Hz
    int axis, side;
    long long first;
};
struct KBorder {
    int face_kind[3][2];   // [axis][side]: 2 PMC, 4 periodic, else 0
    // per H component (0..2) and axis: outer layers and swept ends
    int glo[3][3], ghi[3][3], slo[3][3], shi[3][3], alo[3][3], ahi[3][3];
    int ncl;
    ClonePart cl[12];
    long long cl_cells;
    int nmur;
    MurPart mur[12];
    long long mur_cells;
};

struct KProbes {
    int n;
    const int* comp;
    const long long* idx;
    float* ring;
    int cap;
};

// A volume probe: the sampled nodes (stride multiples of the box) of the
// E or H components; kind 0 accumulates the frequency-domain transform,
// kind 1 keeps time-domain frames in a ring.
struct VolProbe {
    int kind;
    int magnetic;
    int i0, j0, k0, ni, nj, nk;  // first sampled index and counts (stride units)
    int tr[3];
    // frequency domain: acc [nf][3][nk][nj][ni], weights [step - w_n0][nf]
    int nf;
    double2* acc;
    const double2* w;
    int w_n0, w_steps;
    // time domain: ring [cap][3][nk][nj][ni]
    int n_first, n_last, every, cap;
    float* ring;
};

// One near-to-far-field surface (farfield.cu).  A patch is one sampled
// array of a face: a component on one plane over two in-plane ranges;
// acc holds [nf][samples] complex(8), patch p at columns off .. off+n-1
// (inner index fastest).  The E / H weights of the m-th sampled step are
// wE / wH [m][nf].
struct FarPatch {
    int comp, axis, plane;  // sampled component, face normal axis, plane index
    int lo1, hi1, lo2, hi2;  // outer / inner in-plane ranges
    int off, n;
};
constexpr int kFarPatches = 36;  // 6 faces x 6 arrays
struct FarField {
    int nf = 0, ndecim = 1, npatch = 0, samples = 0, w_m = 0;
    int face_patch[6][6];  // patch index per face and slot, -1 if the face is off
    FarPatch patch[kFarPatches];
    double2* acc = nullptr;
    double2* wE = nullptr;
    double2* wH = nullptr;
    // transform inputs kept on the host
    int active[6];
    std::vector<float> freq;
    float cluz = 0, zvac = 0;
    std::vector<float> cell[6];
    int cell_lo[6];
    std::vector<float> phys[3][3];
    int phys_lo[3][3];
};

// Tensor maps of one fused TMA kernel (see tma_fields.cuh for the order).
struct alignas(64) TMaps {
    CUtensorMap m[21];  // 9 field / media maps, then the 12 psi slabs of the side
};

struct StepRef {
    const int* dev_n;  // if non-null, the step index is read from here
    int n;
};

// Device memory arena of a batch (batch.cu): contexts created inside a batch
// take every device buffer from it instead of cudaMalloc.
struct Arena;
void* arena_alloc(Arena* a, size_t bytes);
void arena_free(Arena* a, void* p);

}  // namespace sgpu

struct sgpu_ctx {
    std::string err;
    cudaStream_t stream = nullptr;
    bool own_stream = true;          // false inside a batch (the batch's stream)
    sgpu::Arena* arena = nullptr;    // non-null inside a batch
    int device = 0;
    // geometry
    sgpu_lim alloc[6], sweep[6];
    int ox = 0, oy = 0, oz = 0;
    int nxa = 0, nya = 0, nza = 0;
    int pitch = 0;
    long long plane = 0, vol = 0;
    int num_media = 0;
    double dt = 0;
    // device buffers
    float* F[6] = {};
    int16_t* M[6] = {};
    // the media matrices again as one byte a cell, the copy the TMA-pipelined
    // field kernels stream (they run only while num_media < 256)
    uint8_t* M8[6] = {};
    float *g1 = nullptr, *g2 = nullptr, *gm1 = nullptr, *gm2 = nullptr;
    float *idxe = nullptr, *idye = nullptr, *idze = nullptr, *idxh = nullptr, *idyh = nullptr, *idzh = nullptr;
    std::vector<float> h_g1, h_g2, h_gm1, h_gm2;
    std::vector<uint8_t> h_pec;
    std::vector<float> h_idxe, h_idye, h_idze, h_idxh, h_idyh, h_idzh;  // local-indexed
    bool media_loaded[6] = {};
    // CPML
    sgpu::KCpml cpml{};
    std::vector<void*> cpml_allocs;
    // ADE: electric (disp) and magnetic (mdisp) pole-residue media
    bool disp_on = false, mdisp_on = false;
    sgpu::KDisp disp{}, mdisp{};
    std::vector<sgpu::DispMedium> h_disp_media[2];  // host copies of the media tables [electric, magnetic]
    std::vector<void*> disp_allocs, mdisp_allocs;
    long long disp_irregular[2][3] = {};  // node groups of more than two runs [electric, magnetic][component]
    // borders (PMC / periodic clones, Mur)
    sgpu::KBorder border{};
    std::vector<void*> border_allocs;
    // sources
    struct HostSrcTable {
        std::vector<float> samples;
        int numus;
        float delta;
        int is_pw;
        int has[2] = {0, 0};
        float amax[2] = {0.0f, 0.0f};
    };
    std::vector<HostSrcTable> src_tables;
    struct HostEntry {
        long long node;
        int comp;
        int order;  // sequence number (reference order)
        sgpu::SrcEntry e;
    };
    std::vector<HostEntry> src_host[2];  // [E side, H side]
    sgpu::KSrc src[2]{};
    std::vector<void*> src_allocs[2];
    bool src_dirty = true;
    int src_seq = 0;
    int h_first = -1;  // first half step 2n + side launched (-1: none yet)
    // time
    std::vector<double> h_tiempo;
    int t_n0 = 0;
    double* d_tiempo = nullptr;
    int d_tiempo_count = 0;
    int* d_step = nullptr;
    // probes
    sgpu::KProbes probes{};
    std::vector<void*> probe_allocs;
    long long probe_written = 0;  // rows written in total
    long long probe_read = 0;
    int probe_first_n = -1;
    // volume probes; steps_hi: one past the last step whose probes were launched
    std::vector<sgpu::VolProbe> vprobes;
    std::vector<sgpu::FarField> farfields;
    std::vector<long long> vprobe_read;  // movie frames read so far, per probe
    std::vector<void*> vprobe_allocs;
    int steps_hi = -1;
    // graph
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    // scratch
    unsigned int* d_flag = nullptr;
    // TMA-pipelined fused kernels: tensor maps and the bounded-wait error word
    sgpu::TMaps tme{}, tmh{};
    bool tma_ready = false;
    int family = 1;  // 1: TMA-pipelined fused kernels when available, 0: register-marching kernels
    int* d_err = nullptr;
    long long wait_cycles = 4000000000LL;  // bound of a pipeline wait (clock cycles, ~2 s)
    int wait_drill = 0;                    // failure drill: producers issue no loads
    // a z-slab sub-domain (sgpu_host_create_zslab): sources are kept only on
    // the planes this context sweeps
    bool zslab = false;
    // level-2 host data kept for inspection; host_only contexts (from
    // sgpu_host_plan) own no device resources
    bool host_only = false;
    void* host = nullptr;
    void (*host_free)(void*) = nullptr;
};

namespace sgpu {
sgpu_status set_error(sgpu_ctx* c, sgpu_status code, const std::string& msg);
KGrid kgrid(const sgpu_ctx* c);
// sgpu_create with an optional arena and an external stream (batches).
sgpu_status create_in(const sgpu_grid_desc* d, Arena* arena, cudaStream_t stream, sgpu_ctx** out);
// sgpu_host_create into an arena/stream; `plan` (from sgpu_host_plan) is
// consumed when non-null, else the problem is planned first.  Inside an
// arena every probe keeps its whole trace (nsteps + 1 rows).
sgpu_status host_create_in(const sgpu_problem* p, sgpu_ctx* plan, int max_steps, Arena* arena, cudaStream_t stream,
                           sgpu_ctx** out);
// UpdateFarField for every far field of the context (farfield.cu).
sgpu_status launch_farfields(sgpu_ctx* c, StepRef sr);
void free_farfields(sgpu_ctx* c);
// sgpu_upload_media, with the range check of the indices optional (the
// host set-up's own matrices are in range by construction).
sgpu_status upload_media(sgpu_ctx* c, int comp, const int16_t* mi, bool check);
// Source lists built on the device now (normally built lazily before the
// first launch that needs them).
sgpu_status rebuild_sources(sgpu_ctx* c);
// Copies between a compact column-major box of ax x ay x az elements of es
// bytes in host memory and the same box at the origin of a padded device
// array (rows of `pitch` elements, `rows` rows per plane), on stream `st`,
// through pinned staging (transfer.cu); synchronous.
cudaError_t box_to_device(void* dev, const void* host, size_t es, long long ax, long long ay, long long az, int pitch,
                          long long rows, cudaStream_t st);
cudaError_t box_to_host(void* host, const void* dev, size_t es, long long ax, long long ay, long long az, int pitch,
                        long long rows, cudaStream_t st);
// Refresh the one-byte copy of media matrix comp (after it changed).
sgpu_status narrow_media(sgpu_ctx* c, int comp);
// Whether the TMA-pipelined field kernels can run (tensor maps built and
// every medium index fits the one-byte media copy).
bool tma_usable(const sgpu_ctx* c);
// Tell the device's default memory pool to keep freed memory (once per
// device): the solo contexts and the batch arena allocate from it.
void keep_device_pool(int device);
// Replace the context's medium count and coefficient tables (before the
// first launch): the level-2 host learns the final count only after the
// media matrices are built on the device.
sgpu_status set_media_tables(sgpu_ctx* c, int num_media, const float* g1, const float* g2, const float* gm1,
                             const float* gm2, const uint8_t* is_pec);
// Media matrices built on the device (paint.cu); coordinates absolute,
// boxes inclusive as {x0, x1, y0, y1, z0, z1}.
struct DevicePainter;
DevicePainter* painter_new(sgpu_ctx* c);
void painter_delete(DevicePainter* p);
sgpu_status painter_start(DevicePainter* p, const std::vector<int>& prio);
sgpu_status painter_paint(DevicePainter* p, const std::vector<int>& items7, int idx, int pr);
sgpu_status painter_extrude(DevicePainter* p, int f, const int* r6, int axis, int lo_end, int hi_beg, int lo_src,
                            int hi_src);
sgpu_status painter_first(DevicePainter* p, const std::vector<long long>& task0, const int (*r6)[6], const int (*in6)[6],
                          long long nyo, long long nxo, int nmed1, std::vector<long long>& first);
sgpu_status painter_relabel(DevicePainter* p, const int (*r6)[6], const int (*in6)[6], const std::vector<int16_t>& copy_of);
sgpu_status painter_zero(DevicePainter* p, int f, const int* b6);
sgpu_status painter_finish(DevicePainter* p);
// fn(lo, hi) over [0, n) split across up to 8 host threads, each taking at
// least `grain` units.
void host_parallel(long long n, const std::function<void(long long, long long)>& fn, long long grain = 2048);
}  // namespace sgpu
