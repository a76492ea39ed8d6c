// Media matrices built on the device.
//
// The level-2 host (host_setup.cpp) builds the six int16 media matrices of
// a problem -- read_geomData's region painting (CreateVolumeMM,
// healer.F90:66-243) and CreatePMLmatrix's extrusion across the PML
// (healer.F90:961-1420) with the PEC borders (:1442-1617).  For a problem set
// up alone (sgpu_host_create) the same steps run here on the device arrays
// the context owns, so neither the host painting of ~2 GB of int16 at 512^3
// nor its upload is needed.  The host keeps the decisions that need the
// whole picture (which regions, in what order, which copies of media the PML
// needs and their numbering); every kernel is a per-cell map over a box:
//
//   paint:    cell = idx where the region's priority beats the cell's
//             (E nodes: higher, H nodes: not lower), for all boxes of one
//             region in one launch -- boxes of one region share idx and
//             priority, so overlapping boxes write the same value;
//   extrude:  cells of the PML shell take -|medium| of the first or last
//             inner cell along x, then y (whole x reach), then z (whole x-y
//             reach): three launches, each reading only cells the previous
//             ones finished;
//   first:    for each negative entry, the smallest key of the host's sweep
//             order (component, plane, row, cell) at which it appears;
//   relabel:  negative entries become the numbers the host gave the copies;
//   zero:     medium 0 on the PEC boundary planes.
#include <cuda_runtime.h>

#include <vector>

#include "sgpu_internal.h"

#define PAINT_TRY(ctx, call)                                                                            \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return set_error((ctx), SGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace sgpu {
namespace {

struct PBox {
    int x0, x1, y0, y1, z0, z1;
};

struct PaintItem {
    int comp;
    PBox b;  // absolute, inclusive
};

struct Local {
    int ox, oy, oz, pitch;
    long long plane;
    __device__ __forceinline__ long long at(int i, int j, int k) const {
        return (long long)(i - ox) + (long long)pitch * (j - oy) + plane * (long long)(k - oz);
    }
};

__device__ __forceinline__ long long box_cells(const PBox& b) {
    return (long long)(b.x1 - b.x0 + 1) * (b.y1 - b.y0 + 1) * (b.z1 - b.z0 + 1);
}

__device__ __forceinline__ void box_cell(const PBox& b, long long q, int& i, int& j, int& k) {
    const long long nx = b.x1 - b.x0 + 1, ny = b.y1 - b.y0 + 1;
    i = b.x0 + (int)(q % nx);
    j = b.y0 + (int)((q / nx) % ny);
    k = b.z0 + (int)(q / (nx * ny));
}

// One region: every (box, component) item; blockIdx.y walks the items.
__global__ void k_paint(int16_t* const* M, Local L, const PaintItem* items, int nitems, const int* prio, int idx, int pr) {
    for (int it = blockIdx.y; it < nitems; it += gridDim.y) {
        const PaintItem w = items[it];
        const long long n = box_cells(w.b);
        const bool electric = w.comp < 3;
        int16_t* m = M[w.comp];
        for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
            int i, j, k;
            box_cell(w.b, q, i, j, k);
            const long long c = L.at(i, j, k);
            const int cur = prio[m[c]];
            if (electric ? pr > cur : pr >= cur) m[c] = (int16_t)idx;
        }
    }
}

__device__ __forceinline__ int16_t neg16(int16_t v) { return (int16_t)(v < 0 ? v : -v); }

// The PML extrusion of one component along one axis: the cells of `r`
// below `lo_end` (a < lo_end) take the cell at lo_src, those at or above
// `hi_beg` the cell at hi_src, along axis `axis`, negated.
__global__ void k_extrude(int16_t* m, Local L, PBox r, int axis, int lo_end, int hi_beg, int lo_src, int hi_src) {
    const long long n = box_cells(r);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int p[3];
        box_cell(r, q, p[0], p[1], p[2]);
        const int a = p[axis];
        if (a < lo_end) p[axis] = lo_src;
        else if (a >= hi_beg) p[axis] = hi_src;
        else continue;
        const int16_t v = neg16(m[L.at(p[0], p[1], p[2])]);
        int s[3];
        box_cell(r, q, s[0], s[1], s[2]);
        m[L.at(s[0], s[1], s[2])] = v;
    }
}

__device__ __forceinline__ bool in_shell(int i, int j, int k, const PBox& in) {
    return k < in.z0 || k > in.z1 || j < in.y0 || j > in.y1 || i < in.x0 || i > in.x1;
}

// Smallest sweep key of every negative entry of the shell of r (outside `in`).
// The key grows with q (nxo, nyo cover the box), so within a warp the lowest
// lane holding a value has that value's smallest key: one lane per distinct
// value records it, and only when it beats what is already there (the shell
// is mostly one or two values, which would otherwise serialise on a handful
// of addresses).
__global__ void k_first(const int16_t* m, Local L, PBox r, PBox in, long long task0, long long nyo, long long nxo,
                        unsigned long long* first) {
    const long long n = box_cells(r);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        box_cell(r, q, i, j, k);
        const int v = in_shell(i, j, k, in) ? (int)m[L.at(i, j, k)] : 0;
        const unsigned long long key =
            (unsigned long long)(((task0 + (k - r.z0)) * nyo + (j - r.y0)) * nxo + (i - r.x0));
        const unsigned act = __activemask();
        const unsigned want = __ballot_sync(act, v < 0);
        if (v < 0) {
            const unsigned grp = __match_any_sync(want, v);
            if ((int)(threadIdx.x & 31) == __ffs(grp) - 1 && key < *(volatile unsigned long long*)(first + (-v)))
                atomicMin(first + (-v), key);
        }
    }
}

__global__ void k_relabel(int16_t* m, Local L, PBox r, PBox in, const int16_t* copy_of) {
    const long long n = box_cells(r);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        box_cell(r, q, i, j, k);
        if (!in_shell(i, j, k, in)) continue;
        const long long c = L.at(i, j, k);
        const int v = m[c];
        if (v < 0) m[c] = copy_of[-v];
    }
}

__global__ void k_zero_box(int16_t* m, Local L, PBox b) {
    const long long n = box_cells(b);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        m[L.at(i, j, k)] = 0;
    }
}

__global__ void k_fill_all(int16_t* m, long long n, int16_t v) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        m[q] = v;
}

unsigned blocks_for(long long n) { return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16)); }

}  // namespace

// Device media painting, driven by host_setup.cpp.  Coordinates are
// absolute; boxes are inclusive.  All work goes on the context's stream.
struct DevicePainter {
    sgpu_ctx* c;
    Local L;
    int16_t** d_M = nullptr;  // device copy of the six array pointers
    int* d_prio = nullptr;
    std::vector<void*> scratch;

    explicit DevicePainter(sgpu_ctx* ctx) : c(ctx) {
        L = Local{c->ox, c->oy, c->oz, c->pitch, c->plane};
    }
    ~DevicePainter() {
        cudaStreamSynchronize(c->stream);
        for (void* p : scratch) cudaFree(p);
    }
    template <class T> sgpu_status alloc(T** p, size_t n) {
        if (cudaMalloc((void**)p, n * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            return set_error(c, SGPU_ERR_OOM, "device media painting: out of memory");
        }
        scratch.push_back(*p);
        return SGPU_OK;
    }
    sgpu_status check(const char* what) {
        const cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? SGPU_OK : set_error(c, SGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
    // medium 1 everywhere (the padding of the common box included), and the
    // priority of every medium the regions paint
    sgpu_status start(const std::vector<int>& prio) {
        sgpu_status s;
        if ((s = alloc(&d_M, 6)) || (s = alloc(&d_prio, prio.size()))) return s;
        PAINT_TRY(c, cudaMemcpyAsync(d_M, c->M, 6 * sizeof(int16_t*), cudaMemcpyHostToDevice, c->stream));
        PAINT_TRY(c, cudaMemcpyAsync(d_prio, prio.data(), prio.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        for (int f = 0; f < 6; ++f) k_fill_all<<<blocks_for(c->vol), 256, 0, c->stream>>>(c->M[f], c->vol, 1);
        // the pointer and priority uploads read host memory that must outlive them
        PAINT_TRY(c, cudaStreamSynchronize(c->stream));
        return check("k_fill_all");
    }
    // items: (comp, x0, x1, y0, y1, z0, z1) per (box, component) of one region
    sgpu_status paint(const std::vector<int>& items7, int idx, int pr) {
        const int n = (int)(items7.size() / 7);
        if (n == 0) return SGPU_OK;
        std::vector<PaintItem> it(n);
        long long most = 0;
        for (int q = 0; q < n; ++q) {
            const int* v = &items7[7 * q];
            it[q] = PaintItem{v[0], PBox{v[1], v[2], v[3], v[4], v[5], v[6]}};
            most = std::max<long long>(most, (long long)(v[2] - v[1] + 1) * (v[4] - v[3] + 1) * (v[6] - v[5] + 1));
        }
        PaintItem* d = nullptr;
        sgpu_status s = alloc(&d, it.size());
        if (s) return s;
        PAINT_TRY(c, cudaMemcpyAsync(d, it.data(), it.size() * sizeof(PaintItem), cudaMemcpyHostToDevice, c->stream));
        const dim3 grid((unsigned)std::max<long long>(1, std::min<long long>((most + 255) / 256, 1024)),
                        (unsigned)std::min(n, 65535));
        k_paint<<<grid, 256, 0, c->stream>>>(d_M, L, d, n, d_prio, idx, pr);
        PAINT_TRY(c, cudaStreamSynchronize(c->stream));  // `it` is a local
        return check("k_paint");
    }
    sgpu_status extrude(int f, const int* r6, int axis, int lo_end, int hi_beg, int lo_src, int hi_src) {
        const PBox r{r6[0], r6[1], r6[2], r6[3], r6[4], r6[5]};
        if (r.x1 < r.x0 || r.y1 < r.y0 || r.z1 < r.z0) return SGPU_OK;
        const long long n = (long long)(r.x1 - r.x0 + 1) * (r.y1 - r.y0 + 1) * (r.z1 - r.z0 + 1);
        k_extrude<<<blocks_for(n), 256, 0, c->stream>>>(c->M[f], L, r, axis, lo_end, hi_beg, lo_src, hi_src);
        return check("k_extrude");
    }
    sgpu_status first_keys(int f, const int* r6, const int* in6, long long task0, long long nyo, long long nxo,
                           unsigned long long* d_first) {
        const PBox r{r6[0], r6[1], r6[2], r6[3], r6[4], r6[5]}, in{in6[0], in6[1], in6[2], in6[3], in6[4], in6[5]};
        if (r.x1 < r.x0 || r.y1 < r.y0 || r.z1 < r.z0) return SGPU_OK;
        const long long n = (long long)(r.x1 - r.x0 + 1) * (r.y1 - r.y0 + 1) * (r.z1 - r.z0 + 1);
        k_first<<<blocks_for(n), 256, 0, c->stream>>>(c->M[f], L, r, in, task0, nyo, nxo, d_first);
        return check("k_first");
    }
    sgpu_status relabel(int f, const int* r6, const int* in6, const int16_t* d_copy) {
        const PBox r{r6[0], r6[1], r6[2], r6[3], r6[4], r6[5]}, in{in6[0], in6[1], in6[2], in6[3], in6[4], in6[5]};
        if (r.x1 < r.x0 || r.y1 < r.y0 || r.z1 < r.z0) return SGPU_OK;
        const long long n = (long long)(r.x1 - r.x0 + 1) * (r.y1 - r.y0 + 1) * (r.z1 - r.z0 + 1);
        k_relabel<<<blocks_for(n), 256, 0, c->stream>>>(c->M[f], L, r, in, d_copy);
        return check("k_relabel");
    }
    sgpu_status zero(int f, const int* b6) {
        const PBox b{b6[0], b6[1], b6[2], b6[3], b6[4], b6[5]};
        if (b.x1 < b.x0 || b.y1 < b.y0 || b.z1 < b.z0) return SGPU_OK;
        const long long n = (long long)(b.x1 - b.x0 + 1) * (b.y1 - b.y0 + 1) * (b.z1 - b.z0 + 1);
        k_zero_box<<<blocks_for(n), 256, 0, c->stream>>>(c->M[f], L, b);
        return check("k_zero_box");
    }
};

DevicePainter* painter_new(sgpu_ctx* c) { return new DevicePainter(c); }
void painter_delete(DevicePainter* p) { delete p; }
sgpu_status painter_start(DevicePainter* p, const std::vector<int>& prio) { return p->start(prio); }
sgpu_status painter_paint(DevicePainter* p, const std::vector<int>& items7, int idx, int pr) { return p->paint(items7, idx, pr); }
sgpu_status painter_extrude(DevicePainter* p, int f, const int* r6, int axis, int lo_end, int hi_beg, int lo_src,
                            int hi_src) {
    return p->extrude(f, r6, axis, lo_end, hi_beg, lo_src, hi_src);
}
sgpu_status painter_first(DevicePainter* p, const std::vector<long long>& task0, const int (*r6)[6], const int (*in6)[6],
                          long long nyo, long long nxo, int nmed1, std::vector<long long>& first) {
    unsigned long long* d = nullptr;
    sgpu_status s = p->alloc(&d, (size_t)nmed1);
    if (s) return s;
    PAINT_TRY(p->c, cudaMemsetAsync(d, 0xff, (size_t)nmed1 * sizeof(unsigned long long), p->c->stream));
    for (int f = 0; f < 6; ++f)
        if ((s = p->first_keys(f, r6[f], in6[f], task0[f], nyo, nxo, d))) return s;
    std::vector<unsigned long long> h((size_t)nmed1);
    PAINT_TRY(p->c, cudaMemcpyAsync(h.data(), d, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, p->c->stream));
    PAINT_TRY(p->c, cudaStreamSynchronize(p->c->stream));
    first.assign((size_t)nmed1, 0);
    for (int v = 0; v < nmed1; ++v) first[v] = h[v] == ~0ULL ? -1 : (long long)h[v];
    return SGPU_OK;
}
sgpu_status painter_relabel(DevicePainter* p, const int (*r6)[6], const int (*in6)[6], const std::vector<int16_t>& copy_of) {
    int16_t* d = nullptr;
    sgpu_status s = p->alloc(&d, copy_of.size());
    if (s) return s;
    PAINT_TRY(p->c, cudaMemcpyAsync(d, copy_of.data(), copy_of.size() * sizeof(int16_t), cudaMemcpyHostToDevice, p->c->stream));
    for (int f = 0; f < 6; ++f)
        if ((s = p->relabel(f, r6[f], in6[f], d))) return s;
    PAINT_TRY(p->c, cudaStreamSynchronize(p->c->stream));  // copy_of is the caller's
    return SGPU_OK;
}
sgpu_status painter_zero(DevicePainter* p, int f, const int* b6) { return p->zero(f, b6); }
sgpu_status painter_finish(DevicePainter* p) {
    for (int f = 0; f < 6; ++f) {
        const sgpu_status s = narrow_media(p->c, f);
        if (s) return s;
    }
    PAINT_TRY(p->c, cudaStreamSynchronize(p->c->stream));
    for (int f = 0; f < 6; ++f) p->c->media_loaded[f] = true;
    p->c->src_dirty = true;
    return SGPU_OK;
}

}  // namespace sgpu
