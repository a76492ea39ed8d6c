// Restart files: the records of the reference's flush_and_save_resume and of
// the resume branches of its Init* routines (resuming.F90:113-496,
// borderscpml.F90:348-371 and 481-558, bordersmur.F90:160-305 and 369-454,
// electricdispersive.F90:272-295 and 365-401, magneticdispersive.F90:364-400),
// as Fortran sequential unformatted records: the payload framed by its byte
// length as a 4-byte integer on both sides.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sgpu_internal.h"

using namespace sgpu;

namespace {

constexpr long long kBlock = 1024;  // BLOCK_SIZE of resuming.F90:104

struct Records {
    FILE* f = nullptr;
    bool write = false;
    std::string err;
    bool put(const void* p, size_t n) {
        const int32_t m = (int32_t)n;
        if (fwrite(&m, 4, 1, f) != 1 || (n && fwrite(p, 1, n, f) != n) || fwrite(&m, 4, 1, f) != 1) {
            err = "write failed";
            return false;
        }
        return true;
    }
    bool get(void* p, size_t n) {
        int32_t a = -1, b = -1;
        if (fread(&a, 4, 1, f) != 1) {
            err = "file ends before the expected record";
            return false;
        }
        if ((size_t)a != n) {
            err = "record of " + std::to_string(a) + " bytes where " + std::to_string(n) + " were expected";
            return false;
        }
        if ((n && fread(p, 1, n, f) != n) || fread(&b, 4, 1, f) != 1 || b != a) {
            err = "truncated or malformed record";
            return false;
        }
        return true;
    }
    // one record: write from p, or read into p
    bool rec(void* p, size_t n) { return write ? put(p, n) : get(p, n); }
};

template <class T> cudaError_t d2h(std::vector<T>& h, const T* d, size_t n) {
    h.resize(n);
    return n ? cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost) : cudaSuccess;
}
template <class T> cudaError_t h2d_sync(T* d, const std::vector<T>& h) {
    return h.empty() ? cudaSuccess : cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
}

#define RTRY(call)                                                                     \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) return set_error(c, SGPU_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)
#define RREC(p, n)                                                          \
    do {                                                                    \
        if (!r.rec((p), (n))) return set_error(c, SGPU_ERR_ARG, "resume file: " + r.err); \
    } while (0)

// StoreFields / ReadFields: each (j, k) row of a component's Alloc box in
// records of kBlock values and a remainder record.
sgpu_status fields(sgpu_ctx* c, Records& r) {
    std::vector<float> h;
    for (int f = 0; f < 6; ++f) {
        const sgpu_lim& a = c->alloc[f];
        const long long ax = a.xe - a.xi + 1, ay = a.ye - a.yi + 1, az = a.ze - a.zi + 1;
        h.assign((size_t)(ax * ay * az), 0.0f);
        if (r.write)
            RTRY(box_to_host(h.data(), c->F[f], sizeof(float), ax, ay, az, c->pitch, c->plane / c->pitch, c->stream));
        for (long long k = 0; k < az; ++k)
            for (long long j = 0; j < ay; ++j) {
                float* row = h.data() + ax * (j + ay * k);
                long long i = 0;
                for (; i + kBlock <= ax; i += kBlock) RREC(row + i, kBlock * sizeof(float));
                RREC(row + i, (ax - i) * sizeof(float));
            }
        if (!r.write)
            RTRY(box_to_device(c->F[f], h.data(), sizeof(float), ax, ay, az, c->pitch, c->plane / c->pitch, c->stream));
    }
    return SGPU_OK;
}

// StoreFieldsCPMLBorders: regions Left/Right (Psi_Exy, Psi_Ezy, Psi_Hxy,
// Psi_Hzy), Down/Up (Psi_Eyz, Psi_Exz, Psi_Hyz, Psi_Hxz), Back/Front
// (Psi_Ezx, Psi_Eyx, Psi_Hzx, Psi_Hyx); each array one record per (j, k) row
// of its PMLc box.  Slab [comp][kind]: the kinds of sgpu_internal.h.
sgpu_status cpml(sgpu_ctx* c, Records& r) {
    const int arrays[3][4][2] = {{{0, 0}, {2, 0}, {3, 0}, {5, 0}},
                                 {{1, 0}, {0, 1}, {4, 0}, {3, 1}},
                                 {{2, 1}, {1, 1}, {5, 1}, {4, 1}}};
    std::vector<float> h;
    for (int pair = 0; pair < 3; ++pair)
        for (int side = 0; side < 2; ++side)
            for (int q = 0; q < 4; ++q) {
                const Slab& s = c->cpml.s[arrays[pair][q][0]][arrays[pair][q][1]][side];
                if (!s.psi) continue;
                const long long ny = s.yhi - s.ylo + 1, nz = s.zhi - s.zlo + 1, n = (long long)s.px * ny * nz;
                if (r.write) RTRY(d2h(h, s.psi, (size_t)n));
                else h.assign((size_t)n, 0.0f);
                for (long long k = 0; k < nz; ++k)
                    for (long long j = 0; j < ny; ++j)
                        RREC(h.data() + (s.xlo - s.xb) + s.px * (j + ny * k), (s.xhi - s.xlo + 1) * sizeof(float));
                if (!r.write) RTRY(h2d_sync(s.psi, h));
            }
    return SGPU_OK;
}

// StoreFieldsMURBorders: per part (the store order of sgpu_init_borders) the
// MURc box -- the outer and the first swept layer over the component's sweep
// range of the other two axes -- one record per (j, k) row, the layers in
// increasing coordinate; then the same records of PastPast_, which stays zero.
sgpu_status mur(sgpu_ctx* c, Records& r) {
    std::vector<float> h, zero;
    for (int pass = 0; pass < 2; ++pass)
        for (int p = 0; p < c->border.nmur; ++p) {
            const MurPart& m = c->border.mur[p];
            const long long layer = (long long)m.nu * m.nv;
            if (pass == 0) {
                if (r.write) RTRY(d2h(h, m.past, (size_t)(2 * layer)));
                else h.assign((size_t)(2 * layer), 0.0f);
            }
            // layer index (0 outer, 1 inner) in increasing coordinate
            const int lay[2] = {m.outer < m.inner ? 0 : 1, m.outer < m.inner ? 1 : 0};
            std::vector<float>& src = pass == 0 ? h : zero;
            if (pass == 1) zero.assign((size_t)(2 * layer), 0.0f);
            auto at = [&](int l, long long v, long long u) { return &src[(size_t)(l * layer + v * m.nu + u)]; };
            if (m.axis == 0) {  // rows of two values (x the normal): k = v, j = u
                for (long long v = 0; v < m.nv; ++v)
                    for (long long u = 0; u < m.nu; ++u) {
                        float two[2] = {*at(lay[0], v, u), *at(lay[1], v, u)};
                        RREC(two, sizeof(two));
                        if (!r.write && pass == 0) {
                            *at(lay[0], v, u) = two[0];
                            *at(lay[1], v, u) = two[1];
                        }
                    }
            } else if (m.axis == 1) {  // y the normal: k = v, then the two layers, rows over x = u
                for (long long v = 0; v < m.nv; ++v)
                    for (int l = 0; l < 2; ++l) RREC(at(lay[l], v, 0), m.nu * sizeof(float));
            } else {  // z the normal: the two layers, then j = v, rows over x = u
                for (int l = 0; l < 2; ++l)
                    for (long long v = 0; v < m.nv; ++v) RREC(at(lay[l], v, 0), m.nu * sizeof(float));
            }
            if (!r.write && pass == 0) RTRY(h2d_sync(m.past, h));
        }
    return SGPU_OK;
}

// StoreFieldsEDispersives / StoreFieldsMDispersives: per medium (table
// order), per component, per node (k, j, i order): the previous field, then
// the current of each pole.  A pole folded onto an earlier one holds the
// conjugate of that pole's current.
sgpu_status dispersive(sgpu_ctx* c, Records& r, bool mag) {
    const KDisp& k = mag ? c->mdisp : c->disp;
    const std::vector<DispMedium>& media = c->h_disp_media[mag ? 1 : 0];
    if (!(mag ? c->mdisp_on : c->disp_on) || media.empty()) return SGPU_OK;
    std::vector<uint8_t> med[3];
    std::vector<float> prev[3];
    std::vector<double2> J[3];
    for (int comp = 0; comp < 3; ++comp) {
        const size_t n = (size_t)k.n[comp];
        RTRY(d2h(med[comp], k.med[comp], n));
        if (r.write) {
            RTRY(d2h(prev[comp], k.prev[comp], n));
            RTRY(d2h(J[comp], k.J[comp], n * k.nu_max));
        } else {
            prev[comp].assign(n, 0.0f);
            J[comp].assign(n * k.nu_max, make_double2(0.0, 0.0));
        }
    }
    for (size_t m = 0; m < media.size(); ++m) {
        const DispMedium& dm = media[m];
        bool first[kMaxPolesPerMedium] = {};
        for (int p = 0; p < dm.np; ++p) {
            first[p] = true;
            for (int q = 0; q < p; ++q)
                if (dm.map[q] == dm.map[p]) first[p] = false;
        }
        for (int comp = 0; comp < 3; ++comp) {
            const size_t n = med[comp].size();
            for (size_t q = 0; q < n; ++q) {
                if (med[comp][q] != m) continue;
                RREC(&prev[comp][q], sizeof(float));
                for (int p = 0; p < dm.np; ++p) {
                    double2& slot = J[comp][q * (size_t)std::max(1, k.nu_max) + dm.map[p]];
                    double v[2] = {slot.x, first[p] ? slot.y : -slot.y};
                    RREC(v, sizeof(v));
                    if (!r.write && first[p]) slot = make_double2(v[0], v[1]);
                }
            }
        }
    }
    if (!r.write)
        for (int comp = 0; comp < 3; ++comp) {
            RTRY(h2d_sync(k.prev[comp], prev[comp]));
            RTRY(h2d_sync(k.J[comp], J[comp]));
        }
    return SGPU_OK;
}

sgpu_status body(sgpu_ctx* c, Records& r) {
    sgpu_status s;
    if ((s = fields(c, r))) return s;
    if (c->cpml.on && (s = cpml(c, r))) return s;
    if (c->border.nmur > 0 && (s = mur(c, r))) return s;
    if ((s = dispersive(c, r, false))) return s;
    return dispersive(c, r, true);
}

#pragma pack(push, 1)
struct Header {
    int32_t n;
    double tiempo, dt;
    float eps0, mu0;
};
#pragma pack(pop)
static_assert(sizeof(Header) == 28, "the header record is 28 bytes");

}  // namespace

extern "C" {

sgpu_status sgpu_store_resume(sgpu_ctx* c, const char* path, int last_step, float eps0, float mu0) {
    if (!c || !path) return set_error(c, SGPU_ERR_ARG, "bad resume store");
    if (last_step < c->t_n0 || last_step >= c->t_n0 + (int)c->h_tiempo.size())
        return set_error(c, SGPU_ERR_ARG, "last step outside the time vector");
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return set_error(c, SGPU_ERR_CUDA, cudaGetErrorString(e));
    Records r;
    r.write = true;
    r.f = fopen(path, "wb");
    if (!r.f) return set_error(c, SGPU_ERR_ARG, std::string("cannot open ") + path);
    Header hd{last_step, c->h_tiempo[last_step - c->t_n0], c->dt, eps0, mu0};
    sgpu_status s = r.rec(&hd, sizeof(hd)) ? body(c, r) : set_error(c, SGPU_ERR_ARG, "resume file: " + r.err);
    if (fclose(r.f) != 0 && !s) s = set_error(c, SGPU_ERR_ARG, "resume file: close failed");
    return s;
}

sgpu_status sgpu_load_resume(sgpu_ctx* c, const char* path, int* last_step) {
    if (!c || !path) return set_error(c, SGPU_ERR_ARG, "bad resume load");
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return set_error(c, SGPU_ERR_CUDA, cudaGetErrorString(e));
    Records r;
    r.f = fopen(path, "rb");
    if (!r.f) return set_error(c, SGPU_ERR_ARG, std::string("cannot open ") + path);
    Header hd{};
    sgpu_status s = SGPU_OK;
    if (!r.rec(&hd, sizeof(hd))) s = set_error(c, SGPU_ERR_ARG, "resume file: " + r.err);
    else if (hd.dt != c->dt) s = set_error(c, SGPU_ERR_ARG, "resume file: its dt differs from the set-up's");
    else s = body(c, r);
    if (!s) {
        int extra = fgetc(r.f);
        if (extra != EOF) s = set_error(c, SGPU_ERR_ARG, "resume file: records left over (a different set-up)");
    }
    fclose(r.f);
    if (!s && last_step) *last_step = hd.n;
    if (!s) {
        // a resumed run starts with the plane-wave switch up
        // (timestepping.F90:1219): the next half step run is the first
        c->h_first = -1;
        c->src[0].h_first = c->src[1].h_first = -1;
        if (c->graph) {
            cudaGraphExecDestroy(c->graph);
            c->graph = nullptr;
        }
    }
    return s;
}

}  // extern "C"
