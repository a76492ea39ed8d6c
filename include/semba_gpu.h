/*
 * semba_gpu.h -- C ABI of libsemba_gpu.so, the B200 (sm_100a) implementation
 * of semba-fdtd's Yee leapfrog core: E/H curl updates, CPML psi updates,
 * electric pole-residue ADE, plane-wave TF/SF and nodal sources, with point
 * probes.  Plain pointers and sizes only; no CUDA or torch types.
 *
 * Two levels:
 *
 *  1. The drop-in for the reference's per-step routines.  The Fortran host
 *     keeps its set-up (findbounds, calc_G1G2Gm1Gm2, InitCPMLBorders,
 *     InitEDispersives, InitPlaneWave, InitNodalSources) and hands the arrays
 *     it built to sgpu_create / sgpu_init_*; every Advance_* routine of the
 *     time loop then maps to one sgpu_advance_* call.  The field, media and
 *     coefficient arrays are passed exactly as the Fortran host holds them
 *     (column-major over sgg%Alloc, re-based to 0), so a bind(C) interface
 *     can pass them without copies (semba_gpu_m.F90 beside this header is
 *     that interface).
 *
 *  2. A problem-level host (sgpu_host_*) that restates, in C++, the set-up
 *     of launch_simulation from an NFDE-style problem description (grid,
 *     CPML, materials, plane waves, nodal sources, probes) and then drives
 *     level 1.  This is the caller used by the Python package, the tests and
 *     the benchmark in this repository.
 *
 * Coordinates are the reference's absolute cell indices (sgg%Alloc ranges,
 * which start at -layers-1).  Field components are numbered 0..5 for
 * Ex, Ey, Ez, Hx, Hy, Hz (iEx..iHz of fdetypes.F90:190, minus one).
 *
 * Every entry point returns SGPU_OK (0) or an error code; the text of the
 * last error of a context is available from sgpu_last_error.  A context is
 * not thread-safe: use one context per host thread.  Device work of a
 * context is issued on its own CUDA stream; sgpu_synchronize waits for it.
 */
#ifndef SEMBA_GPU_H
#define SEMBA_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int sgpu_status;
#define SGPU_OK 0
#define SGPU_ERR_ARG 1        /* bad argument or extent                     */
#define SGPU_ERR_OOM 2        /* device or host allocation failed           */
#define SGPU_ERR_CUDA 3       /* CUDA runtime error                         */
#define SGPU_ERR_STATE 4      /* call out of order (e.g. advance before set-up) */
#define SGPU_ERR_NONFINITE 5  /* NaN/Inf found by sgpu_check_finite         */
#define SGPU_ERR_TIMEOUT 6    /* a bounded device wait ran out              */
#define SGPU_ERR_UNSUPPORTED 7
#define SGPU_ERR_SIZE 8       /* input larger than the entry point's stated maximum */

typedef struct sgpu_ctx sgpu_ctx;

typedef struct { int xi, xe, yi, ye, zi, ze; } sgpu_lim;

/* ======================================================================== */
/* Level 1: drop-in for the per-step routines                               */
/* ======================================================================== */

/* Grid, coefficient tables and metric arrays, as built by launch_simulation
 * (timestepping.F90:305-370, :565) and findbounds (timestepping.F90:2883).
 * Replaces the field/metric allocation of timestepping.F90:375-403. */
typedef struct {
    sgpu_lim alloc[6];   /* sgg%Alloc(iEx..iHz)                               */
    sgpu_lim sweep[6];   /* sgg%Sweep(iEx..iHz)                               */
    int num_media;       /* sgg%NumMedia; tables hold num_media+1 entries     */
    const float* g1;     /* G1, G2, GM1, GM2 of calc_G1G2Gm1Gm2 after         */
    const float* g2;     /*   InitEDispersives has overwritten the dispersive */
    const float* gm1;    /*   media (calc_constants.F90:36-148,               */
    const float* gm2;    /*   electricdispersive.F90:140-142)                 */
    const uint8_t* is_pec; /* sgg%Med(r)%Is%PEC, used by nodal sources        */
    /* Inverse steps after calc_cpmlconstants has stretched them in the PML:
     * idxe over alloc[Hx].x, idye over alloc[Hy].y, idze over alloc[Hz].z,
     * idxh over alloc[Ex].x, idyh over alloc[Ey].y, idzh over alloc[Ez].z. */
    const float *idxe, *idye, *idze, *idxh, *idyh, *idzh;
    double dt;           /* sgg%dt                                            */
} sgpu_grid_desc;

/* On failure *out may hold a context whose sgpu_last_error explains the
 * failure; destroy it. */
sgpu_status sgpu_create(const sgpu_grid_desc* grid, sgpu_ctx** out);
void sgpu_destroy(sgpu_ctx* ctx);
const char* sgpu_last_error(const sgpu_ctx* ctx);
sgpu_status sgpu_synchronize(sgpu_ctx* ctx);
/* The CUDA stream (a cudaStream_t, passed as a pointer) on which the context
 * issues every launch and copy: a caller orders its own device work against
 * the context's on it (a z-slab halo message, say) without a host wait.
 * No reference counterpart (the reference's routines are synchronous). */
sgpu_status sgpu_get_stream(const sgpu_ctx* ctx, void** stream);

/* Media matrices sggMiEx..sggMiHz (int16, -DCompileWithInt2), column-major
 * over alloc[comp]. */
sgpu_status sgpu_upload_media(sgpu_ctx* ctx, int comp, const int16_t* mi);
/* Field arrays Ex..Hz, column-major over alloc[comp].  Host arrays the
 * driver has pinned (sgpu_pinned_alloc, cudaHostAlloc, cudaHostRegister) are
 * copied directly by the copy engine; others go through the library's
 * pinned staging buffers. */
sgpu_status sgpu_upload_field(sgpu_ctx* ctx, int comp, const float* f);
sgpu_status sgpu_download_field(sgpu_ctx* ctx, int comp, float* f);
/* Page-locked host memory for such arrays (cudaHostAlloc, portable). */
sgpu_status sgpu_pinned_alloc(uint64_t bytes, void** out);
sgpu_status sgpu_pinned_free(void* p);

/* InitCPMLBorders (borderscpml.F90:90-473): the PMLc boxes of the six slab
 * regions per component and the coefficient vectors of calc_cpmlconstants.
 * Region order Down, Up, Left, Right, Back, Front (fdetypes.F90:186).  An
 * absent face has an empty box.  p_be[a], p_ce[a], p_bm[a], p_cm[a] cover
 * alloc[Hx].x (a=0), alloc[Hy].y (a=1), alloc[Hz].z (a=2). */
typedef struct {
    sgpu_lim pmlc[6][6]; /* [component][region] */
    const float *p_be[3], *p_ce[3], *p_bm[3], *p_cm[3];
} sgpu_cpml_desc;
sgpu_status sgpu_init_cpml(sgpu_ctx* ctx, const sgpu_cpml_desc* d);

/* InitEDispersives (electricdispersive.F90:77-298): for each electric
 * dispersive medium its index and the complex(8) Kappa, Beta and G3 of each
 * pole (interleaved re, im; poles of all media concatenated).  The node
 * lists of the reference are rebuilt on the device from the media matrices
 * (every swept E node whose medium is in the list); their state starts at
 * zero as on a fresh start. */
typedef struct {
    int nmedia;
    const int* medium_index;   /* [nmedia] */
    const int* npoles;         /* [nmedia] */
    const double* kappa;       /* [2 * sum(npoles)] */
    const double* beta;
    const double* g3;
} sgpu_edisp_desc;
sgpu_status sgpu_init_edisp(sgpu_ctx* ctx, const sgpu_edisp_desc* d);
/* InitMdispersives (magneticdispersive.F90:79-289): the same description for
 * the magnetic pole-residue media (Kappa, Beta, GM3); the node lists are the
 * swept H nodes of those media. */
sgpu_status sgpu_init_mdisp(sgpu_ctx* ctx, const sgpu_edisp_desc* d);

/* InitPlaneWave (planewaves.F90:72-770) + calc_planewaveconstants
 * (:1494-1510) for one plane wave (one mode).  face[] holds, per face
 * (0..5 = back, front, left, right, down, up), the flag Ilumina* and per
 * component the limits of TrFr / IzDe / AbAr:
 *   lim[face][comp] = {fixed index, lo1, hi1, lo2, hi2}
 * where the two ranges are the varying coordinates in loop order
 * (k then j for back/front, k then i for left/right, j then i for down/up).
 * phys[comp][axis] are Punto%PhysCoor over sweep-1 .. sweep+1. */
typedef struct {
    int active[6];
    int lim[6][6][5];
    float px, py, pz, d0, cluz;
    float fpw[6];
    int numus;
    float deltaevol;
    const float* evol;          /* numus + 1 samples */
    const float* phys[6][3];
    int phys_lo[6][3];
    int phys_n[6][3];
} sgpu_planewave_desc;
sgpu_status sgpu_add_planewave(sgpu_ctx* ctx, const sgpu_planewave_desc* d);

/* InitNodalSources (nodalsources.F90:76-300): one clipped point box of one
 * component. */
typedef struct {
    int comp;                   /* 0..5 */
    int hard;
    sgpu_lim box;
    float amplitude;
    int numus;
    float deltaevol;
    const float* evol;
} sgpu_nodal_desc;
sgpu_status sgpu_add_nodal(sgpu_ctx* ctx, const sgpu_nodal_desc* d);

/* Borders other than CPML.  Face order back, front, left, right, down, up
 * (sgg%Border, fdetypes.F90:468-497).  A PEC face needs no call: it is medium
 * 0 in the media matrices (healer.F90:1442-1617).
 *   pmc[f], periodic[f]: InitOtherBorders (bordersother.F90:36-58); the H
 *     outside the face is cloned by sgpu_advance_pmc_h / _periodic_h.
 *   mur[f]: InitMURBorders (bordersmur.F90:79-314) -- a Mur face, or a CPML
 *     face under -mur1/-mur2; mur_cab1[f] is CAB1 of calc_murconstants
 *     (bordersmur.F90:316-363), num_media+1 values.  The Past_ layers start
 *     at zero (a fresh start). */
typedef struct {
    int pmc[6];
    int periodic[6];
    int mur[6];
    const float* mur_cab1[6];
} sgpu_border_desc;
sgpu_status sgpu_init_borders(sgpu_ctx* ctx, const sgpu_border_desc* d);

/* crea_timevector (timestepping.F90:3230-3240): tiempo(n0 .. n0+count-1). */
sgpu_status sgpu_set_time(sgpu_ctx* ctx, int n0, int count, const double* tiempo);
/* tiempo(n0 .. n0+count-1) of the time vector set last (for output files). */
sgpu_status sgpu_get_time(const sgpu_ctx* ctx, int n0, int count, double* tiempo);

/* Point probes (observation.F90:2633-2668): comp_ijk holds 4 ints per
 * probe (component, i, j, k).  Values are recorded after every whole step
 * into a device ring of capacity_steps rows. */
sgpu_status sgpu_set_probes(sgpu_ctx* ctx, int nprobes, const int* comp_ijk, int capacity_steps);
/* Copy the rows recorded since the last read (at most max_steps) to out
 * (row-major [step][probe]); *nsteps receives the number of rows and
 * *first_n the step index n of the first row. */
sgpu_status sgpu_read_probes(sgpu_ctx* ctx, float* out, int max_steps, int* nsteps, int* first_n);

/* Volume ("movie") probes of observation.F90.  A probe samples the three E
 * (magnetic = 0) or H (magnetic = 1) components at the nodes (i, j, k) of
 * box[6] = XI XE YI YE ZI ZE (absolute cell coordinates, inside Alloc) whose
 * coordinates are multiples of stride[3] (the reference's X/Y/Ztrancos); the
 * sampled node (i, j, k) has index (i/stride[0] - i0, j/stride[1] - j0,
 * k/stride[2] - k0), i0 = XItrancos = XI/stride[0] rounded up
 * (observation.F90:318-331).  Probes are sampled after every whole step,
 * with the point probes.
 *
 * Frequency domain (observation.F90:3527-3600, 1918-1922): after step n the
 * complex(8) accumulators take V(f, c, node) += w(f, n) * F_c(node) with
 *   w(f, n) = dt * exp(-i * 2 pi_f * freq[f] * tiempo(n))       (E)
 *   w(f, n) * exp(-i * 2 pi_f * freq[f] * dt / 2)               (H)
 * pi_f the real(4) pi, each exponential the host's complex(8) exp, formed
 * on the host from the time vector set before the call (steps outside it
 * add nothing). */
typedef struct {
    int magnetic;
    int box[6];
    int stride[3];
    int nfreq;
    const float* freq; /* real(4) frequencies (observation.F90:505-536) */
} sgpu_freq_probe_desc;
sgpu_status sgpu_add_freq_probe(sgpu_ctx* ctx, const sgpu_freq_probe_desc* d, int* id);
/* Time domain: all three components of the sampled box after every step n
 * with n_first <= n < n_last and (n - n_first) % every == 0, kept in a
 * device ring of `capacity` frames. */
typedef struct {
    int magnetic;
    int box[6];
    int stride[3];
    int n_first, n_last, every;
    int capacity;
} sgpu_movie_probe_desc;
sgpu_status sgpu_add_movie_probe(sgpu_ctx* ctx, const sgpu_movie_probe_desc* d, int* id);
/* Sampled nodes per axis of volume probe id and the first sampled index
 * (XItrancos, YItrancos, ZItrancos) in ijk0[3]. */
sgpu_status sgpu_volume_probe_shape(const sgpu_ctx* ctx, int id, int* ni, int* nj, int* nk, int* ijk0);
/* The accumulators of frequency probe id as nfreq x 3 x nk x nj x ni
 * complex(8) values (re, im interleaved, i fastest): the order of the
 * reference's output records (observation.F90:4013-4046). */
sgpu_status sgpu_read_freq_probe(sgpu_ctx* ctx, int id, double* out);
/* The frames of movie probe id recorded since the last read, at most
 * max_frames, as [frame][3][nk][nj][ni] floats; *frames receives their
 * number and *first_n the step of the first.  Frames older than the ring's
 * capacity are gone: the read starts at the oldest one kept. */
sgpu_status sgpu_read_movie_probe(sgpu_ctx* ctx, int id, float* out, int max_frames, int* frames, int* first_n);

/* One call per reference routine, in the order of timestepping.F90:1286-1742
 * (the border calls: after the magnetic CPML and again after the H sources
 * for PMC/periodic, timestepping.F90:1568-1573 and :1636-1641; Mur before the
 * observation, :1711-1712; the magnetic ADE after the first clones, :1582). */
sgpu_status sgpu_advance_ex(sgpu_ctx* ctx);                 /* Advance_Ex :2165 */
sgpu_status sgpu_advance_ey(sgpu_ctx* ctx);                 /* Advance_Ey :2206 */
sgpu_status sgpu_advance_ez(sgpu_ctx* ctx);                 /* Advance_Ez :2250 */
sgpu_status sgpu_advance_electric_cpml(sgpu_ctx* ctx);      /* borderscpml.F90:584 */
sgpu_status sgpu_advance_edispersive_e(sgpu_ctx* ctx);      /* electricdispersive.F90:304 */
sgpu_status sgpu_advance_planewave_e(sgpu_ctx* ctx, int n); /* planewaves.F90:878 */
sgpu_status sgpu_advance_nodal_e(sgpu_ctx* ctx, int n);     /* nodalsources.F90:396 */
sgpu_status sgpu_advance_hx(sgpu_ctx* ctx);                 /* Advance_Hx :2294 */
sgpu_status sgpu_advance_hy(sgpu_ctx* ctx);                 /* Advance_Hy :2334 */
sgpu_status sgpu_advance_hz(sgpu_ctx* ctx);                 /* Advance_Hz :2374 */
sgpu_status sgpu_advance_magnetic_cpml(sgpu_ctx* ctx);      /* borderscpml.F90:881 */
sgpu_status sgpu_advance_planewave_h(sgpu_ctx* ctx, int n); /* planewaves.F90:1180 */
sgpu_status sgpu_advance_nodal_h(sgpu_ctx* ctx, int n);     /* nodalsources.F90:584 */
sgpu_status sgpu_advance_mdispersive_h(sgpu_ctx* ctx);      /* AdvanceMdispersiveH, magneticdispersive.F90:298 */
sgpu_status sgpu_advance_pmc_h(sgpu_ctx* ctx);              /* MinusCloneMagneticPMC, bordersother.F90:65 */
sgpu_status sgpu_advance_periodic_h(sgpu_ctx* ctx);         /* CloneMagneticPeriodic, bordersother.F90:146 */
sgpu_status sgpu_advance_magnetic_mur(sgpu_ctx* ctx);       /* AdvanceMagneticMUR, bordersmur.F90:502 */
sgpu_status sgpu_update_observation(sgpu_ctx* ctx, int n);  /* observation.F90:2540 */

/* Fused forms, same results bit for bit: the E half step (curl + CPML +
 * ADE + TF/SF + nodal), the H half step (curl + CPML + magnetic ADE + TF/SF +
 * nodal + PMC/periodic clones + Mur; the clones before the H sources are left out
 * because nothing between the two clone calls reads the cloned layers), and
 * `count` whole steps n0 .. n0+count-1 including the probe gather, captured
 * into a CUDA graph and replayed. */
sgpu_status sgpu_advance_e(sgpu_ctx* ctx, int n);
sgpu_status sgpu_advance_h(sgpu_ctx* ctx, int n);
sgpu_status sgpu_advance_steps(sgpu_ctx* ctx, int n0, int count);

/* Field-kernel family of the fused half steps: 1 (default when the driver
 * provides tensor maps) streams each tile's planes through a shared-memory
 * ring with TMA bulk-tensor loads; 0 uses register-marching kernels with
 * plain loads.  Both give identical results. */
sgpu_status sgpu_set_kernel_family(sgpu_ctx* ctx, int family);

/* Bound, in SM clock cycles, of every wait inside the TMA-pipelined kernels
 * (a consumer waiting for a plane, the producer waiting for a free stage);
 * default 4e9 (about 2 s).  When a wait runs out the kernel records the
 * place in an error word, stops, waits (with the default bound) for the
 * loads it has in flight and exits; the next sgpu_synchronize returns
 * SGPU_ERR_TIMEOUT and the fields are then undefined.  A failure-detection
 * test shortens it to make the wait expire without a fault. */
sgpu_status sgpu_set_wait_cycles(sgpu_ctx* ctx, int64_t cycles);
/* Failure drill (off by default): while on, the producer warps of the
 * pipelined field kernels issue no loads, so every consumer wait runs out
 * after the wait bound and the next synchronize returns SGPU_ERR_TIMEOUT;
 * nothing is left in flight.  For tests of the timeout path. */
sgpu_status sgpu_set_wait_drill(sgpu_ctx* ctx, int on);

/* Scans the six field components for NaN/Inf on the device; returns
 * SGPU_ERR_NONFINITE if any is found (the host-side counterpart of the
 * reference's energy/NaN stop, errorreport.F90:1433-1460). */
sgpu_status sgpu_check_finite(sgpu_ctx* ctx);

/* sgpu_advance_steps bracketed by CUDA events on the context's stream;
 * *ms receives the device time of the `count` steps. */
sgpu_status sgpu_elapsed_steps(sgpu_ctx* ctx, int n0, int count, float* ms);
/* `count` steps launched directly with CUDA events between the phases;
 * ms6 accumulates the device time of: E curl+CPML, ADE, E sources,
 * H curl+CPML, magnetic ADE + H sources + borders (clones, Mur), probe gather. */
sgpu_status sgpu_profile_steps(sgpu_ctx* ctx, int n0, int count, float* ms6);
/* Algorithmic bytes of one launch of each phase of sgpu_profile_steps:
 * compulsory field/media/psi/ADE-state traffic, without neighbour re-reads
 * or coefficient tables. */
sgpu_status sgpu_algorithmic_bytes(const sgpu_ctx* ctx, double* bytes6);
/* The compulsory bytes of the same phases: every field node read and written
 * once a step with its int16 medium (10 B), every CPML psi point read and
 * written (8 B), every pole-residue node's previous field and stored
 * currents read and written (8 B + 32 B per stored pole); the other field's
 * reads in a half step, neighbour re-reads, node lists and a separate ADE
 * pass's field re-read are not counted (60 B per cell and step over the six
 * components, the bound of a kernel that touches each value once). */
sgpu_status sgpu_compulsory_bytes(const sgpu_ctx* ctx, double* bytes6);
/* Select the CUDA device this library's runtime uses on the calling thread
 * (call before sgpu_create / sgpu_host_create). */
sgpu_status sgpu_select_device(int device);
/* Device memory of contexts outside a batch, and each batch's arena, come
 * from the current device's default memory pool (stream-ordered), which
 * keeps freed memory for the next context or batch; this hands the kept
 * memory back to the driver (waits for the device).  sgpu_batch_create does
 * it only when the pool cannot serve its arena. */
sgpu_status sgpu_trim_device_memory(void);
/* Kernel launches issued per whole step (graph replays add one per chunk). */
sgpu_status sgpu_kernels_per_step(const sgpu_ctx* ctx, int* n);

/* Non-finite scan that allocates no device memory.  No counterpart in the
 * reference: it is for callers that cannot call cudaMalloc where they need
 * the check (a host whose device memory belongs to its own pool allocator, a
 * service loop that forbids allocation after start-up, a watchdog checking a
 * buffer it does not own).  Counts the NaN/Inf values among the n floats at
 * the device pointer `data` and returns the count and the index of the first
 * one (-1 when none) in host memory.  The scan runs on the device that holds
 * `data`: the library's runtime switches to it for the call and back, so the
 * caller's own device selection does not matter.  `stream` is a cudaStream_t
 * of that device passed as a pointer (NULL: its legacy default stream); the
 * call waits for that stream.
 *   - n may be at most 268,435,456 (4096 x 65536); larger n returns
 *     SGPU_ERR_SIZE without touching the data.
 *   - Scratch is a file-scope __device__ array of 512 KiB that every device
 *     loading this library holds until exit.  Its device address is taken
 *     with cudaGetSymbolAddress on the first call on each device, so make
 *     that first call before any stream capture.
 *   - Every call shares the scratch: calls whose work overlaps on a device
 *     (different host threads, or streams that run concurrently) race and
 *     may return each other's results; serialise them. */
sgpu_status sgpu_scan_nonfinite_noalloc(const float* data, uint64_t n, void* stream, uint64_t* count,
                                        int64_t* first_index);

/* Bytes of device memory the context holds. */
sgpu_status sgpu_device_bytes(const sgpu_ctx* ctx, uint64_t* bytes);

/* ======================================================================== */
/* Level 2: problem-level host                                              */
/* ======================================================================== */

/* A material region in NFDE terms: kind 0 = PEC volume, 1 = isotropic
 * dielectric volume, 2 = pole-residue volume.  eps/mu absolute
 * (for a pole-residue region eps is the high-frequency permittivity).
 * Poles: the complex64 residues a11 and b11 = minus the pole, as in
 * preprocess_geom.F90:5196-5199. */
typedef struct {
    int kind;
    float eps, sigma, mu, sigmam;
    int npoles;
    const float* residues;   /* 2*npoles */
    const float* bpoles;     /* 2*npoles */
    int nboxes;
    const int* boxes;        /* 6*nboxes: XI XE YI YE ZI ZE inclusive */
    /* kind 2: magnetic poles (aM11 residues, bM11 = minus the pole,
     * preprocess_geom.F90:5223-5226); mu is then the high-frequency
     * permeability and sigmam its conductivity.  Either set may be empty. */
    int mpoles;
    const float* mresidues;  /* 2*mpoles */
    const float* mbpoles;    /* 2*mpoles */
} sgpu_region;

typedef struct {
    int x1, y1, z1, x2, y2, z2;    /* coor1 / coor2 (cellIntervalsToCoords) */
    float theta, phi, alpha, beta;
    int nsamples;
    const float* samples;
    float dsamples;
} sgpu_planewave_src;

typedef struct {
    int is_elec, is_hard;
    int npoints;
    const int* boxes;   /* 6*npoints */
    const float* amp;   /* 3*npoints: xc yc zc */
    int nsamples;
    const float* samples;
    float dsamples;
} sgpu_nodal_src;

typedef struct {
    int nx, ny, nz;
    const float *desx, *desy, *desz;
    float originx, originy, originz;
    double dt;          /* general%dt */
    int forcecfl;       /* the -cfl switch */
    float cfl;
    int pml_layers[6];  /* back, front, left, right, down, up; >= 1 on CPML faces */
    float pml_order[6];
    float pml_refl[6];
    float alphamax, alphaorder, kappamax;   /* -pmlalpha, -pmlkappa */
    int nregions;
    const sgpu_region* regions;
    int npw;
    const sgpu_planewave_src* pw;
    int nnodal;
    const sgpu_nodal_src* nodal;
    int nprobes;
    const int* probes;  /* 4*nprobes: comp, i, j, k */
    int probe_capacity; /* rows of the device probe ring */
    /* Border kind per face, the tipofrontera codes of nfde_types.F90:67-71:
     * 1 PEC, 2 PMC, 4 periodic, 7 first-order Mur, 9 CPML; 0 reads as 9.
     * Only CPML faces have layers (pml_* of other faces are ignored). */
    int border[6];
    int mur_after_pml;  /* -mur1 / -mur2: first-order Mur on every CPML face too */
} sgpu_problem;

/* Restated set-up of semba_fdtd.F90:1197-1300 and timestepping.F90:305-1014
 * for one problem, then sgpu_create and the sgpu_init_* calls.  The time
 * vector is generated for steps 0 .. max_steps+2.  On failure *out may hold
 * a context whose sgpu_last_error explains it; destroy it. */
sgpu_status sgpu_host_create(const sgpu_problem* p, int max_steps, sgpu_ctx** out);
/* The same set-up on the host only: the context owns no device memory and
 * serves the sgpu_host_* getters (and sgpu_host_footprint for admission
 * control) without a GPU. */
sgpu_status sgpu_host_plan(const sgpu_problem* p, int max_steps, sgpu_ctx** out);
/* Device bytes sgpu_host_create would allocate for this plan: fields, media,
 * CPML psi, ADE state and the probe ring. */
sgpu_status sgpu_host_footprint(const sgpu_ctx* ctx, uint64_t* bytes);
/* Results of the set-up. */
sgpu_status sgpu_host_info(const sgpu_ctx* ctx, double* dt, int* num_media, sgpu_lim* alloc6,
                           sgpu_lim* sweep6, sgpu_lim* sinpml6);
/* The coefficient tables the host built (num_media+1 each). */
sgpu_status sgpu_host_get_g(const sgpu_ctx* ctx, float* g1, float* g2, float* gm1, float* gm2);
/* which as for the oracle: 0..5 Idxe..Idzh, 6..17 P_be, P_ce, P_bm, P_cm. */
sgpu_status sgpu_host_get_metric(const sgpu_ctx* ctx, int which, float* out, int* lo, int* hi);
sgpu_status sgpu_host_get_media(const sgpu_ctx* ctx, int comp, int16_t* out);
/* CAB1 of calc_murconstants for face f (back, front, left, right, down, up),
 * num_media+1 values; SGPU_ERR_ARG when the face has no Mur condition. */
sgpu_status sgpu_host_get_mur_cab1(const sgpu_ctx* ctx, int face, float* out);
/* Z-slab sub-domains: the reference's MPI decomposition along z
 * (mpicomm.F90:122-358, 1507-1677; timestepping.F90:1453-1459, 1661-1669).
 * sgpu_host_create_zslab sets up the problem as sgpu_host_create does and
 * keeps the planes z0..z1 (absolute; the slabs of a decomposition tile the
 * problem's swept z range, the first starting at or below it and the last
 * ending at or above it): every component sweeps its owned planes, and its
 * Alloc range reaches one plane past them on a cut side -- the halo.  After
 * each E half step the slab above must copy Ex and Ey of its first owned
 * plane into this slab's plane z1+1; after each H half step the slab below
 * must copy Hx and Hy of its last owned plane into this slab's plane z0-1
 * (those are the only values the curl of a cut plane reads across the cut).
 * CPML, borders of the x and y faces, ADE and sources are local; z faces
 * belong to the end slabs; point probes are recorded by the slab that owns
 * their plane.  Periodic z faces across slabs are SGPU_ERR_UNSUPPORTED. */
sgpu_status sgpu_host_create_zslab(const sgpu_problem* p, int max_steps, int z0, int z1, sgpu_ctx** out);
/* Device address and byte size of plane z (absolute) of component comp: a
 * contiguous run of the padded layout, identical in size for all slabs of
 * one decomposition (for NCCL or peer copies). */
sgpu_status sgpu_zplane(sgpu_ctx* ctx, int comp, int z, void** ptr, uint64_t* bytes);
/* Copy plane z of component comp from src into dst (same x-y layout; same
 * or peer device), after the work queued on src and before later work on
 * dst; src's later work waits for the copy. */
sgpu_status sgpu_copy_zplane(sgpu_ctx* dst, sgpu_ctx* src, int comp, int z);

/* eps0 and mu0 of the set-up (real(4)), as flush_and_save_resume takes them. */
sgpu_status sgpu_host_get_constants(const sgpu_ctx* ctx, float* eps0, float* mu0);
/* The incident-field column of a point-probe file: Incid as
 * FlushObservationFiles calls it (observation.F90:3826-3875, planewaves.F90:
 * 778-853), the sum over every plane wave of fpw(comp) * evolucion at the
 * PhysCoor of component comp at node (i, j, k), at each of the nt real(4)
 * times t (tiempo(n) for E, tiempo(n) + dt/2 for H); zeros without plane
 * waves.  Host only; the run's plane-wave switch is not touched. */
sgpu_status sgpu_host_incident(const sgpu_ctx* ctx, int comp, int i, int j, int k, int nt, const float* t, float* out);

/* Restart files (resuming.F90:213-496).  sgpu_store_resume writes the
 * records flush_and_save_resume writes, in its order: StoreFields (one
 * record n, tiempo(n), dt, eps0, mu0; then Ex..Hz, each row of the Alloc box
 * in records of at most 1024 values and a remainder record, empty when the
 * row length is a multiple of 1024), StoreFieldsCPMLBorders (the psi arrays
 * region by region, one record per row of each PMLc box), StoreFieldsMURBorders
 * (Past_ then PastPast_ per MURc box; the first-order update leaves PastPast_
 * at zero), StoreFieldsEDispersives and StoreFieldsMDispersives (per medium
 * and component, each node's previous field then its current per pole,
 * complex(8)).  Records are Fortran sequential unformatted: each framed by
 * its byte length as a 4-byte integer.  last_step is the last executed step
 * n, whose tiempo(n) must be in the time vector.  sgpu_load_resume reads such
 * a file back into a context set up for the same problem (the Init*
 * routines' resume branches, same order) and returns n in *last_step; the
 * run goes on at n + 1. */
sgpu_status sgpu_store_resume(sgpu_ctx* ctx, const char* path, int last_step, float eps0, float mu0);
sgpu_status sgpu_load_resume(sgpu_ctx* ctx, const char* path, int* last_step);

/* ------------------------------------------------------------------------
 * Batched form (no counterpart in the reference, which runs one problem per
 * process).  Many independent problems of uneven sizes live in one device
 * arena and advance together: every phase of a step is one persistent
 * kernel over flattened work lists of all instances, and whole steps are
 * replayed from a CUDA graph of 32 captured steps.  Each instance advances
 * with the same per-cell arithmetic as sgpu_host_create, so its probe traces
 * and fields are bit-identical to a solo run.  Instances join at step 0 when
 * added (between calls that advance the batch) and stop after their last
 * step while others go on; the batch's own step counter advances for all.
 * ------------------------------------------------------------------------ */
typedef struct sgpu_batch sgpu_batch;

/* One arena of arena_bytes of device memory (one block from the current
 * device's default memory pool, given back to it by sgpu_batch_destroy),
 * room for max_instances instances. */
sgpu_status sgpu_batch_create(uint64_t arena_bytes, int max_instances, sgpu_batch** out);
void sgpu_batch_destroy(sgpu_batch* b);
const char* sgpu_batch_last_error(const sgpu_batch* b);
/* Set up a problem inside the arena: from `p`, or from `plan` (a host-only
 * context of sgpu_host_plan, consumed: destroy it afterwards as usual).  The
 * instance runs steps 0..nsteps and keeps every probe row on the device.
 * SGPU_ERR_OOM when the arena has no room (nothing is left allocated).
 * Several host threads may add instances to one batch at once (the set-up
 * of each runs on a stream of its own while the batch's queued steps run);
 * the other batch entry points take the batch's lock. */
sgpu_status sgpu_batch_add(sgpu_batch* b, const sgpu_problem* p, sgpu_ctx* plan, int nsteps, int* slot);
/* Free an instance's arena memory and slot (waits for queued work). */
sgpu_status sgpu_batch_remove(sgpu_batch* b, int slot);
/* Queue nsteps batch steps (graph replays of 32, the rest one by one). */
sgpu_status sgpu_batch_advance(sgpu_batch* b, int nsteps);
/* Wait for queued work; SGPU_ERR_TIMEOUT if a bounded wait ran out. */
sgpu_status sgpu_batch_synchronize(sgpu_batch* b);
/* sgpu_batch_advance timed on the device with CUDA events (waits). */
sgpu_status sgpu_batch_elapsed(sgpu_batch* b, int nsteps, float* ms);
/* Steps an instance has completed (queued work counted) and its total. */
sgpu_status sgpu_batch_slot_info(const sgpu_batch* b, int slot, int* steps_done, int* steps_total, int* nprobes);
/* Probe rows 0..rows-1 of an instance ([step][probe] floats; waits). */
sgpu_status sgpu_batch_read_probes(sgpu_batch* b, int slot, float* out, int max_rows, int* rows);
/* The instance's context, for sgpu_download_field and the like (waits). */
sgpu_status sgpu_batch_instance(sgpu_batch* b, int slot, sgpu_ctx** ctx);
/* Arena capacity, bytes in use and the largest free block. */
sgpu_status sgpu_batch_memory(sgpu_batch* b, uint64_t* capacity, uint64_t* in_use, uint64_t* largest_free);
/* Device bytes one instance of this plan takes in a batch arena (every
 * buffer rounded to the arena's 256-byte grain, whole probe traces), and
 * its largest single buffer. */
sgpu_status sgpu_batch_footprint(const sgpu_ctx* plan, uint64_t* bytes, uint64_t* largest);
/* Field kernels of the batch: 1 (default) the persistent TMA-pipelined
 * kernels (each instance's tensor maps in global memory), 0 the
 * register-marching kernels.  Both give identical results. */
sgpu_status sgpu_batch_set_kernel_family(sgpu_batch* b, int family);
/* The wait bound of sgpu_set_wait_cycles for the batch's pipelined kernels;
 * sgpu_batch_synchronize reports an expiry as SGPU_ERR_TIMEOUT. */
sgpu_status sgpu_batch_set_wait_cycles(sgpu_batch* b, int64_t cycles);
/* The failure drill of sgpu_set_wait_drill for the batch's kernels. */
sgpu_status sgpu_batch_set_wait_drill(sgpu_batch* b, int on);
/* Launch shape: z-chunk length (1..1024) of the field work items for the three
 * size classes (Alloc z extent <= 80, <= 160, larger) and persistent CTAs per SM.
 * Either may be NULL / 0 to keep the current value. */
sgpu_status sgpu_batch_set_tuning(sgpu_batch* b, const int* chunk3, int ctas_per_sm);
sgpu_status sgpu_batch_get_tuning(const sgpu_batch* b, int* chunk3, int* ctas_per_sm);
/* Online autotuner: times steps_per_trial real steps of the live instances
 * per candidate (CTAs per SM in 2,3,4,6, then z chunk 128..8 per size class
 * present, a shorter chunk kept only when 3 % faster) and keeps the fastest.
 * The trials advance the instances. */
sgpu_status sgpu_batch_autotune(sgpu_batch* b, int steps_per_trial, int* chunk3, int* ctas_per_sm);
/* Device time of each phase summed over nsteps real steps launched one by
 * one: E field + CPML, ADE, E sources, H field + CPML, H sources and
 * borders, probes. */
sgpu_status sgpu_batch_profile_steps(sgpu_batch* b, int nsteps, float* ms6);
/* The batch step counter (steps queued so far). */
sgpu_status sgpu_batch_steps(const sgpu_batch* b, int* counter);

/* ---- Near-to-far-field transform (farfield.F90) --------------------------
 * InitFarField (farfield.F90:118-1158) for one closed surface.  Faces in the
 * order Tr, Fr, Iz, De, Ab, Ar (x-, x+, y-, y+, z-, z+).  Each face carries
 * two tangential E components, t1 / t2 = (Ez, Ey) on x faces, (Ez, Ex) on y
 * faces, (Ey, Ex) on z faces, and for each the H component that pairs with
 * it (Hy, Hz; Hx, Hz; Hx, Hy), sampled on two planes.
 *   lim[face][t] = {plane, lo1, hi1, lo2, hi2}: the E plane index of
 *     component t and the ranges of its two in-plane indices in the
 *     reference's loop order (k then j on x faces, k then i on y faces,
 *     j then i on z faces): TrFr%I%tra / fro, IzDe%J%izq / der,
 *     AbAr%K%aba / arr and their com / fin limits (farfield.F90:512-580).
 *     The H partner takes the same ranges on planes plane-1 and plane (low
 *     faces) or plane and plane+1 (high faces).
 *   freq[nfreq]: the frequencies, real(4) as the reference lists them.
 *   ndecim, dtdecim: FF%NDecim and FF%dtDecim (farfield.F90:194-199);
 *     UpdateFarField (:1163-1733) samples steps n with mod(n-1, ndecim) = 0.
 *   cluz, zvac, cell[6] = dxe, dye, dze, dxh, dyh, dzh over cell_lo ..
 *   cell_lo+cell_n-1 and phys[c][axis] = Punto%PhysCoor of Ex, Ey, Ez are
 *   for the transform (FlushFarfield, :2408-3423). */
typedef struct {
    int active[6];
    int lim[6][2][5];
    int nfreq;
    const float* freq;
    int ndecim;
    float dtdecim;
    float cluz, zvac;
    const float* cell[6];
    int cell_lo[6];
    int cell_n[6];
    const float* phys[3][3];
    int phys_lo[3][3];
    int phys_n[3][3];
} sgpu_farfield_desc;
sgpu_status sgpu_add_farfield(sgpu_ctx* ctx, const sgpu_farfield_desc* d, int* id);
/* The far-field request of the reference's input (the FarField probe of
 * observation.F90:2050): the box esqx1, esqx2, esqy1, esqy2, esqz1, esqz2
 * in cell indices, the faces to sample, the frequency range and the
 * decimation switch (NF2FFDecim).  Clips the box and fills the descriptor
 * above from the context's host set-up (sgpu_host_create), then adds it.
 * A face on the edge of the non-CPML region is refused as the reference
 * refuses it ("NF2FF STILL UNSUPPORTED"). */
typedef struct {
    int box[6];
    int faces[6];
    float initial_freq, final_freq, freq_step;
    int logarithmic;
    int decimate;
} sgpu_farfield_spec;
sgpu_status sgpu_host_add_farfield(sgpu_ctx* ctx, const sgpu_farfield_spec* s, int* id);
/* Number of frequencies and surface samples (all faces, components and
 * planes) of a far field. */
sgpu_status sgpu_farfield_shape(const sgpu_ctx* ctx, int id, int* nfreq, int* samples);
/* One accumulated surface array: face 0..5, slot 0 / 1 = E t1 / t2, 2 / 3 =
 * the H partner of t1 on its first / second plane, 4 / 5 the same for t2.
 * dims[2] = the counts of the two in-plane indices (loop order, outer
 * first); out = complex(8) [nfreq][outer][inner]. */
sgpu_status sgpu_read_farfield(sgpu_ctx* ctx, int id, int face, int slot, int* dims, double* out);
/* FlushFarfield (farfield.F90:2408-3423): for every frequency and direction
 * (theta from theta_start in theta_step up to theta_stop, the last step
 * clamped; phi likewise), the radiation vectors L, N summed over the faces
 * with arithmetic and geometric means of the two H planes, and from them
 * the row  freq, theta, phi, |Etheta|, arg Etheta, |Ephi|, arg Ephi (the
 * geometric pass), RCS (arithmetic), RCS (geometric).  incident[0..n-1]
 * are the (time, value) pairs of the normalisation file (FileNormalize,
 * farfield.F90:1021-1070); its DFT normalises the RCS.  Rows go to out
 * [max_rows][9]; *rows gets the number of frequency x direction rows. */
typedef struct {
    float theta_start, theta_stop, theta_step;
    float phi_start, phi_stop, phi_step;
} sgpu_farfield_angles;
sgpu_status sgpu_farfield_transform(sgpu_ctx* ctx, int id, const sgpu_farfield_angles* a, const float* incident,
                                    int n_incident, double* out, int max_rows, int* rows);

#ifdef __cplusplus
}
#endif
#endif
