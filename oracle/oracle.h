/*
 * CPU oracle for the semba-fdtd Yee / CPML / pole-residue ADE / TF-SF hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * it is loaded by tests/, by __graft_entry__.smoke() and by the cpu_baseline
 * leg of bench.py, and by nothing else.  It is never the thing measured as
 * the GPU result and the product never links it.
 *
 * It restates, in plain C++17 with OpenMP, the reference's algorithm:
 *   - grid limits, PML padding and time step   (preprocess_geom.F90:5266-5737,
 *                                                semba_fdtd.F90:1197-1300)
 *   - media table and media matrices           (preprocess_geom.F90:421-760,
 *                                                1085-1110, healer.F90:66-243,
 *                                                healer.F90:961-1420)
 *   - update coefficients                       (calc_constants.F90:36-148)
 *   - metric arrays                             (timestepping.F90:314-370)
 *   - CPML                                      (borderscpml.F90:90-473, 584-1176,
 *                                                1465-1733)
 *   - PEC, PMC, periodic and first-order Mur    (healer.F90:1442-1617,
 *     borders                                    bordersother.F90:65-190,
 *                                                bordersmur.F90:79-363, 502-1653)
 *   - electric pole-residue ADE                 (electricdispersive.F90:77-362)
 *   - magnetic pole-residue ADE                 (magneticdispersive.F90:79-360)
 *   - plane-wave TF/SF                          (planewaves.F90:72-853, 878-1510)
 *   - nodal sources                             (nodalsources.F90:76-583)
 *   - point probes                              (observation.F90:2633-2668)
 *   - the leapfrog loop order                   (timestepping.F90:1248-1981)
 * following the reference's operation order and its real4/real8/complex8
 * promotion rules.  The template parameter R is the field kind RKIND: float
 * is the reference FP32 build, double the -DCompileWithReal8 accuracy oracle.
 *
 * Parity status: the reference Fortran cannot be compiled in this container
 * (no Fortran compiler; its json-fortran/ngspice/lapack dependencies are
 * absent), and the reference ships no golden vectors for this path, so the
 * oracle is pinned by known-answer tests (tests/test_oracle_kat.py) and the
 * reference's parser fixture, not by reference outputs: parity unpinned.
 */
#ifndef SEMBA_ORACLE_H
#define SEMBA_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* A material region in NFDE terms (nfde_types.F90).  kind: 0 = PEC volume,
 * 1 = isotropic dielectric volume, 2 = pole-residue volume (electric and/or
 * magnetic poles).
 * eps/mu are absolute (F/m, H/m) as stored by the NFDE structures; for a
 * dispersive region eps is eps11 (the high-frequency permittivity). */
typedef struct {
    int kind;
    float eps, sigma, mu, sigmam;
    int npoles;
    const float* residues; /* 2*npoles: complex64 residues a11 (re, im)        */
    const float* bpoles;   /* 2*npoles: complex64 b11 = minus the pole (re, im) */
    int nboxes;
    const int* boxes;      /* 6*nboxes: XI XE YI YE ZI ZE, inclusive cell coords */
    /* kind 2 only: magnetic poles (aM11 residues, bM11 = minus the pole),
     * with mu the high-frequency permeability and sigmam its conductivity */
    int mpoles;
    const float* mresidues; /* 2*mpoles */
    const float* mbpoles;   /* 2*mpoles */
} orc_region;

typedef struct {
    int x1, y1, z1, x2, y2, z2;      /* coor1 / coor2 after cellIntervalsToCoords */
    float theta, phi, alpha, beta;   /* direction and polarisation angles       */
    int nsamples;                    /* numus + 1                               */
    const float* samples;
    float dsamples;
} orc_planewave;

typedef struct {
    int is_elec, is_hard;
    int npoints;
    const int* boxes;                /* 6*npoints */
    const float* amp;                /* 3*npoints: xc, yc, zc */
    int nsamples;
    const float* samples;
    float dsamples;
} orc_nodal;

typedef struct {
    int nx, ny, nz;
    const float *desx, *desy, *desz;
    float originx, originy, originz;
    double dt;                       /* general%dt from the case file */
    int forcecfl;                    /* -cfl switch given             */
    float cfl;
    /* face order of the reference: back(x-), front(x+), left(y-), right(y+),
     * down(z-), up(z+).  Layers of a CPML face must be >= 1; other faces have
     * none and their pml_* entries are ignored. */
    int pml_layers[6];
    float pml_order[6];
    float pml_refl[6];
    float alphamax, alphaorder, kappamax;
    int nregions;
    const orc_region* regions;
    int npw;
    const orc_planewave* pw;
    int nnodal;
    const orc_nodal* nodal;
    int nprobes;
    const int* probes;               /* 4*nprobes: comp(0..5 = Ex..Hz), i, j, k */
    /* Border kind per face, the tipofrontera codes of nfde_types.F90:67-71:
     * 1 PEC, 2 PMC, 4 periodic, 7 first-order Mur, 9 CPML (0 reads as 9). */
    int border[6];
    int mur_after_pml;               /* -mur1/-mur2: Mur also on every CPML face */
} orc_problem;

/* Extents of one component (sgg%Alloc, sgg%Sweep) in the reference's
 * absolute cell coordinates. */
typedef struct { int xi, xe, yi, ye, zi, ze; } orc_lim;

/* Returns 0 on success.  fp64 != 0 selects the double-precision variant. */
int orc_create(const orc_problem* p, int fp64, int nthreads, void** handle);
void orc_destroy(void* h);
/* Advance steps n0 .. n1-1 (the reference's loop variable n), recording
 * probes after each step into rows [n - n0] of out (nprobes per row), if
 * out is non-null. */
int orc_run(void* h, int n0, int n1, float* probe_out);
/* Frequency-domain volume probe (observation.F90:318-331, 3527-3600) over
 * box[6] (XI XE YI YE ZI ZE) sampled at multiples of stride[3], E (magnetic
 * 0) or H (1), accumulated after every step that orc_run advances; returns
 * its id or -1. */
int orc_add_freq_probe(void* h, int magnetic, const int* box, const int* stride, int nfreq, const float* freq);
/* shape4 = nfreq, nk, nj, ni; out = nfreq x 3 x nk x nj x ni complex(8)
 * values (re, im interleaved). */
int orc_read_freq_probe(void* h, int id, int* shape4, double* out);
/* Restart files in the records of resuming.F90's flush_and_save_resume
 * (fields, CPML psi, Mur Past_/PastPast_, electric and magnetic ADE state);
 * last_step is the last executed step n.  Load returns 0 and n on success. */
/* Far field (farfield.F90): InitFarField for the box esqx1..esqz2, the faces
 * Tr, Fr, Iz, De, Ab, Ar to sample, the frequency range and NF2FFDecim
 * (returns the id, -2 for a face on a PEC/PMC border); the accumulated
 * arrays (face, slot 0..5 as sgpu_read_farfield); FlushFarfield's rows
 * (angles = theta start, stop, step, phi start, stop, step; incident =
 * (time, value) pairs). */
int orc_add_farfield(void* h, const int* box, const int* faces, float fi, float ff, float fs, int logarithmic,
                     int decimate);
int orc_read_farfield(void* h, int id, int face, int slot, int* dims, double* out);
int orc_farfield_transform(void* h, int id, const float* angles, const float* incident, int n_incident, double* out,
                           int max_rows, int* rows);
int orc_store_resume(void* h, const char* path, int last_step);
int orc_load_resume(void* h, const char* path, int* last_step);
/* Grid description after set-up. */
int orc_get_lims(void* h, orc_lim* alloc6, orc_lim* sweep6, orc_lim* sinpml6);
double orc_get_dt(void* h);
int orc_get_num_media(void* h);
/* Copy a field component (0..5) into a float buffer laid out over Alloc in
 * Fortran (column-major) order. */
int orc_get_field(void* h, int comp, float* out);
int orc_get_field_f64(void* h, int comp, double* out);
/* Overwrite a field component (known-answer tests set initial states). */
int orc_set_field(void* h, int comp, const float* in);
int orc_get_media(void* h, int comp, short* out);
/* Coefficient tables, for cross-checks of the set-up: g1,g2,gm1,gm2 each
 * num_media+1 floats. */
int orc_get_g(void* h, float* g1, float* g2, float* gm1, float* gm2);
/* which: 0..5 = Idxe Idye Idze Idxh Idyh Idzh, 6..17 = P_be_x,y,z P_ce_x,y,z
 * P_bm_x,y,z P_cm_x,y,z; arrays cover the Alloc range of the matching
 * component axis (see orc_get_metric_range). */
int orc_get_metric(void* h, int which, float* out);
int orc_get_metric_range(void* h, int which, int* lo, int* hi);
/* Per dispersive medium m (0-based in creation order): numpoles, kappa,
 * beta, g3 as interleaved doubles (re, im).  orc_get_mdisp: the same for
 * the magnetic media (GM3 in g3). */
int orc_get_edisp(void* h, int m, int* medium_index, int* npoles, double* kappa,
                  double* beta, double* g3);
int orc_get_mdisp(void* h, int m, int* medium_index, int* npoles, double* kappa,
                  double* beta, double* g3);
double orc_get_time(void* h, int n);
/* CAB1 of calc_murconstants (bordersmur.F90:316-363) for face f (back, front,
 * left, right, down, up), num_media+1 values; returns 1 when the face has no
 * Mur condition. */
int orc_get_mur_cab1(void* h, int face, float* out);
/* Incid as the observation flush calls it: the incident field of component
 * comp at node (i, j, k) summed over the plane waves, at nt real(4) times. */
/* OpenMP threads of the following orc_run calls. */
void orc_set_threads(void* h, int nthreads);
int orc_incident(void* h, int comp, int i, int j, int k, int nt, const float* t, float* out);
/* Checks the library's quotient by dt, RN(q + (a - dt*q)*y) with y = RN(1/dt)
 * and q = RN(a*y) (two FMAs), against IEEE division a/dt for n operands
 * drawn from `seed` over the whole finite exponent range that does not
 * underflow; returns the number of differing results. */
long orc_check_div_dt(double dt, long n, unsigned long long seed);

#ifdef __cplusplus
}
#endif
#endif
