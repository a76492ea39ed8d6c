! semba_gpu_m -- Fortran 2003 (iso_c_binding) interface to libsemba_gpu.so.
!
! Mirrors include/semba_gpu.h one to one: every struct is a bind(C) derived
! type with the same members in the same order (C arrays [a][b] appear as
! Fortran arrays (b, a)), and every entry point is a bind(C) interface with
! the C name.  Conventions of the interfaces:
!
!   * handles (sgpu_ctx*, sgpu_batch*) are type(c_ptr), passed by value;
!     functions that create one return it in a type(c_ptr) argument;
!   * scalars the C side takes by value are `value` arguments;
!   * descriptors (const sgpu_*_desc*) are the derived types, by reference;
!   * bulk arrays (fields, media, metrics, traces, tables) are type(c_ptr),
!     value: pass c_loc of the Fortran array, which must be contiguous and
!     laid out as the header states (the field and media arrays exactly as
!     launch_simulation allocates them, column-major over sgg%Alloc);
!   * small results (counts, step indices, timings, limits) are Fortran
!     variables or fixed-size arrays by reference;
!   * file names are c_char arrays ending in c_null_char:
!     trim(name)//c_null_char.
!
! Each entry point returns SGPU_OK (0) or one of the SGPU_ERR_* codes; the
! message of a context's last error is sgpu_error_message(ctx).
!
! The per-step entry points replace the routine calls of the reference's
! time loop, timestepping.F90:1286-1742, one for one (Advance_Ex ->
! sgpu_advance_ex, AdvanceelectricCPML -> sgpu_advance_electric_cpml, ...).
module semba_gpu_m
   use iso_c_binding
   implicit none
   private :: c_strlen

   integer(c_int), parameter :: SGPU_OK = 0, SGPU_ERR_ARG = 1, SGPU_ERR_OOM = 2, SGPU_ERR_CUDA = 3, &
                                SGPU_ERR_STATE = 4, SGPU_ERR_NONFINITE = 5, SGPU_ERR_TIMEOUT = 6, &
                                SGPU_ERR_UNSUPPORTED = 7, SGPU_ERR_SIZE = 8

   ! ---- level 1: descriptors of the reference's set-up ---------------------
   type, bind(C) :: sgpu_lim
      integer(c_int) :: xi, xe, yi, ye, zi, ze
   end type sgpu_lim

   type, bind(C) :: sgpu_grid_desc
      type(sgpu_lim) :: alloc(6)
      type(sgpu_lim) :: sweep(6)
      integer(c_int) :: num_media
      type(c_ptr) :: g1, g2, gm1, gm2
      type(c_ptr) :: is_pec
      type(c_ptr) :: idxe, idye, idze, idxh, idyh, idzh
      real(c_double) :: dt
   end type sgpu_grid_desc

   type, bind(C) :: sgpu_cpml_desc
      type(sgpu_lim) :: pmlc(6, 6)          ! (region, component)
      type(c_ptr) :: p_be(3), p_ce(3), p_bm(3), p_cm(3)
   end type sgpu_cpml_desc

   type, bind(C) :: sgpu_edisp_desc
      integer(c_int) :: nmedia
      type(c_ptr) :: medium_index
      type(c_ptr) :: npoles
      type(c_ptr) :: kappa
      type(c_ptr) :: beta
      type(c_ptr) :: g3
   end type sgpu_edisp_desc

   type, bind(C) :: sgpu_planewave_desc
      integer(c_int) :: active(6)
      integer(c_int) :: lim(5, 6, 6)        ! (item, component, face)
      real(c_float) :: px, py, pz, d0, cluz
      real(c_float) :: fpw(6)
      integer(c_int) :: numus
      real(c_float) :: deltaevol
      type(c_ptr) :: evol
      type(c_ptr) :: phys(3, 6)             ! (axis, component)
      integer(c_int) :: phys_lo(3, 6)
      integer(c_int) :: phys_n(3, 6)
   end type sgpu_planewave_desc

   type, bind(C) :: sgpu_nodal_desc
      integer(c_int) :: comp
      integer(c_int) :: hard
      type(sgpu_lim) :: box
      real(c_float) :: amplitude
      integer(c_int) :: numus
      real(c_float) :: deltaevol
      type(c_ptr) :: evol
   end type sgpu_nodal_desc

   type, bind(C) :: sgpu_border_desc
      integer(c_int) :: pmc(6)
      integer(c_int) :: periodic(6)
      integer(c_int) :: mur(6)
      type(c_ptr) :: mur_cab1(6)
   end type sgpu_border_desc

   type, bind(C) :: sgpu_freq_probe_desc
      integer(c_int) :: magnetic
      integer(c_int) :: box(6)
      integer(c_int) :: stride(3)
      integer(c_int) :: nfreq
      type(c_ptr) :: freq
   end type sgpu_freq_probe_desc

   type, bind(C) :: sgpu_movie_probe_desc
      integer(c_int) :: magnetic
      integer(c_int) :: box(6)
      integer(c_int) :: stride(3)
      integer(c_int) :: n_first, n_last, every
      integer(c_int) :: capacity
   end type sgpu_movie_probe_desc

   ! ---- level 2: problem description -------------------------------------
   type, bind(C) :: sgpu_region
      integer(c_int) :: kind
      real(c_float) :: eps, sigma, mu, sigmam
      integer(c_int) :: npoles
      type(c_ptr) :: residues
      type(c_ptr) :: bpoles
      integer(c_int) :: nboxes
      type(c_ptr) :: boxes
      integer(c_int) :: mpoles
      type(c_ptr) :: mresidues
      type(c_ptr) :: mbpoles
   end type sgpu_region

   type, bind(C) :: sgpu_planewave_src
      integer(c_int) :: x1, y1, z1, x2, y2, z2
      real(c_float) :: theta, phi, alpha, beta
      integer(c_int) :: nsamples
      type(c_ptr) :: samples
      real(c_float) :: dsamples
   end type sgpu_planewave_src

   type, bind(C) :: sgpu_nodal_src
      integer(c_int) :: is_elec, is_hard
      integer(c_int) :: npoints
      type(c_ptr) :: boxes
      type(c_ptr) :: amp
      integer(c_int) :: nsamples
      type(c_ptr) :: samples
      real(c_float) :: dsamples
   end type sgpu_nodal_src

   type, bind(C) :: sgpu_problem
      integer(c_int) :: nx, ny, nz
      type(c_ptr) :: desx, desy, desz
      real(c_float) :: originx, originy, originz
      real(c_double) :: dt
      integer(c_int) :: forcecfl
      real(c_float) :: cfl
      integer(c_int) :: pml_layers(6)
      real(c_float) :: pml_order(6)
      real(c_float) :: pml_refl(6)
      real(c_float) :: alphamax, alphaorder, kappamax
      integer(c_int) :: nregions
      type(c_ptr) :: regions
      integer(c_int) :: npw
      type(c_ptr) :: pw
      integer(c_int) :: nnodal
      type(c_ptr) :: nodal
      integer(c_int) :: nprobes
      type(c_ptr) :: probes
      integer(c_int) :: probe_capacity
      integer(c_int) :: border(6)
      integer(c_int) :: mur_after_pml
   end type sgpu_problem

   ! ---- near-to-far-field transform --------------------------------------
   type, bind(C) :: sgpu_farfield_desc
      integer(c_int) :: active(6)
      integer(c_int) :: lim(5, 2, 6)        ! (item, tangential component, face)
      integer(c_int) :: nfreq
      type(c_ptr) :: freq
      integer(c_int) :: ndecim
      real(c_float) :: dtdecim
      real(c_float) :: cluz, zvac
      type(c_ptr) :: cell(6)
      integer(c_int) :: cell_lo(6)
      integer(c_int) :: cell_n(6)
      type(c_ptr) :: phys(3, 3)             ! (axis, component)
      integer(c_int) :: phys_lo(3, 3)
      integer(c_int) :: phys_n(3, 3)
   end type sgpu_farfield_desc

   type, bind(C) :: sgpu_farfield_spec
      integer(c_int) :: box(6)
      integer(c_int) :: faces(6)
      real(c_float) :: initial_freq, final_freq, freq_step
      integer(c_int) :: logarithmic
      integer(c_int) :: decimate
   end type sgpu_farfield_spec

   type, bind(C) :: sgpu_farfield_angles
      real(c_float) :: theta_start, theta_stop, theta_step
      real(c_float) :: phi_start, phi_stop, phi_step
   end type sgpu_farfield_angles

   interface
      ! ---- context -------------------------------------------------------
      integer(c_int) function sgpu_create(grid, out) bind(C, name="sgpu_create")
         import :: c_int, c_ptr, sgpu_grid_desc
         type(sgpu_grid_desc), intent(in) :: grid
         type(c_ptr), intent(out) :: out
      end function sgpu_create
      subroutine sgpu_destroy(ctx) bind(C, name="sgpu_destroy")
         import :: c_ptr
         type(c_ptr), value :: ctx
      end subroutine sgpu_destroy
      type(c_ptr) function sgpu_last_error(ctx) bind(C, name="sgpu_last_error")
         import :: c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_last_error
      integer(c_int) function sgpu_synchronize(ctx) bind(C, name="sgpu_synchronize")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_synchronize
      integer(c_int) function sgpu_get_stream(ctx, stream) bind(C, name="sgpu_get_stream")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         type(c_ptr), intent(out) :: stream  ! the context's cudaStream_t
      end function sgpu_get_stream
      integer(c_int) function sgpu_upload_media(ctx, comp, mi) bind(C, name="sgpu_upload_media")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: comp
         type(c_ptr), value :: mi            ! c_loc(sggMiEx) .. c_loc(sggMiHz), integer(2)
      end function sgpu_upload_media
      integer(c_int) function sgpu_upload_field(ctx, comp, f) bind(C, name="sgpu_upload_field")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: comp
         type(c_ptr), value :: f             ! c_loc(Ex) .. c_loc(Hz)
      end function sgpu_upload_field
      integer(c_int) function sgpu_download_field(ctx, comp, f) bind(C, name="sgpu_download_field")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: comp
         type(c_ptr), value :: f
      end function sgpu_download_field
      integer(c_int) function sgpu_pinned_alloc(bytes, out) bind(C, name="sgpu_pinned_alloc")
         import :: c_int, c_ptr, c_int64_t
         integer(c_int64_t), value :: bytes
         type(c_ptr), intent(out) :: out     ! c_f_pointer it onto the field array
      end function sgpu_pinned_alloc
      integer(c_int) function sgpu_pinned_free(p) bind(C, name="sgpu_pinned_free")
         import :: c_int, c_ptr
         type(c_ptr), value :: p
      end function sgpu_pinned_free

      ! ---- set-up of the per-step routines ---------------------------------
      integer(c_int) function sgpu_init_cpml(ctx, d) bind(C, name="sgpu_init_cpml")
         import :: c_int, c_ptr, sgpu_cpml_desc
         type(c_ptr), value :: ctx
         type(sgpu_cpml_desc), intent(in) :: d
      end function sgpu_init_cpml
      integer(c_int) function sgpu_init_edisp(ctx, d) bind(C, name="sgpu_init_edisp")
         import :: c_int, c_ptr, sgpu_edisp_desc
         type(c_ptr), value :: ctx
         type(sgpu_edisp_desc), intent(in) :: d
      end function sgpu_init_edisp
      integer(c_int) function sgpu_init_mdisp(ctx, d) bind(C, name="sgpu_init_mdisp")
         import :: c_int, c_ptr, sgpu_edisp_desc
         type(c_ptr), value :: ctx
         type(sgpu_edisp_desc), intent(in) :: d
      end function sgpu_init_mdisp
      integer(c_int) function sgpu_add_planewave(ctx, d) bind(C, name="sgpu_add_planewave")
         import :: c_int, c_ptr, sgpu_planewave_desc
         type(c_ptr), value :: ctx
         type(sgpu_planewave_desc), intent(in) :: d
      end function sgpu_add_planewave
      integer(c_int) function sgpu_add_nodal(ctx, d) bind(C, name="sgpu_add_nodal")
         import :: c_int, c_ptr, sgpu_nodal_desc
         type(c_ptr), value :: ctx
         type(sgpu_nodal_desc), intent(in) :: d
      end function sgpu_add_nodal
      integer(c_int) function sgpu_init_borders(ctx, d) bind(C, name="sgpu_init_borders")
         import :: c_int, c_ptr, sgpu_border_desc
         type(c_ptr), value :: ctx
         type(sgpu_border_desc), intent(in) :: d
      end function sgpu_init_borders
      integer(c_int) function sgpu_set_time(ctx, n0, count, tiempo) bind(C, name="sgpu_set_time")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: n0, count
         type(c_ptr), value :: tiempo        ! c_loc(sgg%tiempo(n0))
      end function sgpu_set_time
      integer(c_int) function sgpu_get_time(ctx, n0, count, tiempo) bind(C, name="sgpu_get_time")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: n0, count
         type(c_ptr), value :: tiempo        ! real(c_double) :: tiempo(count)
      end function sgpu_get_time

      ! ---- observation -----------------------------------------------------
      integer(c_int) function sgpu_set_probes(ctx, nprobes, comp_ijk, capacity_steps) bind(C, name="sgpu_set_probes")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: nprobes
         type(c_ptr), value :: comp_ijk      ! integer(c_int) :: comp_ijk(4, nprobes)
         integer(c_int), value :: capacity_steps
      end function sgpu_set_probes
      integer(c_int) function sgpu_read_probes(ctx, out, max_steps, nsteps, first_n) bind(C, name="sgpu_read_probes")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         type(c_ptr), value :: out           ! real(c_float) :: out(nprobes, max_steps)
         integer(c_int), value :: max_steps
         integer(c_int), intent(out) :: nsteps, first_n
      end function sgpu_read_probes
      integer(c_int) function sgpu_add_freq_probe(ctx, d, id) bind(C, name="sgpu_add_freq_probe")
         import :: c_int, c_ptr, sgpu_freq_probe_desc
         type(c_ptr), value :: ctx
         type(sgpu_freq_probe_desc), intent(in) :: d
         integer(c_int), intent(out) :: id
      end function sgpu_add_freq_probe
      integer(c_int) function sgpu_add_movie_probe(ctx, d, id) bind(C, name="sgpu_add_movie_probe")
         import :: c_int, c_ptr, sgpu_movie_probe_desc
         type(c_ptr), value :: ctx
         type(sgpu_movie_probe_desc), intent(in) :: d
         integer(c_int), intent(out) :: id
      end function sgpu_add_movie_probe
      integer(c_int) function sgpu_volume_probe_shape(ctx, id, ni, nj, nk, ijk0) bind(C, name="sgpu_volume_probe_shape")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: id
         integer(c_int), intent(out) :: ni, nj, nk
         integer(c_int), intent(out) :: ijk0(3)
      end function sgpu_volume_probe_shape
      integer(c_int) function sgpu_read_freq_probe(ctx, id, out) bind(C, name="sgpu_read_freq_probe")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: id
         type(c_ptr), value :: out           ! complex(c_double_complex) :: out(ni, nj, nk, 3, nfreq)
      end function sgpu_read_freq_probe
      integer(c_int) function sgpu_read_movie_probe(ctx, id, out, max_frames, frames, first_n) &
            bind(C, name="sgpu_read_movie_probe")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: id
         type(c_ptr), value :: out           ! real(c_float) :: out(ni, nj, nk, 3, max_frames)
         integer(c_int), value :: max_frames
         integer(c_int), intent(out) :: frames, first_n
      end function sgpu_read_movie_probe

      ! ---- one call per reference routine (timestepping.F90:1286-1742) ------
      integer(c_int) function sgpu_advance_ex(ctx) bind(C, name="sgpu_advance_ex")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_ex
      integer(c_int) function sgpu_advance_ey(ctx) bind(C, name="sgpu_advance_ey")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_ey
      integer(c_int) function sgpu_advance_ez(ctx) bind(C, name="sgpu_advance_ez")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_ez
      integer(c_int) function sgpu_advance_electric_cpml(ctx) bind(C, name="sgpu_advance_electric_cpml")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_electric_cpml
      integer(c_int) function sgpu_advance_edispersive_e(ctx) bind(C, name="sgpu_advance_edispersive_e")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_edispersive_e
      integer(c_int) function sgpu_advance_planewave_e(ctx, n) bind(C, name="sgpu_advance_planewave_e")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: n
      end function sgpu_advance_planewave_e
      integer(c_int) function sgpu_advance_nodal_e(ctx, n) bind(C, name="sgpu_advance_nodal_e")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: n
      end function sgpu_advance_nodal_e
      integer(c_int) function sgpu_advance_hx(ctx) bind(C, name="sgpu_advance_hx")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_hx
      integer(c_int) function sgpu_advance_hy(ctx) bind(C, name="sgpu_advance_hy")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_hy
      integer(c_int) function sgpu_advance_hz(ctx) bind(C, name="sgpu_advance_hz")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_hz
      integer(c_int) function sgpu_advance_magnetic_cpml(ctx) bind(C, name="sgpu_advance_magnetic_cpml")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_magnetic_cpml
      integer(c_int) function sgpu_advance_planewave_h(ctx, n) bind(C, name="sgpu_advance_planewave_h")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: n
      end function sgpu_advance_planewave_h
      integer(c_int) function sgpu_advance_nodal_h(ctx, n) bind(C, name="sgpu_advance_nodal_h")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: n
      end function sgpu_advance_nodal_h
      integer(c_int) function sgpu_advance_mdispersive_h(ctx) bind(C, name="sgpu_advance_mdispersive_h")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_mdispersive_h
      integer(c_int) function sgpu_advance_pmc_h(ctx) bind(C, name="sgpu_advance_pmc_h")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_pmc_h
      integer(c_int) function sgpu_advance_periodic_h(ctx) bind(C, name="sgpu_advance_periodic_h")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_periodic_h
      integer(c_int) function sgpu_advance_magnetic_mur(ctx) bind(C, name="sgpu_advance_magnetic_mur")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_advance_magnetic_mur
      integer(c_int) function sgpu_update_observation(ctx, n) bind(C, name="sgpu_update_observation")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: n
      end function sgpu_update_observation

      ! ---- fused forms -----------------------------------------------------
      integer(c_int) function sgpu_advance_e(ctx, n) bind(C, name="sgpu_advance_e")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: n
      end function sgpu_advance_e
      integer(c_int) function sgpu_advance_h(ctx, n) bind(C, name="sgpu_advance_h")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: n
      end function sgpu_advance_h
      integer(c_int) function sgpu_advance_steps(ctx, n0, count) bind(C, name="sgpu_advance_steps")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: n0, count
      end function sgpu_advance_steps
      integer(c_int) function sgpu_set_kernel_family(ctx, family) bind(C, name="sgpu_set_kernel_family")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: family
      end function sgpu_set_kernel_family
      integer(c_int) function sgpu_set_wait_cycles(ctx, cycles) bind(C, name="sgpu_set_wait_cycles")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: ctx
         integer(c_int64_t), value :: cycles
      end function sgpu_set_wait_cycles
      integer(c_int) function sgpu_set_wait_drill(ctx, on) bind(C, name="sgpu_set_wait_drill")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: on
      end function sgpu_set_wait_drill
      integer(c_int) function sgpu_check_finite(ctx) bind(C, name="sgpu_check_finite")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function sgpu_check_finite
      integer(c_int) function sgpu_elapsed_steps(ctx, n0, count, ms) bind(C, name="sgpu_elapsed_steps")
         import :: c_int, c_ptr, c_float
         type(c_ptr), value :: ctx
         integer(c_int), value :: n0, count
         real(c_float), intent(out) :: ms
      end function sgpu_elapsed_steps
      integer(c_int) function sgpu_profile_steps(ctx, n0, count, ms6) bind(C, name="sgpu_profile_steps")
         import :: c_int, c_ptr, c_float
         type(c_ptr), value :: ctx
         integer(c_int), value :: n0, count
         real(c_float), intent(out) :: ms6(6)
      end function sgpu_profile_steps
      integer(c_int) function sgpu_algorithmic_bytes(ctx, bytes6) bind(C, name="sgpu_algorithmic_bytes")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: bytes6(6)
      end function sgpu_algorithmic_bytes
      integer(c_int) function sgpu_compulsory_bytes(ctx, bytes6) bind(C, name="sgpu_compulsory_bytes")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: bytes6(6)
      end function sgpu_compulsory_bytes
      integer(c_int) function sgpu_trim_device_memory() bind(C, name="sgpu_trim_device_memory")
         import :: c_int
      end function sgpu_trim_device_memory
      integer(c_int) function sgpu_select_device(device) bind(C, name="sgpu_select_device")
         import :: c_int
         integer(c_int), value :: device
      end function sgpu_select_device
      integer(c_int) function sgpu_kernels_per_step(ctx, n) bind(C, name="sgpu_kernels_per_step")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), intent(out) :: n
      end function sgpu_kernels_per_step
      integer(c_int) function sgpu_scan_nonfinite_noalloc(data, n, stream, count, first_index) &
            bind(C, name="sgpu_scan_nonfinite_noalloc")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: data          ! device memory
         integer(c_int64_t), value :: n
         type(c_ptr), value :: stream
         integer(c_int64_t), intent(out) :: count, first_index
      end function sgpu_scan_nonfinite_noalloc
      integer(c_int) function sgpu_device_bytes(ctx, bytes) bind(C, name="sgpu_device_bytes")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: ctx
         integer(c_int64_t), intent(out) :: bytes
      end function sgpu_device_bytes

      ! ---- level 2: problem-level host --------------------------------------
      integer(c_int) function sgpu_host_create(p, max_steps, out) bind(C, name="sgpu_host_create")
         import :: c_int, c_ptr, sgpu_problem
         type(sgpu_problem), intent(in) :: p
         integer(c_int), value :: max_steps
         type(c_ptr), intent(out) :: out
      end function sgpu_host_create
      integer(c_int) function sgpu_host_plan(p, max_steps, out) bind(C, name="sgpu_host_plan")
         import :: c_int, c_ptr, sgpu_problem
         type(sgpu_problem), intent(in) :: p
         integer(c_int), value :: max_steps
         type(c_ptr), intent(out) :: out
      end function sgpu_host_plan
      integer(c_int) function sgpu_host_footprint(ctx, bytes) bind(C, name="sgpu_host_footprint")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: ctx
         integer(c_int64_t), intent(out) :: bytes
      end function sgpu_host_footprint
      integer(c_int) function sgpu_host_info(ctx, dt, num_media, alloc6, sweep6, sinpml6) bind(C, name="sgpu_host_info")
         import :: c_int, c_ptr, c_double, sgpu_lim
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: dt
         integer(c_int), intent(out) :: num_media
         type(sgpu_lim), intent(out) :: alloc6(6), sweep6(6), sinpml6(6)
      end function sgpu_host_info
      integer(c_int) function sgpu_host_get_g(ctx, g1, g2, gm1, gm2) bind(C, name="sgpu_host_get_g")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         type(c_ptr), value :: g1, g2, gm1, gm2   ! real(c_float) :: g1(0:num_media), ...
      end function sgpu_host_get_g
      integer(c_int) function sgpu_host_get_metric(ctx, which, out, lo, hi) bind(C, name="sgpu_host_get_metric")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: which
         type(c_ptr), value :: out
         integer(c_int), intent(out) :: lo, hi
      end function sgpu_host_get_metric
      integer(c_int) function sgpu_host_get_media(ctx, comp, out) bind(C, name="sgpu_host_get_media")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: comp
         type(c_ptr), value :: out
      end function sgpu_host_get_media
      integer(c_int) function sgpu_host_get_mur_cab1(ctx, face, out) bind(C, name="sgpu_host_get_mur_cab1")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: face
         type(c_ptr), value :: out
      end function sgpu_host_get_mur_cab1
      integer(c_int) function sgpu_host_create_zslab(p, max_steps, z0, z1, out) bind(C, name="sgpu_host_create_zslab")
         import :: c_int, c_ptr, sgpu_problem
         type(sgpu_problem), intent(in) :: p
         integer(c_int), value :: max_steps, z0, z1
         type(c_ptr), intent(out) :: out
      end function sgpu_host_create_zslab
      integer(c_int) function sgpu_zplane(ctx, comp, z, ptr, bytes) bind(C, name="sgpu_zplane")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: ctx
         integer(c_int), value :: comp, z
         type(c_ptr), intent(out) :: ptr     ! device address
         integer(c_int64_t), intent(out) :: bytes
      end function sgpu_zplane
      integer(c_int) function sgpu_copy_zplane(dst, src, comp, z) bind(C, name="sgpu_copy_zplane")
         import :: c_int, c_ptr
         type(c_ptr), value :: dst, src
         integer(c_int), value :: comp, z
      end function sgpu_copy_zplane
      integer(c_int) function sgpu_host_get_constants(ctx, eps0, mu0) bind(C, name="sgpu_host_get_constants")
         import :: c_int, c_ptr, c_float
         type(c_ptr), value :: ctx
         real(c_float), intent(out) :: eps0, mu0
      end function sgpu_host_get_constants
      integer(c_int) function sgpu_host_incident(ctx, comp, i, j, k, nt, t, out) bind(C, name="sgpu_host_incident")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: comp, i, j, k, nt
         type(c_ptr), value :: t             ! real(c_float) :: t(nt)
         type(c_ptr), value :: out           ! real(c_float) :: out(nt)
      end function sgpu_host_incident

      ! ---- restart files (resuming.F90:213-496) ------------------------------
      integer(c_int) function sgpu_store_resume(ctx, path, last_step, eps0, mu0) bind(C, name="sgpu_store_resume")
         import :: c_int, c_ptr, c_char, c_float
         type(c_ptr), value :: ctx
         character(kind=c_char), intent(in) :: path(*)
         integer(c_int), value :: last_step
         real(c_float), value :: eps0, mu0
      end function sgpu_store_resume
      integer(c_int) function sgpu_load_resume(ctx, path, last_step) bind(C, name="sgpu_load_resume")
         import :: c_int, c_ptr, c_char
         type(c_ptr), value :: ctx
         character(kind=c_char), intent(in) :: path(*)
         integer(c_int), intent(out) :: last_step
      end function sgpu_load_resume

      ! ---- batched form --------------------------------------------------------
      integer(c_int) function sgpu_batch_create(arena_bytes, max_instances, out) bind(C, name="sgpu_batch_create")
         import :: c_int, c_ptr, c_int64_t
         integer(c_int64_t), value :: arena_bytes
         integer(c_int), value :: max_instances
         type(c_ptr), intent(out) :: out
      end function sgpu_batch_create
      subroutine sgpu_batch_destroy(b) bind(C, name="sgpu_batch_destroy")
         import :: c_ptr
         type(c_ptr), value :: b
      end subroutine sgpu_batch_destroy
      type(c_ptr) function sgpu_batch_last_error(b) bind(C, name="sgpu_batch_last_error")
         import :: c_ptr
         type(c_ptr), value :: b
      end function sgpu_batch_last_error
      integer(c_int) function sgpu_batch_add(b, p, plan, nsteps, slot) bind(C, name="sgpu_batch_add")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         type(c_ptr), value :: p             ! c_loc(problem) or c_null_ptr
         type(c_ptr), value :: plan          ! from sgpu_host_plan, or c_null_ptr
         integer(c_int), value :: nsteps
         integer(c_int), intent(out) :: slot
      end function sgpu_batch_add
      integer(c_int) function sgpu_batch_remove(b, slot) bind(C, name="sgpu_batch_remove")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         integer(c_int), value :: slot
      end function sgpu_batch_remove
      integer(c_int) function sgpu_batch_advance(b, nsteps) bind(C, name="sgpu_batch_advance")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         integer(c_int), value :: nsteps
      end function sgpu_batch_advance
      integer(c_int) function sgpu_batch_synchronize(b) bind(C, name="sgpu_batch_synchronize")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
      end function sgpu_batch_synchronize
      integer(c_int) function sgpu_batch_elapsed(b, nsteps, ms) bind(C, name="sgpu_batch_elapsed")
         import :: c_int, c_ptr, c_float
         type(c_ptr), value :: b
         integer(c_int), value :: nsteps
         real(c_float), intent(out) :: ms
      end function sgpu_batch_elapsed
      integer(c_int) function sgpu_batch_slot_info(b, slot, steps_done, steps_total, nprobes) &
            bind(C, name="sgpu_batch_slot_info")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         integer(c_int), value :: slot
         integer(c_int), intent(out) :: steps_done, steps_total, nprobes
      end function sgpu_batch_slot_info
      integer(c_int) function sgpu_batch_read_probes(b, slot, out, max_rows, rows) bind(C, name="sgpu_batch_read_probes")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         integer(c_int), value :: slot
         type(c_ptr), value :: out           ! real(c_float) :: out(nprobes, max_rows)
         integer(c_int), value :: max_rows
         integer(c_int), intent(out) :: rows
      end function sgpu_batch_read_probes
      integer(c_int) function sgpu_batch_instance(b, slot, ctx) bind(C, name="sgpu_batch_instance")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         integer(c_int), value :: slot
         type(c_ptr), intent(out) :: ctx
      end function sgpu_batch_instance
      integer(c_int) function sgpu_batch_memory(b, capacity, in_use, largest_free) bind(C, name="sgpu_batch_memory")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: b
         integer(c_int64_t), intent(out) :: capacity, in_use, largest_free
      end function sgpu_batch_memory
      integer(c_int) function sgpu_batch_footprint(plan, bytes, largest) bind(C, name="sgpu_batch_footprint")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: plan
         integer(c_int64_t), intent(out) :: bytes, largest
      end function sgpu_batch_footprint
      integer(c_int) function sgpu_batch_set_kernel_family(b, family) bind(C, name="sgpu_batch_set_kernel_family")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         integer(c_int), value :: family
      end function sgpu_batch_set_kernel_family
      integer(c_int) function sgpu_batch_set_wait_cycles(b, cycles) bind(C, name="sgpu_batch_set_wait_cycles")
         import :: c_int, c_ptr, c_int64_t
         type(c_ptr), value :: b
         integer(c_int64_t), value :: cycles
      end function sgpu_batch_set_wait_cycles
      integer(c_int) function sgpu_batch_set_wait_drill(b, on) bind(C, name="sgpu_batch_set_wait_drill")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         integer(c_int), value :: on
      end function sgpu_batch_set_wait_drill
      integer(c_int) function sgpu_batch_set_tuning(b, chunk3, ctas_per_sm) bind(C, name="sgpu_batch_set_tuning")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         type(c_ptr), value :: chunk3        ! c_loc(chunk(1:3)) or c_null_ptr
         integer(c_int), value :: ctas_per_sm
      end function sgpu_batch_set_tuning
      integer(c_int) function sgpu_batch_get_tuning(b, chunk3, ctas_per_sm) bind(C, name="sgpu_batch_get_tuning")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         integer(c_int), intent(out) :: chunk3(3)
         integer(c_int), intent(out) :: ctas_per_sm
      end function sgpu_batch_get_tuning
      integer(c_int) function sgpu_batch_autotune(b, steps_per_trial, chunk3, ctas_per_sm) bind(C, name="sgpu_batch_autotune")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         integer(c_int), value :: steps_per_trial
         integer(c_int), intent(out) :: chunk3(3)
         integer(c_int), intent(out) :: ctas_per_sm
      end function sgpu_batch_autotune
      integer(c_int) function sgpu_batch_profile_steps(b, nsteps, ms6) bind(C, name="sgpu_batch_profile_steps")
         import :: c_int, c_ptr, c_float
         type(c_ptr), value :: b
         integer(c_int), value :: nsteps
         real(c_float), intent(out) :: ms6(6)
      end function sgpu_batch_profile_steps
      integer(c_int) function sgpu_batch_steps(b, counter) bind(C, name="sgpu_batch_steps")
         import :: c_int, c_ptr
         type(c_ptr), value :: b
         integer(c_int), intent(out) :: counter
      end function sgpu_batch_steps

      ! ---- near-to-far-field transform (farfield.F90) ---------------------------
      integer(c_int) function sgpu_add_farfield(ctx, d, id) bind(C, name="sgpu_add_farfield")
         import :: c_int, c_ptr, sgpu_farfield_desc
         type(c_ptr), value :: ctx
         type(sgpu_farfield_desc), intent(in) :: d
         integer(c_int), intent(out) :: id
      end function sgpu_add_farfield
      integer(c_int) function sgpu_host_add_farfield(ctx, s, id) bind(C, name="sgpu_host_add_farfield")
         import :: c_int, c_ptr, sgpu_farfield_spec
         type(c_ptr), value :: ctx
         type(sgpu_farfield_spec), intent(in) :: s
         integer(c_int), intent(out) :: id
      end function sgpu_host_add_farfield
      integer(c_int) function sgpu_farfield_shape(ctx, id, nfreq, samples) bind(C, name="sgpu_farfield_shape")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: id
         integer(c_int), intent(out) :: nfreq, samples
      end function sgpu_farfield_shape
      integer(c_int) function sgpu_read_farfield(ctx, id, face, slot, dims, out) bind(C, name="sgpu_read_farfield")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: id, face, slot
         integer(c_int), intent(out) :: dims(2)
         type(c_ptr), value :: out           ! complex(c_double_complex) :: out(inner, outer, nfreq), or c_null_ptr
      end function sgpu_read_farfield
      integer(c_int) function sgpu_farfield_transform(ctx, id, a, incident, n_incident, out, max_rows, rows) &
            bind(C, name="sgpu_farfield_transform")
         import :: c_int, c_ptr, sgpu_farfield_angles
         type(c_ptr), value :: ctx
         integer(c_int), value :: id
         type(sgpu_farfield_angles), intent(in) :: a
         type(c_ptr), value :: incident      ! real(c_float) :: incident(2, n_incident), (time, value) pairs
         integer(c_int), value :: n_incident
         type(c_ptr), value :: out           ! real(c_double) :: out(9, max_rows)
         integer(c_int), value :: max_rows
         integer(c_int), intent(out) :: rows
      end function sgpu_farfield_transform
   end interface

   interface
      function c_strlen(s) bind(C, name="strlen")
         import :: c_ptr, c_size_t
         type(c_ptr), value :: s
         integer(c_size_t) :: c_strlen
      end function c_strlen
   end interface

contains

   ! The text of a context's last error as a Fortran string.
   function sgpu_error_message(ctx) result(msg)
      type(c_ptr), intent(in) :: ctx
      character(len=:), allocatable :: msg
      type(c_ptr) :: p
      character(kind=c_char), pointer :: chars(:)
      integer :: i, n
      p = sgpu_last_error(ctx)
      if (.not. c_associated(p)) then
         msg = ''
         return
      end if
      n = int(c_strlen(p))
      call c_f_pointer(p, chars, [n])
      allocate (character(len=n) :: msg)
      do i = 1, n
         msg(i:i) = chars(i)
      end do
   end function sgpu_error_message

end module semba_gpu_m
