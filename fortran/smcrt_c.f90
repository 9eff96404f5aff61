!> smcrt_c -- Fortran 2008 iso_c_binding interface to libsmcrt_b200.so, the B200
!> photon-packet transport library whose C ABI is include/smcrt.h.
!>
!> signedMCRT (Fortran 2018) links this module to hand its per-packet transport
!> loop -- the OpenMP region of pathlength_scatter (src/kernelsMod.f90:239-326),
!> weight_scatter (:59-160) and test_kernel (:390-437) -- to the GPU.  Every
!> derived type below is interoperable with the C struct of the same name
!> (component order, kinds and array shapes match; C arrays are row-major, so a C
!> double m[4][3] is a Fortran real(c_double) :: m(3, 4) with m(j, i) = M[i][j]).
!> Every C entry point has an interface.  Conventions:
!>   * C pointers that may be NULL, and device pointers (names ending in _dev),
!>     are type(c_ptr), value: pass c_loc(x), a CUDA device address, or c_null_ptr;
!>   * required host arrays are assumed-size dummies (passed by address);
!>   * uint64_t seeds are integer(c_int64_t) (the same 64 bits);
!>   * every integer(c_int32_t) function returns a smcrt_status code (0 = SMCRT_OK);
!>     smcrt_error_message() returns the last failure's text.
!> Build: gfortran -c smcrt_c.f90; link with -L<repo>/signedmcrt_b200/lib -lsmcrt_b200.
module smcrt_c
    use, intrinsic :: iso_c_binding
    implicit none
    private :: c_strlen

    integer(c_int32_t), parameter :: SMCRT_ABI_VERSION_EXPECTED = 5

    ! smcrt_status
    integer(c_int32_t), parameter :: SMCRT_OK = 0, SMCRT_ERR_ARG = 1, SMCRT_ERR_SCENE = 2, SMCRT_ERR_CUDA = 3, &
                                     SMCRT_ERR_DEVICE = 4, SMCRT_ERR_TIMEOUT = 5, SMCRT_ERR_NO_DEVICE = 6
    ! smcrt_prim_kind (src/sdfs/sdfs.f90:494-735)
    integer(c_int32_t), parameter :: SMCRT_SPHERE = 1, SMCRT_BOX = 2, SMCRT_TORUS = 3, SMCRT_CYLINDER = 4, &
                                     SMCRT_TRIPRISM = 5, SMCRT_SEGMENT = 6, SMCRT_CAPSULE = 7, SMCRT_CONE = 8, &
                                     SMCRT_EGG = 9, SMCRT_PLANE = 10
    ! smcrt_csg_op (src/sdfs/sdfModifiers.f90:412-475)
    integer(c_int32_t), parameter :: SMCRT_OP_NONE = 0, SMCRT_OP_UNION = 1, SMCRT_OP_SMOOTH_UNION = 2, &
                                     SMCRT_OP_SUBTRACTION = 3, SMCRT_OP_INTERSECTION = 4
    ! smcrt_modifier (src/sdfs/sdfModifiers.f90:273-375)
    integer(c_int32_t), parameter :: SMCRT_MOD_NONE = 0, SMCRT_MOD_ONION = 1, SMCRT_MOD_REVOLUTION = 2, &
                                     SMCRT_MOD_EXTRUDE = 3, SMCRT_MOD_ELONGATE = 4, SMCRT_MOD_TWIST = 5, &
                                     SMCRT_MOD_BEND = 6
    ! smcrt_source_kind (src/photon.f90)
    integer(c_int32_t), parameter :: SMCRT_SRC_POINT = 1, SMCRT_SRC_PENCIL = 2, SMCRT_SRC_UNIFORM = 3, &
                                     SMCRT_SRC_CIRCULAR = 4, SMCRT_SRC_ANNULUS = 5, SMCRT_SRC_FOCUS = 6
    integer(c_int32_t), parameter :: SMCRT_ANNULUS_TOPHAT = 0, SMCRT_ANNULUS_GAUSSIAN = 1
    ! smcrt_detector_kind (src/detectors/detectors.f90)
    integer(c_int32_t), parameter :: SMCRT_DET_CIRCLE = 1, SMCRT_DET_ANNULUS = 2, SMCRT_DET_CAMERA = 3
    ! smcrt_kernel_kind, smcrt_precision
    integer(c_int32_t), parameter :: SMCRT_KERNEL_PATHLENGTH = 0, SMCRT_KERNEL_WEIGHT = 1, SMCRT_KERNEL_TEST = 2
    integer(c_int32_t), parameter :: SMCRT_FP32 = 0, SMCRT_FP64 = 1
    integer(c_int32_t), parameter :: SMCRT_ORDER_WALK_LAST = 1, SMCRT_ORDER_INTERACT_LAST = 2

    type, bind(C) :: smcrt_prim
        integer(c_int32_t) :: kind, nmods
        real(c_double)     :: transform(3, 4)   ! transform(j, i) = reference M(i, j), rows i = 1..4
        real(c_double)     :: params(8)
        integer(c_int32_t) :: mods(2)           ! innermost first
        real(c_double)     :: mod_params(3, 2)  ! mod_params(:, k) belongs to mods(k)
    end type smcrt_prim

    type, bind(C) :: smcrt_region
        integer(c_int32_t) :: first_prim, nprims, op, layer_id
        real(c_double)     :: k, mus, mua, hgg, n
    end type smcrt_region

    type, bind(C) :: smcrt_scene
        integer(c_int32_t) :: nregions, nprims
        type(c_ptr)        :: regions, prims   ! c_loc(regions(1)), c_loc(prims(1))
    end type smcrt_scene

    type, bind(C) :: smcrt_grid
        integer(c_int32_t) :: nxg, nyg, nzg, reserved
        real(c_double)     :: xmax, ymax, zmax
    end type smcrt_grid

    type, bind(C) :: smcrt_source
        integer(c_int32_t) :: kind, annulus_type
        real(c_double)     :: pos(3), dir(3), point1(3), point2(3), point3(3)
        real(c_double)     :: radius, radius_hi, beta, z_inset
    end type smcrt_source

    type, bind(C) :: smcrt_detector
        integer(c_int32_t) :: kind, layer, nbins, reserved
        real(c_double)     :: pos(3), dir(3), r1, r2, maxval, p2(3), p3(3)
    end type smcrt_detector

    type, bind(C) :: smcrt_options
        integer(c_int32_t) :: kernel, precision, end_early, block_size, blocks_per_sm, max_trace_steps
        real(c_double)     :: eps, normal_h
        integer(c_int32_t) :: instance, timeout_ms
        type(c_ptr)        :: stream
        integer(c_int32_t) :: private_stream, tally_copies, scene_memory, variance, nearest_cache
        integer(c_int32_t) :: shared_fluence, group_order, reserved(3)
    end type smcrt_options

    type, bind(C) :: smcrt_stats
        real(c_double)     :: nscatt
        integer(c_int64_t) :: packets, sdf_evals, voxel_segments, trace_steps, scatters, fresnel_events, &
                              reflections, kills_step_cap, kills_error, rng_draws
        real(c_double)     :: moments(24), kernel_ms
        integer(c_int32_t) :: device_status, reserved
        integer(c_int64_t) :: h2d_bytes, d2h_bytes, variance_overflows, reserved2(5)
    end type smcrt_stats

    type, bind(C) :: smcrt_packet_state
        real(c_double)     :: pos(3), dir(3), weight
        integer(c_int32_t) :: layer, nscatt, ndraws, flags
    end type smcrt_packet_state

    type, bind(C) :: smcrt_tuning
        integer(c_int32_t) :: tally_copies, shared_bins
        real(c_double)     :: packets_per_s
        integer(c_int32_t) :: trials, block_size, slots_per_thread, ctas_per_sm, nearest_cache, shared_fluence
        integer(c_int32_t) :: group_order, reserved
    end type smcrt_tuning

    type, bind(C) :: smcrt_region_optics
        real(c_double)     :: mus, mua, hgg, n
    end type smcrt_region_optics

    interface
        integer(c_int32_t) function smcrt_abi_version() bind(C, name="smcrt_abi_version")
            import :: c_int32_t
        end function smcrt_abi_version

        type(c_ptr) function smcrt_last_error() bind(C, name="smcrt_last_error")
            import :: c_ptr
        end function smcrt_last_error

        integer(c_int32_t) function smcrt_create(scene, grid, source, dets, ndet, opts, ctx) &
                bind(C, name="smcrt_create")
            import :: c_int32_t, c_ptr, smcrt_scene, smcrt_grid, smcrt_source, smcrt_detector, smcrt_options
            type(smcrt_scene), intent(in)    :: scene
            type(smcrt_grid), intent(in)     :: grid
            type(smcrt_source), intent(in)   :: source
            type(smcrt_detector), intent(in) :: dets(*)
            integer(c_int32_t), value        :: ndet
            type(smcrt_options), intent(in)  :: opts
            type(c_ptr), intent(out)         :: ctx
        end function smcrt_create

        subroutine smcrt_destroy(ctx) bind(C, name="smcrt_destroy")
            import :: c_ptr
            type(c_ptr), value :: ctx
        end subroutine smcrt_destroy

        integer(c_int64_t) function smcrt_detector_bins(ctx) bind(C, name="smcrt_detector_bins")
            import :: c_int64_t, c_ptr
            type(c_ptr), value :: ctx
        end function smcrt_detector_bins

        ! jmean (nxg*nyg*nzg FP64, column-major) and det_bins: c_loc(...) or c_null_ptr
        integer(c_int32_t) function smcrt_run(ctx, nphotons, seed, jmean, det_bins, stats) bind(C, name="smcrt_run")
            import :: c_int32_t, c_int64_t, c_ptr
            type(c_ptr), value        :: ctx
            integer(c_int64_t), value :: nphotons, seed
            type(c_ptr), value        :: jmean, det_bins, stats
        end function smcrt_run

        integer(c_int32_t) function smcrt_adjoint(ctx, nphotons, seed, w_dev, gbins_dev, region_group, ngroups, &
                                                  grad, stats) bind(C, name="smcrt_adjoint")
            import :: c_int32_t, c_int64_t, c_ptr, c_double
            type(c_ptr), value             :: ctx
            integer(c_int64_t), value      :: nphotons, seed
            type(c_ptr), value             :: w_dev, gbins_dev
            integer(c_int32_t), intent(in) :: region_group(*)
            integer(c_int32_t), value      :: ngroups
            real(c_double), intent(out)    :: grad(*)
            type(c_ptr), value             :: stats
        end function smcrt_adjoint

        integer(c_int32_t) function smcrt_autotune(ctx, trial_packets, seed, result) bind(C, name="smcrt_autotune")
            import :: c_int32_t, c_int64_t, c_ptr
            type(c_ptr), value        :: ctx
            integer(c_int64_t), value :: trial_packets, seed
            type(c_ptr), value        :: result
        end function smcrt_autotune

        integer(c_int32_t) function smcrt_run_device(ctx, first, count, seed, jmean_dev, det_bins_dev, stats) &
                bind(C, name="smcrt_run_device")
            import :: c_int32_t, c_int64_t, c_ptr
            type(c_ptr), value        :: ctx
            integer(c_int64_t), value :: first, count, seed
            type(c_ptr), value        :: jmean_dev, det_bins_dev, stats
        end function smcrt_run_device

        ! second-moment runs of a context created with opts%variance /= 0
        integer(c_int32_t) function smcrt_run_moments(ctx, nphotons, seed, jmean, jmean2, det_bins, stats) &
                bind(C, name="smcrt_run_moments")
            import :: c_int32_t, c_int64_t, c_ptr
            type(c_ptr), value        :: ctx
            integer(c_int64_t), value :: nphotons, seed
            type(c_ptr), value        :: jmean, jmean2, det_bins, stats
        end function smcrt_run_moments

        integer(c_int32_t) function smcrt_run_device_moments(ctx, first, count, seed, jmean_dev, jmean2_dev, &
                                                             det_bins_dev, stats) &
                bind(C, name="smcrt_run_device_moments")
            import :: c_int32_t, c_int64_t, c_ptr
            type(c_ptr), value        :: ctx
            integer(c_int64_t), value :: first, count, seed
            type(c_ptr), value        :: jmean_dev, jmean2_dev, det_bins_dev, stats
        end function smcrt_run_device_moments

        integer(c_int32_t) function smcrt_replay(ctx, uniforms, offsets, npackets, jmean, det_bins, states, stats) &
                bind(C, name="smcrt_replay")
            import :: c_int32_t, c_int64_t, c_ptr, c_double
            type(c_ptr), value             :: ctx
            real(c_double), intent(in)     :: uniforms(*)
            integer(c_int64_t), intent(in) :: offsets(*)
            integer(c_int64_t), value      :: npackets
            type(c_ptr), value             :: jmean, det_bins, states, stats
        end function smcrt_replay

        integer(c_int32_t) function smcrt_batch_create(scene, grid, source, dets, ndet, opts, ninst, batch) &
                bind(C, name="smcrt_batch_create")
            import :: c_int32_t, c_ptr, smcrt_scene, smcrt_grid, smcrt_source, smcrt_detector, smcrt_options
            type(smcrt_scene), intent(in)    :: scene
            type(smcrt_grid), intent(in)     :: grid
            type(smcrt_source), intent(in)   :: source
            type(smcrt_detector), intent(in) :: dets(*)
            integer(c_int32_t), value        :: ndet
            type(smcrt_options), intent(in)  :: opts
            integer(c_int32_t), value        :: ninst
            type(c_ptr), intent(out)         :: batch
        end function smcrt_batch_create

        integer(c_int32_t) function smcrt_batch_set_optics(batch, optics) bind(C, name="smcrt_batch_set_optics")
            import :: c_int32_t, c_ptr, smcrt_region_optics
            type(c_ptr), value                    :: batch
            type(smcrt_region_optics), intent(in) :: optics(*)   ! optics(i*nregions + r + 1)
        end function smcrt_batch_set_optics

        integer(c_int32_t) function smcrt_batch_launch(batch, nphotons, seeds, use_graph) &
                bind(C, name="smcrt_batch_launch")
            import :: c_int32_t, c_int64_t, c_ptr
            type(c_ptr), value             :: batch
            integer(c_int64_t), intent(in) :: nphotons(*), seeds(*)
            integer(c_int32_t), value      :: use_graph
        end function smcrt_batch_launch

        integer(c_int32_t) function smcrt_batch_wait(batch, jmean, det_bins, per_instance, total) &
                bind(C, name="smcrt_batch_wait")
            import :: c_int32_t, c_ptr
            type(c_ptr), value :: batch, jmean, det_bins, per_instance, total
        end function smcrt_batch_wait

        integer(c_int32_t) function smcrt_batch_device_tallies(batch, jmean_dev, det_bins_dev) &
                bind(C, name="smcrt_batch_device_tallies")
            import :: c_int32_t, c_ptr
            type(c_ptr), value       :: batch
            type(c_ptr), intent(out) :: jmean_dev, det_bins_dev
        end function smcrt_batch_device_tallies

        integer(c_int64_t) function smcrt_batch_stream(batch) bind(C, name="smcrt_batch_stream")
            import :: c_int64_t, c_ptr
            type(c_ptr), value :: batch
        end function smcrt_batch_stream

        subroutine smcrt_batch_destroy(batch) bind(C, name="smcrt_batch_destroy")
            import :: c_ptr
            type(c_ptr), value :: batch
        end subroutine smcrt_batch_destroy

        ! ctxs: array of smcrt_ctx pointers; jmeans/det_bins: arrays of c_loc(...) or c_null_ptr
        integer(c_int32_t) function smcrt_run_batched(ctxs, ninst, nphotons, seeds, jmeans, det_bins, stats) &
                bind(C, name="smcrt_run_batched")
            import :: c_int32_t, c_int64_t, c_ptr, smcrt_stats
            type(c_ptr), intent(in)          :: ctxs(*)
            integer(c_int32_t), value        :: ninst
            integer(c_int64_t), intent(in)   :: nphotons(*), seeds(*)
            type(c_ptr), intent(in)          :: jmeans(*), det_bins(*)
            type(smcrt_stats), intent(inout) :: stats(*)
        end function smcrt_run_batched

        integer(c_int32_t) function smcrt_run_device_static(scene, grid, source, dets, ndet, opts, first, count, &
                                                            seed, jmean_dev, det_bins_dev, stats) &
                bind(C, name="smcrt_run_device_static")
            import :: c_int32_t, c_int64_t, c_ptr, smcrt_scene, smcrt_grid, smcrt_source, smcrt_detector, &
                      smcrt_options
            type(smcrt_scene), intent(in)    :: scene
            type(smcrt_grid), intent(in)     :: grid
            type(smcrt_source), intent(in)   :: source
            type(smcrt_detector), intent(in) :: dets(*)
            integer(c_int32_t), value        :: ndet
            type(smcrt_options), intent(in)  :: opts
            integer(c_int64_t), value        :: first, count, seed
            type(c_ptr), value               :: jmean_dev, det_bins_dev, stats
        end function smcrt_run_device_static

        integer(c_int64_t) function smcrt_static_scratch_bytes() bind(C, name="smcrt_static_scratch_bytes")
            import :: c_int64_t
        end function smcrt_static_scratch_bytes

        integer(c_int32_t) function smcrt_render(scene, precision, samples, extent, image) bind(C, name="smcrt_render")
            import :: c_int32_t, c_double, c_float, smcrt_scene
            type(smcrt_scene), intent(in)  :: scene
            integer(c_int32_t), value      :: precision
            integer(c_int32_t), intent(in) :: samples(3)
            real(c_double), intent(in)     :: extent(3)
            real(c_float), intent(out)     :: image(*)
        end function smcrt_render

        integer(c_int32_t) function smcrt_render_device(scene, precision, samples, extent, image_dev, stream) &
                bind(C, name="smcrt_render_device")
            import :: c_int32_t, c_double, c_ptr, smcrt_scene
            type(smcrt_scene), intent(in)  :: scene
            integer(c_int32_t), value      :: precision
            integer(c_int32_t), intent(in) :: samples(3)
            real(c_double), intent(in)     :: extent(3)
            type(c_ptr), value             :: image_dev, stream
        end function smcrt_render_device

        integer(c_int32_t) function smcrt_eval_sdf(scene, precision, pts, npts, out) bind(C, name="smcrt_eval_sdf")
            import :: c_int32_t, c_int64_t, c_double, smcrt_scene
            type(smcrt_scene), intent(in) :: scene
            integer(c_int32_t), value     :: precision
            real(c_double), intent(in)    :: pts(*)
            integer(c_int64_t), value     :: npts
            real(c_double), intent(out)   :: out(*)
        end function smcrt_eval_sdf

        integer(c_int32_t) function smcrt_calc_normal(scene, region0, h, pts, npts, out_xyz) &
                bind(C, name="smcrt_calc_normal")
            import :: c_int32_t, c_int64_t, c_double, smcrt_scene
            type(smcrt_scene), intent(in) :: scene
            integer(c_int32_t), value     :: region0
            real(c_double), value         :: h
            real(c_double), intent(in)    :: pts(*)
            integer(c_int64_t), value     :: npts
            real(c_double), intent(out)   :: out_xyz(*)
        end function smcrt_calc_normal

        integer(c_int32_t) function smcrt_fresnel(precision, dir_in, normal, n1, n2, n, refl) &
                bind(C, name="smcrt_fresnel")
            import :: c_int32_t, c_int64_t, c_double
            integer(c_int32_t), value   :: precision
            real(c_double), intent(in)  :: dir_in(*), normal(*), n1(*), n2(*)
            integer(c_int64_t), value   :: n
            real(c_double), intent(out) :: refl(*)
        end function smcrt_fresnel

        integer(c_int32_t) function smcrt_reflect_refract(precision, dir_in, normal, n1, n2, u, n, dir_out, &
                                                          reflected) bind(C, name="smcrt_reflect_refract")
            import :: c_int32_t, c_int64_t, c_double
            integer(c_int32_t), value       :: precision
            real(c_double), intent(in)      :: dir_in(*), normal(*), n1(*), n2(*), u(*)
            integer(c_int64_t), value       :: n
            real(c_double), intent(out)     :: dir_out(*)
            integer(c_int32_t), intent(out) :: reflected(*)
        end function smcrt_reflect_refract

        integer(c_int32_t) function smcrt_scatter_dir(precision, dir_in, g, u, n, dir_out) &
                bind(C, name="smcrt_scatter_dir")
            import :: c_int32_t, c_int64_t, c_double
            integer(c_int32_t), value   :: precision
            real(c_double), intent(in)  :: dir_in(*), g(*), u(*)
            integer(c_int64_t), value   :: n
            real(c_double), intent(out) :: dir_out(*)
        end function smcrt_scatter_dir

        integer(c_int32_t) function smcrt_emit(scene, grid, source, precision, first, npk, seed, pos, dir, layer) &
                bind(C, name="smcrt_emit")
            import :: c_int32_t, c_int64_t, c_double, smcrt_scene, smcrt_grid, smcrt_source
            type(smcrt_scene), intent(in)   :: scene
            type(smcrt_grid), intent(in)    :: grid
            type(smcrt_source), intent(in)  :: source
            integer(c_int32_t), value       :: precision
            integer(c_int64_t), value       :: first, npk, seed
            real(c_double), intent(out)     :: pos(*), dir(*)
            integer(c_int32_t), intent(out) :: layer(*)
        end function smcrt_emit

        integer(c_int32_t) function smcrt_philox(key2, ctr4, n, out4) bind(C, name="smcrt_philox")
            import :: c_int32_t, c_int64_t
            integer(c_int32_t), intent(in)  :: key2(*), ctr4(*)
            integer(c_int64_t), value       :: n
            integer(c_int32_t), intent(out) :: out4(*)
        end function smcrt_philox

        integer(c_size_t) function c_strlen(s) bind(C, name="strlen")
            import :: c_size_t, c_ptr
            type(c_ptr), value :: s
        end function c_strlen
    end interface

contains

    !> The message of the last failed call on this thread, as a Fortran string.
    function smcrt_error_message() result(msg)
        character(len=:), allocatable :: msg
        character(kind=c_char), pointer :: chars(:)
        type(c_ptr) :: p
        integer :: i, n
        p = smcrt_last_error()
        if (.not. c_associated(p)) then
            msg = ""
            return
        end if
        n = int(c_strlen(p))
        call c_f_pointer(p, chars, [n])
        allocate(character(len=n) :: msg)
        do i = 1, n
            msg(i:i) = chars(i)
        end do
    end function smcrt_error_message

end module smcrt_c
