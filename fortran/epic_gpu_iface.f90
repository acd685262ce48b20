! =============================================================================
! ISO_C_BINDING interfaces of the B200 EPIC step (include/epic_gpu.h).
! Replaces, under ENABLE_B200, the calls of the run loop at
! src/3d/epic3d.f90:137-151: create, set_parcels, init_correction, then one
! epic_gpu_step per iteration of the run loop and get_parcels at output steps.
! =============================================================================
module epic_gpu_iface
    use iso_c_binding
    implicit none

    integer(c_int), parameter :: EPIC_OK = 0

    type, bind(C) :: epic_cfg
        integer(c_int32_t) :: nx, ny, nz
        real(c_double)     :: lower(3), extent(3)
        real(c_double)     :: size_factor, grow_factor, shrink_factor
        integer(c_int32_t) :: n_per_cell
        real(c_double)     :: lambda_max, min_vratio
        integer(c_int32_t) :: correction_iters
        real(c_double)     :: gradient_pref, max_compression
        real(c_double)     :: t_initial, t_limit, alpha
        integer(c_int32_t) :: precise_stop, use_fixed_dt
        real(c_double)     :: fixed_dt
        integer(c_int32_t) :: rk_order
        real(c_double)     :: gravity, L_v, c_p, theta_0, q_0, height_c, ang_vel, lat_degrees
        integer(c_int32_t) :: l_planetary_vorticity
        integer(c_int32_t) :: bndry_zeta_zero(2)
        integer(c_int64_t) :: capacity
        integer(c_int32_t) :: precision
        integer(c_int32_t) :: keep_order
        ! damping (options.f90:112-122): the reference's logicals as 0 / 1
        real(c_double)     :: damping_vorticity_prefactor, damping_scalars_prefactor
        integer(c_int32_t) :: damping_vorticity, damping_surface_vorticity
        integer(c_int32_t) :: damping_scalars, damping_surface_scalars
        integer(c_int32_t) :: labels, label_seed
    end type epic_cfg

    type, bind(C) :: epic_step_info
        real(c_double)     :: t, dt
        integer(c_int64_t) :: n_parcels, n_splits, n_merges
        real(c_double)     :: parcel_stats(18)
        real(c_double)     :: field_stats(11)
    end type epic_step_info

    interface
        integer(c_int) function epic_gpu_default_config(cfg) bind(C, name="epic_gpu_default_config")
            import :: c_int, epic_cfg
            type(epic_cfg), intent(inout) :: cfg
        end function

        integer(c_int) function epic_gpu_create(cfg, ctx) bind(C, name="epic_gpu_create")
            import :: c_int, c_ptr, epic_cfg
            type(epic_cfg), intent(in) :: cfg
            type(c_ptr), intent(out)   :: ctx
        end function

        subroutine epic_gpu_destroy(ctx) bind(C, name="epic_gpu_destroy")
            import :: c_ptr
            type(c_ptr), value :: ctx
        end subroutine

        type(c_ptr) function epic_gpu_last_error(ctx) bind(C, name="epic_gpu_last_error")
            import :: c_ptr
            type(c_ptr), value :: ctx
        end function

        integer(c_int) function epic_gpu_set_parcels(ctx, n, pos, vor, B, vol, buoy, hum) &
                bind(C, name="epic_gpu_set_parcels")
            import :: c_int, c_int64_t, c_ptr, c_double
            type(c_ptr), value         :: ctx
            integer(c_int64_t), value  :: n
            real(c_double), intent(in) :: pos(3, *), vor(3, *), B(5, *), vol(*), buoy(*), hum(*)
        end function

        integer(c_int) function epic_gpu_get_parcels(ctx, cap, n, pos, vor, B, vol, buoy, hum) &
                bind(C, name="epic_gpu_get_parcels")
            import :: c_int, c_int64_t, c_ptr, c_double
            type(c_ptr), value          :: ctx
            integer(c_int64_t), value   :: cap
            integer(c_int64_t)          :: n
            real(c_double), intent(out) :: pos(3, *), vor(3, *), B(5, *), vol(*), buoy(*), hum(*)
        end function

        integer(c_int) function epic_gpu_init_correction(ctx) bind(C, name="epic_gpu_init_correction")
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function

        integer(c_int) function epic_gpu_step(ctx, t, info) bind(C, name="epic_gpu_step")
            import :: c_int, c_ptr, c_double, epic_step_info
            type(c_ptr), value   :: ctx
            real(c_double)       :: t
            type(epic_step_info) :: info
        end function

        ! setup_fields_and_parcels from a field file: parcel_default,
        ! init_parcels_from_grids, set_zeta_boundary_flag (vortg(:,:,:,1:3))
        integer(c_int) function epic_gpu_init_from_grids(ctx, vortg, tbuoyg, humg, zeta_flags) &
                bind(C, name="epic_gpu_init_from_grids")
            import :: c_int, c_int32_t, c_ptr, c_double
            type(c_ptr), value          :: ctx
            real(c_double), intent(in)  :: vortg(*), tbuoyg(*), humg(*)
            integer(c_int32_t)          :: zeta_flags(2)
        end function

        ! read_bndry_fluxes: binc, hinc as read from the flux file (y, x)
        integer(c_int) function epic_gpu_set_bndry_fluxes(ctx, bflux, hflux) &
                bind(C, name="epic_gpu_set_bndry_fluxes")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value         :: ctx
            real(c_double), intent(in) :: bflux(*), hflux(*)
        end function

        integer(c_int) function epic_gpu_get_field(ctx, field_id, out) bind(C, name="epic_gpu_get_field")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value     :: ctx
            integer(c_int), value  :: field_id
            real(c_double)         :: out(*)
        end function
        ! labels (cfg%labels = 1): parcels%label, parcels%dilution
        integer(c_int) function epic_gpu_get_labels(ctx, cap, n, label, dilution) &
                bind(C, name="epic_gpu_get_labels")
            import :: c_int, c_int64_t, c_ptr, c_double
            type(c_ptr), value            :: ctx
            integer(c_int64_t), value     :: cap
            integer(c_int64_t)            :: n
            integer(c_int64_t)            :: label(*)
            real(c_double)                :: dilution(*)
        end function

        integer(c_int) function epic_gpu_set_labels(ctx, n, label, dilution) &
                bind(C, name="epic_gpu_set_labels")
            import :: c_int, c_int64_t, c_ptr, c_double
            type(c_ptr), value            :: ctx
            integer(c_int64_t), value     :: n
            integer(c_int64_t), intent(in) :: label(*)
            real(c_double), intent(in)    :: dilution(*)
        end function

        ! parcel and field files in the reference's netCDF layout (epic_nc.h):
        ! write_netcdf_parcels / read_netcdf_parcels (restart) /
        ! write_netcdf_fields / read_netcdf_fields + init_parcels_from_grids;
        ! path is a NUL-terminated string (trim(name) // c_null_char)
        integer(c_int) function epic_gpu_write_parcels_nc(ctx, path, t) &
                bind(C, name="epic_gpu_write_parcels_nc")
            import :: c_int, c_ptr, c_char, c_double
            type(c_ptr), value            :: ctx
            character(kind=c_char)        :: path(*)
            real(c_double), value         :: t
        end function

        integer(c_int) function epic_gpu_read_parcels_nc(ctx, path, t) &
                bind(C, name="epic_gpu_read_parcels_nc")
            import :: c_int, c_ptr, c_char, c_double
            type(c_ptr), value            :: ctx
            character(kind=c_char)        :: path(*)
            real(c_double)                :: t
        end function

        integer(c_int) function epic_gpu_write_fields_nc(ctx, path, t) &
                bind(C, name="epic_gpu_write_fields_nc")
            import :: c_int, c_ptr, c_char, c_double
            type(c_ptr), value            :: ctx
            character(kind=c_char)        :: path(*)
            real(c_double), value         :: t
        end function

        integer(c_int) function epic_gpu_init_from_field_file(ctx, path, zeta_flags) &
                bind(C, name="epic_gpu_init_from_field_file")
            import :: c_int, c_int32_t, c_ptr, c_char
            type(c_ptr), value            :: ctx
            character(kind=c_char)        :: path(*)
            integer(c_int32_t)            :: zeta_flags(2)
        end function

        ! allocation-free vorticity correction on device arrays the caller owns
        ! (OpenACC / CUDA Fortran: pass the device addresses, e.g. from
        ! host_data use_device); no cudaMalloc, a fixed scratch inside the
        ! library, n <= 67108864; dvor_out may be c_null_ptr
        integer(c_int) function epic_gpu_apply_vortcor_noalloc(n, vol, vor, vor_bar, dvor_out, stream) &
                bind(C, name="epic_gpu_apply_vortcor_noalloc")
            import :: c_int, c_int64_t, c_ptr, c_double
            integer(c_int64_t), value  :: n
            type(c_ptr), value         :: vol, vor
            real(c_double), intent(in) :: vor_bar(3)
            type(c_ptr), value         :: dvor_out
            type(c_ptr), value         :: stream
        end function
    end interface

end module epic_gpu_iface
