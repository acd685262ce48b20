/*
 * epic_gpu.h -- C ABI of the B200-native EPIC 3-D parcel step.
 *
 * The reference has no plugin API: the 3-D step is a set of Fortran module
 * procedures acting on module-global state (parcels, fields, inversion
 * tables, options).  Each entry point below replaces one of those calls; the
 * cited file:line is the reference procedure whose semantics it reproduces
 * (paths relative to the EPIC source tree, version 0.14.3).
 *
 * Conventions
 *   - All arithmetic of the plain form is IEEE FP64.
 *   - Parcel arrays use the reference's Fortran layout: an attribute with
 *     c components is a column-major (c, n) array, i.e. the c components of
 *     parcel 0 come first (parcel_container.f90:29-56).  Parcel indices in
 *     the merge/split reports are 1-based like the reference's.
 *   - Gridded fields are exchanged as (nz+3) x ny x nx arrays, z fastest,
 *     z = -1 .. nz+1 (the reference's vertical halo), y = 0 .. ny-1,
 *     x = 0 .. nx-1 (periodic; the reference's x/y halo columns are
 *     periodic copies of these, field_mpi.f90:765-1018).
 *   - Every function returns EPIC_OK (0) or one of the EPIC_ERR_* codes and
 *     leaves a message for epic_gpu_last_error().  The reference aborts via
 *     mpi_exit_on_error (mpi_utils.f90:15-31) in the same situations.
 *   - A context is not thread-safe; it owns one CUDA stream and all device
 *     memory of one simulation.  Host arrays are never retained.
 */
#ifndef EPIC_GPU_H
#define EPIC_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EPIC_OK               0
#define EPIC_ERR_CONFIG       1  /* invalid configuration (options.f90, parameters.f90:93-165) */
#define EPIC_ERR_CAPACITY     2  /* parcel container full (parcel_split.f90:93-98 would resize) */
#define EPIC_ERR_NUMERICAL    3  /* B33 division by small number, dt <= 0, no near neighbour */
#define EPIC_ERR_CUDA         4  /* CUDA runtime error */
#define EPIC_ERR_TIMEOUT      5  /* a bounded device wait gave up */
#define EPIC_ERR_ARG          6  /* bad argument (null pointer, size) */
#define EPIC_ERR_STATE        7  /* call out of order (e.g. step before set_parcels) */
#define EPIC_ERR_PARCEL_COUNT 8  /* par2grid parcel count check (parcel_interpl.f90:248-250) */
#define EPIC_ERR_IO           9  /* file missing, unreadable or of another layout (include/epic_nc.h) */

/* Field identifiers for epic_gpu_get_field / epic_gpu_set_field
 * (fields.f90:21-51). */
enum epic_field_id {
    EPIC_FIELD_VELOG_X = 0, EPIC_FIELD_VELOG_Y = 1, EPIC_FIELD_VELOG_Z = 2,
    EPIC_FIELD_VORTG_X = 3, EPIC_FIELD_VORTG_Y = 4, EPIC_FIELD_VORTG_Z = 5,
    EPIC_FIELD_VTEND_X = 6, EPIC_FIELD_VTEND_Y = 7, EPIC_FIELD_VTEND_Z = 8,
    /* velocity gradient tensor: du/dx du/dy du/dz dv/dx dv/dy dv/dz dw/dx dw/dy */
    EPIC_FIELD_VELGRAD_0 = 9,  /* .. 16 */
    EPIC_FIELD_TBUOYG = 17, EPIC_FIELD_DBUOYG = 18, EPIC_FIELD_HUMG = 19,
    EPIC_FIELD_VOLG = 20,
    EPIC_FIELD_NPARG = 21, EPIC_FIELD_NSPARG = 22,   /* returned as doubles */
    EPIC_FIELD_COUNT = 23
};

/* Precision forms. */
#define EPIC_PRECISION_FP64  0   /* plain: every quantity FP64 */
#define EPIC_PRECISION_MIXED 1   /* FP32 attributes/interpolation/FFTs, FP64 positions,
                                    volume, RK position update, B33 and tridiagonal */

/* Run configuration: the reference's &EPIC and &PHYSICS namelists plus the
 * domain read from its field file (options.f90:35-122, physics.f90:47-89,
 * parameters.f90:93-165).  Fill with epic_gpu_default_config first. */
typedef struct epic_cfg {
    int32_t nx, ny, nz;             /* grid cells                               */
    double  lower[3];               /* domain origin                            */
    double  extent[3];              /* domain size                              */
    /* parcel options (options.f90:83-97) */
    double  size_factor;            /* 1.0                                      */
    double  grow_factor;            /* 1.2                                      */
    double  shrink_factor;          /* 0.8                                      */
    int32_t n_per_cell;             /* 8                                        */
    double  lambda_max;             /* 4.0                                      */
    double  min_vratio;             /* 20.0                                     */
    int32_t correction_iters;       /* 2                                        */
    double  gradient_pref;          /* 1.8                                      */
    double  max_compression;        /* 0.5                                      */
    /* time options (options.f90:101-110) */
    double  t_initial;              /* 0                                        */
    double  t_limit;                /* 0                                        */
    double  alpha;                  /* 0.2                                      */
    int32_t precise_stop;           /* 0                                        */
    int32_t use_fixed_dt;           /* 0                                        */
    double  fixed_dt;               /* 1.0                                      */
    int32_t rk_order;               /* 4 (5-stage) or 3                         */
    /* physics (physics.f90:47-89) */
    double  gravity, L_v, c_p, theta_0, q_0, height_c, ang_vel, lat_degrees;
    int32_t l_planetary_vorticity;  /* 0                                        */
    /* boundary (options.f90:35-50, parameters.f90:168-217) */
    int32_t bndry_zeta_zero[2];     /* l_bndry_zeta_zero(lower, upper)          */
    /* device capacity in parcels (0 = derive like max_num_parcels,
       parameters.f90:152-163) */
    int64_t capacity;
    int32_t precision;              /* EPIC_PRECISION_*                         */
    int32_t keep_order;             /* 1: keep the reference's parcel order     */
    /* damping (options.f90:112-122, parcel_damping.f90:43-225); at most one
       of damping_vorticity / damping_surface_vorticity and of
       damping_scalars / damping_surface_scalars */
    double  damping_vorticity_prefactor;   /* 1.0                            */
    double  damping_scalars_prefactor;     /* 1.0                            */
    int32_t damping_vorticity;             /* 0                              */
    int32_t damping_surface_vorticity;     /* 0                              */
    int32_t damping_scalars;               /* 0                              */
    int32_t damping_surface_scalars;       /* 0                              */
    /* labels (the reference's ENABLE_LABELS build): a 64-bit label and a
       dilution per parcel, set at initialisation, copied by split and chosen
       at random, weighted by volume, in merge (parcel_merge.f90:181-203) */
    int32_t labels;                        /* 0: off                          */
    int32_t label_seed;                    /* key of the merge's random draws */
} epic_cfg;

/* Per-step report (epic3d.f90:135-153 plus the statistics the reference
 * computes every step, parcel_diagnostics.f90:26-44,
 * field_diagnostics.f90:21-32). */
typedef struct epic_step_info {
    double  t;                      /* time after the step                      */
    double  dt;                     /* time step used                           */
    int64_t n_parcels;              /* parcels after the step                   */
    int64_t n_splits;               /* parcels added by parcel_split            */
    int64_t n_merges;               /* small parcels merged by parcel_merge     */
    double  parcel_stats[18];       /* IDX_APE .. IDX_MAX_BUOY, 0-based         */
    double  field_stats[11];        /* IDX_RMS_V .. IDX_MIN_BUOY, 0-based       */
} epic_step_info;

typedef struct epic_ctx epic_ctx;

/* Defaults of options.f90 / physics.f90 for an nx*ny*nz grid. */
int epic_gpu_default_config(epic_cfg* cfg);

/* Allocate the device state for one simulation (replaces field_alloc,
 * parcels%allocate, init_inversion: fields.f90:59-101,
 * parcel_ellipsoid.f90:86-133, inversion_utils.f90:79-253). */
int epic_gpu_create(const epic_cfg* cfg, epic_ctx** out);
void epic_gpu_destroy(epic_ctx* ctx);
const char* epic_gpu_last_error(const epic_ctx* ctx);
int epic_gpu_sync(epic_ctx* ctx);

/* Copy parcels in/out (Fortran container layout, parcel_container.f90:18-106).
 * pos, vor: (3,n); B: (5,n) = B11,B12,B13,B22,B23; vol, buoy, hum: (n). */
int epic_gpu_set_parcels(epic_ctx* ctx, int64_t n, const double* pos, const double* vor,
                         const double* B, const double* vol, const double* buoy,
                         const double* hum);
int epic_gpu_get_parcels(epic_ctx* ctx, int64_t cap, int64_t* n, double* pos, double* vor,
                         double* B, double* vol, double* buoy, double* hum);
int epic_gpu_num_parcels(epic_ctx* ctx, int64_t* n);
/* Labels and dilutions of the parcels (cfg.labels = 1; EPIC_ERR_STATE
 * otherwise), in the order of epic_gpu_get_parcels.  set_parcels zeroes them;
 * the initial states set label = 1 + the regular-position index of
 * init_regular_positions and dilution = 0 (parcel_init.f90:135-139). */
int epic_gpu_get_labels(epic_ctx* ctx, int64_t cap, int64_t* n, int64_t* label, double* dilution);
int epic_gpu_set_labels(epic_ctx* ctx, int64_t n, const int64_t* label, const double* dilution);

/* Initial states generated on the device (no host arrays), the parcels of
 * init_regular_positions / parcel_default (parcel_init.f90:31-152):
 * n_per_cell = npd^3 parcels per cell at the sub-cell centres, z outermost.
 *   EPIC_INIT_THERMAL: spheroids of the cell aspect ratio (parcel_default),
 *     zero vorticity and humidity, buoyancy sum_b amp_b exp(-r_b^2 / 0.25)
 *     plus seeded U(-1e-3, 1e-3), positions jittered by seeded
 *     U(-0.1 dx, 0.1 dx) per component (z kept inside the domain);
 *   EPIC_INIT_BELTRAMI: spheres, vorticity of the Beltrami modes (k, l, m)
 *     (models/3d/beltrami_3d.f90:103-122), no buoyancy.
 * Random numbers are SplitMix64 keyed by (seed, parcel index, component), the
 * generator of the Python package (epic_b200/initial.py), so both produce
 * the same state (positions bit for bit; exp, sin and cos to their last bit).
 * Replaces set_parcels + the host generator; call init_correction after. */
#define EPIC_INIT_THERMAL  0
#define EPIC_INIT_BELTRAMI 1
#define EPIC_INIT_DEFAULT  2   /* parcel_default alone (epic_gpu_init_from_grids) */
typedef struct epic_init_spec {
    int32_t  kind;            /* EPIC_INIT_*                                   */
    int32_t  n_per_cell;      /* a cube: 1, 8, 27, ...                         */
    uint64_t seed;            /* thermal noise                                 */
    int32_t  k, l, m;         /* Beltrami modes                                */
    int32_t  n_bubbles;       /* thermal: 1 .. 4                               */
    double   bubble[4][4];    /* thermal: centre x, y, z and amplitude         */
} epic_init_spec;
int epic_gpu_init_state(epic_ctx* ctx, const epic_init_spec* spec);

/* The start of a run from a field file (utils.f90:223-234): parcel_default
 * with init_regular_positions and init_refine (parcel_init.f90:31-166; cfg
 * n_per_cell parcels per cell, split until lambda < lambda_max),
 * init_parcels_from_grids (:170-203: every parcel takes the trilinear
 * interpolation of the fields at its centre) and set_zeta_boundary_flag
 * (parameters.f90:168-217), whose result replaces the configuration's
 * bndry_zeta_zero and is returned in zeta_flags (may be NULL).  vortg holds
 * the x, y, z components one after the other, each a field in the layout of
 * epic_gpu_set_field like tbuoyg and humg (NULL: zero humidity); rows 0..nz
 * are read.  Call init_correction after. */
int epic_gpu_init_from_grids(epic_ctx* ctx, const double* vortg, const double* tbuoyg, const double* humg,
                             int32_t zeta_flags[2]);

/* Autotuner (no counterpart in the reference): times the candidate launch
 * shapes of this context on its own parcels and grid -- the lane grouping of
 * the par2grid / vol2grid scatters and the horizontal FFT path -- and keeps
 * the fastest.  Every candidate computes the same result; only calls that
 * leave the state unchanged are timed (par2grid, vol2grid, FFTs into work
 * arrays).  Call after set_parcels / init_state; out may be NULL. */
typedef struct epic_tuning {
    int32_t lg_par2grid, lg_vol2grid, fft_path;
    int32_t reserved;
    double  ms_par2grid, ms_vol2grid, ms_fft;   /* best times */
} epic_tuning;
int epic_gpu_autotune(epic_ctx* ctx, epic_tuning* out);
/* LS-RK accumulators (delta_pos(3,n), delta_vor(3,n), strain(8,n), delta_b(5,n)). */
int epic_gpu_get_parcel_rk(epic_ctx* ctx, int64_t cap, int64_t* n, double* delta_pos,
                           double* delta_vor, double* strain, double* delta_b);
int epic_gpu_set_parcel_rk(epic_ctx* ctx, int64_t n, const double* delta_pos,
                           const double* delta_vor, const double* delta_b);

/* Gridded fields in the layout described above. */
int epic_gpu_get_field(epic_ctx* ctx, int field_id, double* out);
int epic_gpu_set_field(epic_ctx* ctx, int field_id, const double* in);

/* init_parcel_correction (parcel_correction.f90:42-83): vor_bar = sum(v w)/sum(v). */
int epic_gpu_init_correction(epic_ctx* ctx);
/* apply_vortcor (parcel_correction.f90:89-138). */
int epic_gpu_apply_vortcor(epic_ctx* ctx);
/* par2grid (parcel_interpl.f90:146-323); reuse = l_reuse. */
int epic_gpu_par2grid(epic_ctx* ctx, int reuse);
/* vor2vel + vel2vgrad (inversion.f90:25-317). */
int epic_gpu_vor2vel(epic_ctx* ctx);
/* vorticity_tendency (inversion.f90:321-404). */
int epic_gpu_vorticity_tendency(epic_ctx* ctx);
/* get_time_step (rk_utils.f90:70-183). */
int epic_gpu_time_step(epic_ctx* ctx, double t, double* dt);
/* grid2par (parcel_interpl.f90:405-470); add = present(add) .and. add. */
int epic_gpu_grid2par(epic_ctx* ctx, int add);
/* ls_rk_step (ls_rk.f90:88-136): advances t by dt. */
int epic_gpu_rk_step(epic_ctx* ctx, double* t, double* dt);
/* parcel_merge (parcel_merge.f90:47-108) incl. find_nearest/resolve_tree
 * (parcel_nearest.f90:375-1377) with single-rank semantics; n_merge out. */
int epic_gpu_merge(epic_ctx* ctx, int64_t* n_merge);
/* The merge pairs of the last merge, by epic_gpu_merge or inside epic_gpu_step
 * (isma, iclo; 1-based container indices, m order).  They stay on the device
 * until this call copies them (it synchronises the context's stream). */
int epic_gpu_get_merge_pairs(epic_ctx* ctx, int64_t cap, int64_t* n, int32_t* isma,
                             int32_t* iclo);
/* parcel_split (parcel_split.f90:37-198); n_split out. */
int epic_gpu_split(epic_ctx* ctx, int64_t* n_split);
/* apply_laplace / apply_gradient (parcel_correction.f90:142-259). */
int epic_gpu_apply_laplace(epic_ctx* ctx, int reuse);
int epic_gpu_apply_gradient(epic_ctx* ctx, int reuse);
/* vol2grid (parcel_interpl.f90:92-135). */
int epic_gpu_vol2grid(epic_ctx* ctx, int reuse);
/* calculate_parcel_diagnostics / calculate_field_diagnostics
 * (parcel_diagnostics.f90:51-159, field_diagnostics.f90:40-154). */
int epic_gpu_parcel_diagnostics(epic_ctx* ctx, double stats[18]);
int epic_gpu_field_diagnostics(epic_ctx* ctx, double stats[11]);
/* parcel_damp (parcel_damping.f90:43-78): par2grid, vor2vel, z-halo
 * reflection, get_strain_magnitude_field (rk_utils.f90:186-214) and
 * perturbation_damping (parcel_damping.f90:82-222) with the support points of
 * that par2grid.  ls_rk_step calls it after the last stage when any damping
 * flag of the configuration is set; a no-op otherwise. */
int epic_gpu_parcel_damp(epic_ctx* ctx, double dt);
/* Surface fluxes of buoyancy and humidity (bndry_fluxes.f90:100-175): bflux
 * and hflux are ny x nx arrays, y fastest (the 'bflux' / 'hflux' datasets of
 * the reference's flux file, m^2/s^3 and 1/s times m).  Stored scaled by
 * 2 / dz; from then on ls_rk_step bounds dt by alpha (dz / max|binc|)^(1/3)
 * (bndry_fluxes_time_step, :180-205; not with a fixed dt) and adds the fluxes
 * to the parcels below lower + dz before the first stage (apply_bndry_fluxes,
 * :209-247).  hflux may be NULL (zero humidity flux); bflux == NULL turns the
 * fluxes off (the reference's empty flux_file). */
int epic_gpu_set_bndry_fluxes(epic_ctx* ctx, const double* bflux, const double* hflux);
/* apply_bndry_fluxes (bndry_fluxes.f90:209-247) alone, for a given dt. */
int epic_gpu_apply_bndry_fluxes(epic_ctx* ctx, double dt);
/* One iteration of the run loop (epic3d.f90:135-153): apply_vortcor,
 * ls_rk_step, parcel_merge, parcel_split, correction_iters x
 * (apply_laplace, apply_gradient). */
int epic_gpu_step(epic_ctx* ctx, double* t, epic_step_info* info);

/* Allocation-free vorticity correction.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc: codes whose device memory belongs
 * to another runtime's pool or budget (a Fortran code keeping its parcel
 * arrays in OpenACC or CUDA Fortran device memory), or time loops that must
 * not take an allocation's implicit synchronisation.  vol (n) and vor (3, n)
 * are device arrays owned by the caller; vor is corrected in place by
 * dvor = sum(V w) / sum(V) - vor_bar (the volume-weighted mean vorticity
 * minus its initial value), which is also returned in dvor_out (host; NULL
 * skips the copy and the stream synchronisation).  stream is a cudaStream_t
 * (NULL = default stream).  The only scratch is a fixed 128 KiB __device__
 * array in the library (kept by every GPU that loads it); n above 67,108,864
 * returns EPIC_ERR_CAPACITY.  Every call outside a stream capture looks up
 * that array's device address on the current device; a call on a capturing
 * stream reuses the address of the last call outside a capture, so make a
 * first call on each device before any capture.  All calls share the array:
 * calls whose kernels overlap on the GPU race. */
int epic_gpu_apply_vortcor_noalloc(int64_t n, const double* vol, double* vor, const double vor_bar[3],
                                   double dvor_out[3], void* stream);

/* ------------------------------------------------------------------------
 * Instrumentation.  These have no counterpart in the reference; they expose
 * the context's CUDA stream and CUDA-event timings of one named kernel
 * ("p2g", "g2p", "fft", "merge", ...) for measurement. */
int epic_gpu_get_stream(epic_ctx* ctx, void** stream);
int epic_gpu_profile_kernel(epic_ctx* ctx, const char* name);
int epic_gpu_kernel_time(epic_ctx* ctx, double* total_ms, int64_t* launches);
int epic_gpu_launch_count(int64_t* n);

#ifdef __cplusplus
}
#endif

#endif /* EPIC_GPU_H */
