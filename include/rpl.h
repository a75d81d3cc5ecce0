/*
 * rpl.h -- C-ABI of librpl.so, the B200 (sm_100a) implementation of Ripple.jl's
 * time-step hot path: SSP-RK3 stages fused with WENO5 Doppler transport and
 * spectral refraction, the Q-transform Doppler velocity, and the wind-input /
 * whitecapping source terms.
 *
 * Plain C types only: pointers, sizes, scalars. One CUDA stream per handle; a
 * handle is not thread-safe, different handles may be used from different
 * threads. Every entry point returns an rpl_status; on failure
 * rpl_last_error() returns a thread-local message. No entry point traps or
 * aborts on bad input. Host arrays passed in are copied; the library never
 * keeps a caller's pointer after the call returns.
 *
 * Array layout RPL_LAYOUT_XFAST: element (i,j,m,n) of an (Nx,Ny,Nk,Np) array at
 * i + Nx*(j + Ny*(m + Nk*n)), i.e. the interior of the reference's ProductField
 * flat_data (src/ProductFields/product_field.jl:65-82) without its halo and
 * z slab. 2-D (Nx,Ny) and 3-D (Nx,Ny,Nz|Nk) arrays follow the same x-fastest rule.
 *
 * Reference interfaces each entry point replaces are cited per declaration
 * (paths inside NumericalEarth/Ripple.jl).
 */
#ifndef RPL_H
#define RPL_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RPL_ABI_VERSION 2

typedef struct rpl_handle rpl_handle;

typedef enum rpl_status {
    RPL_OK = 0,
    RPL_ERR_ARGUMENT = 1,     /* bad descriptor, size or pointer (reference: ArgumentError) */
    RPL_ERR_DT = 2,           /* dt <= 0 or non-finite (time_step.jl:120) */
    RPL_ERR_NONFINITE = 3,    /* non-finite input values */
    RPL_ERR_CUDA = 4,         /* CUDA runtime error */
    RPL_ERR_OOM = 5,          /* device allocation failed or would exceed the memory limit */
    RPL_ERR_STATE = 6,        /* call out of order (e.g. refraction step before rpl_set_currents) */
    RPL_ERR_UNSUPPORTED = 7,  /* configuration outside the B200 path (e.g. non-periodic x,y) */
    RPL_ERR_DEVICE = 8        /* a kernel raised its error word (non-finite state produced) */
} rpl_status;

typedef enum rpl_precision { RPL_FP64 = 0, RPL_FP32 = 1 } rpl_precision;
typedef enum rpl_dtype { RPL_F64 = 0, RPL_F32 = 1 } rpl_dtype;
typedef enum rpl_layout { RPL_LAYOUT_XFAST = 0 } rpl_layout;

typedef enum rpl_transport {
    RPL_TRANSPORT_NONE = 0,        /* no transport (source-only columns) */
    RPL_TRANSPORT_REFRACTION = 1,  /* wave_current_refraction.jl:74-151 (needs rpl_set_currents) */
    RPL_TRANSPORT_INTRINSIC = 2    /* intrinsic_transport.jl:14-68 */
} rpl_transport;

typedef enum rpl_depth_kind {
    RPL_DEPTH_INFINITE = 0,  /* deep water, cell-averaged c_g (transport.jl:61-70) */
    RPL_DEPTH_CONSTANT = 1,  /* cell-centre finite-depth c_g (transport.jl:72-83) */
    RPL_DEPTH_FIELD = 2      /* per-(i,j) depth, x fastest */
} rpl_depth_kind;

typedef enum rpl_wind_kind {
    RPL_WIND_NONE = 0,
    RPL_WIND_UNIFORM = 1,    /* scalar U10 and direction */
    RPL_WIND_HOLLAND = 2,    /* HollandHurricaneWind + LinearStormTrack, evaluated on the device */
    RPL_WIND_FIELD = 3       /* per-(i,j) U10 and direction from rpl_set_wind_field */
} rpl_wind_kind;

/* Model descriptor: the data SpectralWaveModel(grid, spectral_grid; depth, ...) carries
 * (src/Models/spectral_wave_model.jl:155-211) restricted to this path. */
typedef struct rpl_desc {
    int32_t abi_version;        /* RPL_ABI_VERSION */
    int32_t precision;          /* rpl_precision of the state and stencil arithmetic */
    int32_t transport;          /* rpl_transport */
    int32_t device;             /* CUDA device ordinal */
    int64_t Nx, Ny, Nk, Np;     /* physical cells and (kappa, phi) bins */
    double dx, dy;              /* first(xspacings(grid)), first(yspacings(grid)) */
    const double* xnodes;       /* Nx cell centres (wind evaluation) */
    const double* ynodes;       /* Ny cell centres */
    int32_t periodic_x, periodic_y;  /* must both be 1 for any transport (tendencies.jl:43-50) */
    const double* kappa;        /* Nk centres, strictly increasing, > 0 */
    const double* kappa_faces;  /* Nk+1 faces */
    const double* phi;          /* Np centres */
    const double* phi_faces;    /* Np+1 faces */
    int32_t depth_kind;         /* rpl_depth_kind: model depth for dispersion */
    double depth_constant;
    const double* depth_field;  /* Nx*Ny */
    double gravity;             /* 9.81 in the reference */
    int64_t memory_limit_bytes; /* 0: no limit; else creation fails with RPL_ERR_OOM above it */
    const double* xspacings;    /* Nx cell widths Δx(i) and Ny cell heights Δy(j): the total action sums */
    const double* yspacings;    /* m0(i,j)·Δx(i)·Δy(j) (diagnostic_operations.jl:492-503); NULL: dx, dy */
} rpl_desc;

/* Source bundle: PrecomputedSources(wind_input=PressureCorrelationInput(...),
 * dissipation=LocalSaturationDissipation(...)) (src/Physics/Packages/precomputed_sources.jl:179-191),
 * or either term alone (stress_cap = 0 reproduces a bare PressureCorrelationInput). */
typedef struct rpl_sources {
    int32_t wind_kind;          /* rpl_wind_kind */
    int32_t stress_cap;         /* 1: wave-supported stress cap (precomputed_sources.jl:282-326) */
    int32_t drag_form;          /* 0: BulkWindDrag(:linear), 1: BulkWindDrag(:capped) (drag.jl:77-86) */
    int32_t rotation;           /* Holland: +1 counterclockwise, -1 clockwise */
    double wind_speed, wind_direction;           /* RPL_WIND_UNIFORM */
    double vmax, rmax, radius, shape_parameter;  /* RPL_WIND_HOLLAND (winds.jl:200-229) */
    double inflow_angle, background_x, background_y;
    int64_t n_track;            /* 0: fixed centre (track_x[0], track_y[0]) */
    const double* track_t;      /* LinearStormTrack times (winds.jl:115-152) */
    const double* track_x;
    const double* track_y;
    /* PressureCorrelationInput parameters (pressure_correlation.jl:39-52) */
    double beta_max, z_alpha, p_in, alpha0, rho_air, rho_water, von_karman, wind_gravity;
    /* LocalSaturationDissipation parameters (local_saturation.jl:18-28) */
    int32_t has_dissipation;
    int32_t reserved;
    double C_ds, B_r, ds_p, sigma_power, ds_gravity;
} rpl_sources;

/* Replaces SpectralWaveModel construction (spectral_wave_model.jl:155-211): validates the descriptor,
 * allocates the device state (three state buffers, coefficient tables) and builds the c_g tables
 * (transport.jl:111-139). The action starts at zero like WaveActionField (product_field.jl:310). */
int rpl_create(const rpl_desc* desc, rpl_handle** out);
int rpl_destroy(rpl_handle* h);

/* Replaces build_coupling(PrescribedVelocities) + update_coupling! (lagrangian_velocities.jl:286-292,
 * current_coupling.jl:127-138): Q-transform Doppler velocity U and dU/dkappa on the device
 * (doppler_velocity.jl:45-82, q_kernel.jl:60-116) and their periodic gradients
 * (wave_current_refraction.jl:7-39). u, v: (Nx,Ny,Nz) x fastest; z_faces: Nz+1 increasing;
 * q_depth: column depth for the projection (grid depth for InfiniteDepth, lagrangian_velocities.jl:192-194). */
int rpl_set_currents(rpl_handle* h, int64_t Nz, const double* z_faces,
                     int32_t q_depth_kind, double q_depth_constant, const double* q_depth_field,
                     const double* u, const double* v, double small_mu);
/* Replaces update_coupling!(coupling::CWCMPrescribedCurrentCoupling) after the current fields changed
 * (current_coupling.jl:127-138): recomputes the Doppler velocity, its gradients and the stage
 * coefficients from new u, v ((Nx,Ny,Nz) x fastest, host memory) on the Q grid of the last
 * rpl_set_currents, in stream order and without allocating, so time-varying currents can be refreshed
 * every step. The copies are stream-ordered: pinned host buffers must stay unchanged until the next
 * rpl_sync. Values are not scanned on the host; non-finite currents surface as RPL_ERR_DEVICE from the
 * step that uses them. */
int rpl_update_currents(rpl_handle* h, const double* u, const double* v);
/* The same with u, v in device memory on the handle's device (read in stream order, not copied). */
int rpl_update_currents_device(rpl_handle* h, const double* u, const double* v);
/* Replaces build_coupling(PseudomomentumVelocities) + CWCMPseudomomentumCoupling
 * (lagrangian_velocities.jl:294-311, current_coupling.jl:93-118): builds the vertical overlap tables of
 * the Q transform (pseudomomentum.jl:68-121; one Nk x Nk pair for RPL_DEPTH_CONSTANT, one per (i,j) for
 * RPL_DEPTH_FIELD) and the first-moment measures (polar_wavevector_grid.jl:73-110). From then on every
 * RK3 stage and rpl_tendency recompute the Doppler velocity from that stage's action
 * (current_coupling.jl:140-143, tendencies.jl:103-107, pseudomomentum.jl:123-138,316-342). Needs
 * RPL_TRANSPORT_REFRACTION and Nk <= 256; z_faces: Nz+1 increasing; q_depth as for rpl_set_currents.
 * A later rpl_set_currents switches back to prescribed currents. The coupling starts at zero. */
int rpl_set_pseudomomentum(rpl_handle* h, int64_t Nz, const double* z_faces, int32_t q_depth_kind,
                           double q_depth_constant, const double* q_depth_field, double small_mu);
/* Replaces update_coupling!(model) (current_coupling.jl:140-148): with pseudomomentum velocities,
 * recomputes the coupling from the current action; with prescribed currents, nothing to do. */
int rpl_update_coupling(rpl_handle* h);
/* Copies the cached coupling fields to the host (coupling.Ux/Uy/dUxdkappa/dUydkappa and
 * coupling.Ux_x/Ux_y/Uy_x/Uy_y of current_coupling.jl:19-39); any pointer may be NULL. (Nx,Ny,Nk) each. */
int rpl_get_coupling(rpl_handle* h, double* Ux, double* Uy, double* dUxdk, double* dUydk,
                     double* Uxx, double* Uxy, double* Uyx, double* Uyy);

/* Replaces SpectralWaveModel(...; propagation_smoothing=SpatialAveraging(; αs, αn)) and
 * apply_propagation_smoothing! after every step (propagation_smoothing.jl:20-199, time_step.jl:168):
 * kind 1 = SpatialAveraging (Tolman 2002 GSE alleviation), 0 = none. The averaging runs on the device
 * after each RK3 step, in the state's precision with FP64 corner positions. */
int rpl_set_propagation_smoothing(rpl_handle* h, int32_t kind, double alpha_s, double alpha_n);

/* Replaces the sources kwarg + prepare_sources (precomputed_sources.jl:386-394). */
int rpl_set_sources(rpl_handle* h, const rpl_sources* s);
/* Host-evaluated wind (any wind struct of src/Forcing/winds.jl) for RPL_WIND_FIELD: (Nx,Ny) arrays. */
int rpl_set_wind_field(rpl_handle* h, const double* U10, const double* direction);

/* Source terms of a SourceTermSet (src/Sources/Sources.jl:5-11,443-449) whose tendency is linear in the
 * action: each adds positive - damping * N with (positive, damping) from split_growth_rate (wind input)
 * or split_damping_rate (dissipation) of its rate (Sources.jl:430-434). */
typedef enum rpl_term_kind {
    RPL_TERM_EXPONENTIAL_WIND = 1, /* ExponentialWindInput (Sources.jl:32-39,492-496): rate times the cell
                                      average of max(cos(phi - direction), 0)^p[0], p[0] a nonnegative integer */
    RPL_TERM_WAVE_AGE_WIND = 2,    /* WaveAgeWindInput (Sources.jl:67-95,522-554): p = (inverse wave-age
                                      threshold, power, spreading power), gravity */
    RPL_TERM_WHITECAPPING = 3,     /* WhitecappingDissipation (Sources.jl:105-122,583-598): p = (saturation
                                      threshold, saturation power, wavenumber power, reference wavenumber) */
    RPL_TERM_MEAN_SPECTRUM = 4     /* MeanSpectrumWhitecapping (mean_spectrum.jl:20-111): p = (C_ds, delta1,
                                      delta2, mean exponent), gravity */
} rpl_term_kind;
#define RPL_MAX_TERMS 8

typedef struct rpl_source_term {
    int32_t kind;               /* rpl_term_kind */
    int32_t reserved;
    double rate;                /* a Number rate, or rate_field (Nx,Ny, x fastest) when not NULL */
    const double* rate_field;
    double direction;           /* wind direction of the wind-input terms */
    double speed;               /* WaveAgeWindInput speed, or speed_field (Nx,Ny) when not NULL */
    const double* speed_field;
    double p[4];                /* per kind, see rpl_term_kind */
    double gravity;
} rpl_source_term;

/* Replaces sources=SourceTermSet(terms...) (or one such term) on this path: up to RPL_MAX_TERMS terms,
 * evaluated on the device before every stage (per-(i,j) moments by a warp per column, then a rate per
 * cell-bin) and applied inside the stage kernels; count = 0 removes them. May be combined with
 * rpl_set_sources (the bundle's tendency comes first). Fields are copied. */
int rpl_set_source_terms(rpl_handle* h, const rpl_source_term* terms, int32_t count);

/* Replaces set!(model, N=array) / set!(::ProductField, ::AbstractArray) (set.jl:20-30,44-48). */
int rpl_set_action(rpl_handle* h, const void* N, int32_t dtype, int32_t layout);
/* Replaces interior(model.action) (product_field.jl:232-235). */
int rpl_get_action(rpl_handle* h, void* N, int32_t dtype, int32_t layout);
/* Device-resident variants: N points to device memory on the handle's device (same layout). */
int rpl_set_action_device(rpl_handle* h, const void* N, int32_t dtype, int32_t layout);
int rpl_get_action_device(rpl_handle* h, void* N, int32_t dtype, int32_t layout);

/* Clock (Oceananigans Clock of spectral_wave_model.jl:148): time and iteration. */
int rpl_set_clock(rpl_handle* h, double time, int64_t iteration);
int rpl_get_clock(rpl_handle* h, double* time, int64_t* iteration);

/* Replaces time_step!(model, dt) with timestepper=:RK3 (time_step.jl:119-170), nsteps times.
 * Returns after the stream has drained and the kernels' error word was checked. */
int rpl_step(rpl_handle* h, double dt, int64_t nsteps);
/* Same launches, no final synchronisation or error-word check (use rpl_sync). */
int rpl_step_async(rpl_handle* h, double dt, int64_t nsteps);
/* Launches exactly one RK3 stage (1, 2 or 3) of the step starting at the current clock; for
 * per-kernel timing. Stage 3 advances the clock. */
int rpl_stage_async(rpl_handle* h, double dt, int32_t stage);
/* Part of one RK3 stage for a decomposed domain (no counterpart in the reference): the stage kernel
 * updates rows row0 .. row0+nrows-1 only (nrows may be 0); RPL_STAGE_PREPARE first runs the stage's
 * column-local preparation kernels (wind, stress cap, pseudomomentum refresh, source-term rates) over
 * every row, RPL_STAGE_FINISH completes the stage (after stage 3: SpatialAveraging, clock advance).
 * A stage split into launches gives exactly the full stage when the row ranges cover the rows once, the
 * first launch prepares and the last finishes. rpl_stage_async(h, dt, s) is
 * rpl_stage_rows_async(h, dt, s, 0, Ny, RPL_STAGE_PREPARE | RPL_STAGE_FINISH). */
#define RPL_STAGE_PREPARE 1
#define RPL_STAGE_FINISH 2
/* With RPL_STAGE_FINISH on stage 3 of a model with SpatialAveraging: finish the stage without the
 * averaging (stage 3's result stays in the stage buffer A, rpl_rows_get which 1), so that a decomposed
 * domain can refresh A's halo rows first and then average with rpl_smooth_rows_async. */
#define RPL_STAGE_DEFER_SMOOTH 4
int rpl_stage_rows_async(rpl_handle* h, double dt, int32_t stage, int64_t row0, int64_t nrows, int32_t flags);
/* The SpatialAveraging of a step (propagation_smoothing.jl:60-199, time_step.jl:168) for rows
 * row0 .. row0+nrows-1 only: reads the stage buffer A (stage 3's result after RPL_STAGE_DEFER_SMOOTH),
 * writes N. The rows an averaged row reads are up to its corners' reach away (within one row on the
 * 3 x 3 path); they are the caller's to provide. y_offset: the model's row 0 is row y_offset of a
 * larger grid (a slab of a decomposed domain; else 0); the corner positions are computed at the larger
 * grid's row indices so that they round as in the undecomposed model. RPL_ERR_STATE without
 * SpatialAveraging. */
int rpl_smooth_rows_async(rpl_handle* h, double dt, int64_t row0, int64_t nrows, int64_t y_offset);
int rpl_sync(rpl_handle* h);
/* Use the caller's CUDA stream (a cudaStream_t on the handle's device) instead of the handle's own. */
int rpl_set_stream(rpl_handle* h, void* stream);

/* Replaces compute_tendencies!(model) (tendencies.jl:18-41,82-101): G of the current action
 * (transport plus sources) copied to the host in FP64. For testing. */
int rpl_tendency(rpl_handle* h, double* G, int32_t layout);

/* Replaces m0, significant_wave_height, root_mean_square_wavenumber, mean_direction
 * (moments.jl:33-123, bulk_statistics.jl:9) as (Nx,Ny) fields and total_action (bulk_statistics.jl:87-91)
 * as a scalar; FP64 with compensated sums on the device. Any pointer may be NULL. */
int rpl_diagnostics(rpl_handle* h, double* m0, double* hs, double* krms, double* mean_dir,
                    double* total_action);

/* The diagnostics of rpl_diagnostics written to device memory on the handle's device, enqueued on the
 * handle's stream without waiting (a per-step time series needs no host round trip); any pointer may
 * be NULL. */
int rpl_diagnostics_device(rpl_handle* h, double* m0, double* hs, double* krms, double* mean_dir,
                           double* total_action);

/* Row copies for a y-slab domain decomposition (no counterpart in the reference, which runs one domain
 * per architecture). which: 0 = N (the step's state, input of stage 1), 1 = A (input of stage 2),
 * 2 = B (input of stage 3). Rows row0 .. row0+nrows-1 of every direction move between the state buffer
 * and a packed device buffer of (Np, nrows, Nx, Nk) words of the state's type (kappa fastest),
 * stream-ordered on the handle's stream without waiting. A decomposed step copies each slab's
 * boundary rows out, exchanges them, copies them into the halo rows, then runs rpl_stage_async. */
int rpl_rows_get(rpl_handle* h, int32_t which, int64_t row0, int64_t nrows, void* dst);
int rpl_rows_set(rpl_handle* h, int32_t which, int64_t row0, int64_t nrows, const void* src);
/* The same copies on the caller's stream (a cudaStream_t on the handle's device), so that an exchange
 * can run beside the stage kernel of the rows that do not read the halo (rpl_stage_rows_async). */
int rpl_rows_get_on(rpl_handle* h, int32_t which, int64_t row0, int64_t nrows, void* dst, void* stream);
int rpl_rows_set_on(rpl_handle* h, int32_t which, int64_t row0, int64_t nrows, const void* src, void* stream);

/* Replaces fetch_output(field::ProductField, model) = interior(field) (OceananigansIntegration.jl:7-9)
 * for output writers: enqueues a copy of the current action, converted to `dtype` in RPL_LAYOUT_XFAST,
 * into `host` (Nx*Ny*Nk*Np values) and returns at once. The conversion runs on the handle's stream
 * into a staging buffer in device memory (allocated at the first call; RPL_ERR_OOM beyond the memory
 * limit); the device-to-host copy runs on a second stream while later steps proceed. `host` must stay
 * valid until rpl_snapshot_wait; pinned memory (rpl_host_alloc) lets the copy overlap the steps. A new
 * snapshot waits on the device for the previous copy. */
int rpl_snapshot_async(rpl_handle* h, void* host, int32_t dtype);
/* Blocks until the last snapshot has reached the host. */
int rpl_snapshot_wait(rpl_handle* h);
/* Page-locked host memory for snapshots and state transfers (cudaHostAlloc / cudaFreeHost). */
int rpl_host_alloc(int64_t bytes, void** ptr);
int rpl_host_free(void* ptr);

/* Largest Nx*Ny that rpl_diagnostics_static accepts (2048 x 2048 cells). */
#define RPL_STATIC_MAX_COLUMNS 4194304

/* No counterpart in the reference. The diagnostics of rpl_diagnostics for a wave action the caller
 * already holds on the device, for callers that must not allocate device memory when they ask for
 * them: a host framework whose device memory belongs entirely to its own pool allocator (Julia's
 * CUDA.jl pool, PyTorch's caching allocator), or work enqueued while such a framework captures a
 * stream. Needs no handle and allocates nothing: every pointer is device memory on the calling
 * thread's current device. N: (Nx,Ny,Nk,Np) RPL_LAYOUT_XFAST of dtype; measures: 4*Nk*Np FP64 in
 * the order spectral weights, first-moment x, first-moment y, second-moment trace (each (Nk,Np),
 * kappa fastest; polar_wavevector_grid.jl:44-47,73-115); outputs m0, hs, krms, mean_dir ((Nx,Ny))
 * and total (1 value) may each be NULL. Kernels go on `stream` (a cudaStream_t, NULL = default).
 * The only scratch, the per-block partial sums of the total action, is a fixed 256 KiB array inside
 * the library that every GPU loading librpl.so keeps until the process exits, so Nx*Ny is limited to
 * RPL_STATIC_MAX_COLUMNS (larger grids return RPL_ERR_ARGUMENT). dx and dy are the cell widths of a
 * uniform horizontal grid (every cell's area is dx*dy in the total); a stretched grid's total action
 * needs rpl_diagnostics, which takes each cell's own widths. Every call reuses that array, so
 * calls that may overlap on the GPU (different streams, different host threads) race and must be
 * ordered by the caller. The first call on each device looks up the array's device address and may
 * load the library's kernels onto that device; make that first call before any stream capture. */
int rpl_diagnostics_static(const void* N, int32_t dtype, int64_t Nx, int64_t Ny, int64_t Nk, int64_t Np,
                           const double* measures, double dx, double dy, double* m0, double* hs,
                           double* krms, double* mean_dir, double* total, void* stream);

/* ---- Ensemble (batching form) ----
 * No counterpart in the reference, which advances one model per time_step! call (time_step.jl:119-170);
 * a Julia caller would otherwise loop time_step! over its members. An ensemble advances many
 * independent FP32 models ("members", each made by rpl_create and set up as usual: currents, action)
 * by one SSP-RK3 step each with three launches in total: per stage one persistent kernel whose CTAs
 * take (member, tile) work items from an atomic counter. One step (counter reset + three launches)
 * is captured once in a CUDA graph and replayed. Members must be FP32, on one device, share one
 * transport kind (refraction or intrinsic), have no sources, 4 <= Nk <= 32 with Nk % 4 == 0 and
 * Nx, Ny >= 3. Each member keeps its own dt; every step advances every member's clock by its dt.
 * The tile shape of each size class (Nx, Ny, Nk, Np, transport, depth kind) comes from the autotuner
 * (rpl_ensemble_autotune) or, untuned, a default per Nk. */
typedef struct rpl_ensemble rpl_ensemble;

typedef struct rpl_ensemble_options {
    int32_t abi_version;          /* RPL_ABI_VERSION */
    int32_t use_graph;            /* 1: replay one captured CUDA graph per step; 0: three launches */
    int32_t autotune;             /* 1: tune size classes missing from the cache during creation */
    int32_t direct_cells;         /* > 0: members of at least this many cells (Nx*Ny) take their own
                                     single-model stage launches inside the step, the rest share the
                                     persistent launches; 0: every member in the persistent launches */
    const char* autotune_cache;   /* text file of tuned shapes, read at creation and appended to by
                                     the autotuner; NULL: no file */
} rpl_ensemble_options;

int rpl_ensemble_create(rpl_handle* const* members, const double* dt, int32_t count,
                        const rpl_ensemble_options* options, rpl_ensemble** out);
int rpl_ensemble_destroy(rpl_ensemble* e);
/* nsteps RK3 steps of every member; returns after the work drained and every member's error word was
 * checked. The _async form only enqueues (the members' streams wait for it); rpl_ensemble_sync checks. */
int rpl_ensemble_step(rpl_ensemble* e, int64_t nsteps);
int rpl_ensemble_step_async(rpl_ensemble* e, int64_t nsteps);
/* The baseline: the same steps as per-member sequential launches of the single-model kernels. */
int rpl_ensemble_step_sequential_async(rpl_ensemble* e, int64_t nsteps);
int rpl_ensemble_sync(rpl_ensemble* e);
/* Times every candidate tile shape of each size class (stage-1 launches into the members' scratch
 * buffers, the state is not changed) and keeps the fastest; force = 0 keeps shapes found in the cache. */
int rpl_ensemble_autotune(rpl_ensemble* e, int32_t force);
/* Tile shape used for member i: kappa-pair lanes per cell, tile width and height in cells. */
int rpl_ensemble_shape(const rpl_ensemble* e, int32_t member, int32_t* lanes, int32_t* tile_x, int32_t* tile_y);
/* Run on the caller's CUDA stream (cudaStream_t on the members' device); invalidates the graph. */
int rpl_ensemble_set_stream(rpl_ensemble* e, void* stream);

/* ---- Learned source (the learned form) ----
 * No counterpart in the reference. A small MLP stands in for the per-cell source-term tendency of
 * PrecomputedSources (precomputed_sources.jl:396-439: stress-capped wind input + whitecapping): inputs
 * are the cell's Nk*Np-bin log action spectrum and 4 extras (U10 / 30, sin and cos of the wind
 * direction, log10(depth) / 4), three GELU hidden layers, output y per bin with source rate S / N =
 * target_scale * sinh(y); the stage then adds N * rate. BF16 weights and activations, FP32
 * accumulation on the tensor cores (tcgen05), FP32 master weights trained with Adam by the library's
 * own forward and backward kernels. Training data come from the plain FP32 sources
 * (rpl_learned_sample). Cells whose inputs leave the training ranges fall back to the plain sources. */
typedef struct rpl_mlp rpl_mlp;

typedef struct rpl_mlp_desc {
    int32_t abi_version;   /* RPL_ABI_VERSION */
    int32_t nbins;         /* spectral inputs and outputs (Nk * Np), a multiple of 128 */
    int32_t hidden;        /* width of the three hidden layers, a multiple of 256 */
    int32_t rows;          /* rows of one pass (training batch capacity, inference chunk), multiple of 128 */
    int32_t device;
    int32_t reserved;
    uint64_t seed;         /* weight initialisation */
    float feature_shift;   /* input x = (log(max(N, log_floor)) - feature_shift) / feature_scale */
    float feature_scale;
    float log_floor;
    float target_scale;    /* network output y = asinh(rate / target_scale) */
} rpl_mlp_desc;

int rpl_mlp_create(const rpl_mlp_desc* d, rpl_mlp** out);
int rpl_mlp_destroy(rpl_mlp* m);
/* Stream of the network's work (a cudaStream_t on its device; NULL: the legacy default stream). Until
 * this is called the network uses a non-blocking stream of its own. The device arrays passed to
 * rpl_mlp_train_step / _gradients / _forward are read and written in that stream's order, so a caller
 * whose allocator recycles memory per stream (PyTorch's) passes its own stream. */
int rpl_mlp_set_stream(rpl_mlp* m, void* stream);
/* Parameters as one FP32 vector: W1 (hidden x nbins), W1e (hidden x 4), b1, W2 (hidden x hidden), b2, W3,
 * b3, W4 (nbins x hidden), b4 (nbins); matrices row-major (output index slowest). */
int rpl_mlp_param_count(const rpl_mlp* m, int64_t* count);
int rpl_mlp_get_params(rpl_mlp* m, float* host);
int rpl_mlp_set_params(rpl_mlp* m, const float* host);
/* Training rows live on the device: X (n x nbins BF16 features), E (n x 4 FP32 extras), T (n x nbins FP32
 * targets). `rows` (device int32, B of them, B a multiple of 128 and <= desc.rows, each < n) picks the
 * batch. Loss = mean squared error over the batch's outputs. rpl_mlp_train_step applies one Adam step
 * (lr, betas 0.9 / 0.999, eps 1e-8; loss may be NULL); rpl_mlp_gradients returns the gradient (host,
 * parameter layout) and the loss without updating. */
int rpl_mlp_train_step(rpl_mlp* m, const void* X, const float* E, const float* T, const int32_t* rows,
                       int32_t B, float lr, double* loss);
int rpl_mlp_gradients(rpl_mlp* m, const void* X, const float* E, const float* T, const int32_t* rows,
                      int32_t B, float* grads, double* loss);
/* Network output Y (n x nbins FP32, device) for n rows of device X, E; n a multiple of 128. */
int rpl_mlp_forward(rpl_mlp* m, const void* X, const float* E, int64_t n, float* Y);
/* The tensor-core GEMM alone (for testing): C (M x N FP32) = A (M x K BF16) * B (N x K BF16)^T, device
 * row-major arrays, M % 128 == 0, N % 128 == 0, K % 64 == 0; stream NULL = default. */
int rpl_gemm_bf16(const void* A, const void* B, float* C, int32_t M, int32_t N, int32_t K, void* stream);
/* rpl_gemm_bf16 with every barrier wait bounded by `wait_limit` polls (0: the default, 2^24). A wait that
 * runs out ends the kernel cleanly (loads and MMAs in flight drained, tensor memory freed) and the call
 * returns RPL_ERR_DEVICE; the context stays usable. No counterpart in the reference: it lets a caller
 * (or a test) check the abort path of the tensor-core kernels without a device fault. */
int rpl_gemm_bf16_bounded(const void* A, const void* B, float* C, int32_t M, int32_t N, int32_t K,
                          uint32_t wait_limit, void* stream);
/* Training pairs of the FP32 handle's current state and clock from its plain sources: for every cell c
 * (c = i + Nx j) row c of X, E and T (device arrays of Nx*Ny rows; T = asinh(rate / target_scale)). */
int rpl_learned_sample(rpl_handle* h, const rpl_mlp* m, void* X, float* E, float* T);
/* Use `m` (NULL: back to the plain sources) for the handle's sources. lo, hi: host arrays of nbins + 4
 * input bounds; a cell with any input outside [lo, hi] uses the plain sources. ylo, yhi (nbins each, or
 * both NULL): bounds the network outputs are clamped to before they become rates (the range of the
 * training targets keeps an extrapolating network from producing rates no source ever had). */
int rpl_set_learned_source(rpl_handle* h, rpl_mlp* m, const float* lo, const float* hi, const float* ylo,
                           const float* yhi);
/* Trust gate of the learned source (no counterpart in the reference): a cell whose network rates would
 * change some bin by more than max_rate_dt of itself in one step (|rate| * dt > max_rate_dt) takes the
 * plain sources for that stage, like an out-of-distribution cell. 0 (the default) disables the gate. */
int rpl_set_learned_gate(rpl_handle* h, double max_rate_dt);
/* Network outputs y of the most recent stage (host, Nx*Ny rows of nbins, row c = cell i + Nx j). */
int rpl_learned_outputs(rpl_handle* h, float* Y);
/* Cells that fell back to the plain sources in the most recent stage. */
int rpl_learned_fallback_cells(rpl_handle* h, int64_t* count);
/* Since rpl_set_learned_source: cell-stages that took the plain sources (out of distribution or gated)
 * and all cell-stages (cells x stages run with the learned source). */
int rpl_learned_fallback_totals(rpl_handle* h, int64_t* fallback_cell_stages, int64_t* cell_stages);

/* Device bytes held by the handle. */
int rpl_device_bytes(rpl_handle* h, int64_t* bytes);
/* Thread-local message of the last failing call on this thread ("" if none). */
const char* rpl_last_error(void);
/* ABI version the library was built with. */
int rpl_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif
