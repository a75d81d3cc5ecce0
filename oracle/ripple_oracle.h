/*
 * ripple_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of Ripple.jl's time-step path (NumericalEarth/Ripple.jl).
 * It is the correctness oracle for the CUDA library and the timed CPU baseline.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * arm load it; the product path (librpl.so) never links, loads or calls it.
 *
 * Parity status: pinned against the reference's own known-answer tests
 * (Q-transform integrals and Doppler sums, barotropic currents, WENO5 sinusoid
 * transport, RK3 source column, Holland wind and storm track, bulk drag); the
 * fused 4-D refraction kernel and multi-step RK3 trajectories have no golden
 * vectors in the reference, so for those the restatement itself is the pin.
 *
 * Layout of every 4-D array: x fastest, i.e. element (i,j,m,n) at
 * i + Nx*(j + Ny*(m + Nk*n)), the interior of the reference's
 * ProductField flat_data (src/ProductFields/product_field.jl:65-82) without halo.
 */
#ifndef RIPPLE_ORACLE_H
#define RIPPLE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORA_TRANSPORT_NONE = 0, ORA_TRANSPORT_REFRACTION = 1, ORA_TRANSPORT_INTRINSIC = 2 };
enum { ORA_WIND_NONE = 0, ORA_WIND_UNIFORM = 1, ORA_WIND_HOLLAND = 2, ORA_WIND_FIELD = 3 };

typedef struct ora_holland {
    double vmax, rmax, radius, shape_parameter, inflow_angle;
    double background_x, background_y;
    int32_t rotation;          /* +1 counterclockwise, -1 clockwise */
    int32_t n_track;           /* 0: fixed centre (center_x[0], center_y[0]) */
    const double* track_t;     /* n_track strictly increasing times */
    const double* center_x;    /* n_track (or 1) centres */
    const double* center_y;
} ora_holland;

/* Source terms of a SourceTermSet (src/Sources/Sources.jl:5-11,443-449) whose tendency is linear in the
 * action: positive - damping * N with (positive, damping) from split_growth_rate / split_damping_rate
 * (Sources.jl:430-434). */
enum {
    ORA_TERM_EXPONENTIAL_WIND = 1, /* ExponentialWindInput (Sources.jl:32-39,492-501): p[0] spreading power */
    ORA_TERM_WAVE_AGE_WIND = 2,    /* WaveAgeWindInput (Sources.jl:67-95,522-559): p[0] inverse wave-age
                                      threshold, p[1] power, p[2] spreading power, gravity */
    ORA_TERM_WHITECAPPING = 3,     /* WhitecappingDissipation (Sources.jl:105-122,583-598): p[0] saturation
                                      threshold, p[1] saturation power, p[2] wavenumber power,
                                      p[3] reference wavenumber */
    ORA_TERM_MEAN_SPECTRUM = 4     /* MeanSpectrumWhitecapping (mean_spectrum.jl:20-115): p[0] C_ds,
                                      p[1] delta1, p[2] delta2, p[3] p, gravity */
};

typedef struct ora_term {
    int32_t kind;
    int32_t pad;
    double rate;                /* source_value of a Number; rate_field (Nx,Ny) x fastest when not NULL */
    const double* rate_field;
    double direction;           /* wind direction of the wind-input terms (a Number) */
    double speed;               /* WaveAgeWindInput speed; speed_field (Nx,Ny) when not NULL */
    const double* speed_field;
    double p[4];
    double gravity;
} ora_term;

typedef struct ora_model {
    int64_t Nx, Ny, Nk, Np;
    double dx, dy;                       /* first(xspacings), first(yspacings) */
    const double* xnodes;                /* Nx cell centres */
    const double* ynodes;                /* Ny cell centres */
    const double* kappa;                 /* Nk centres */
    const double* kappa_faces;           /* Nk+1 */
    const double* phi;                   /* Np centres */
    const double* phi_faces;             /* Np+1 */
    const double* weights;               /* (Nk,Np) m fastest */
    int32_t transport;
    int32_t cg_per_cell;                 /* 0: cg tables (Nk,Np); 1: (Nx,Ny,Nk,Np) */
    const double* cg_x;
    const double* cg_y;
    /* refraction inputs, (Nx,Ny,Nk) x fastest */
    const double* Ux; const double* Uy;
    const double* Uxx; const double* Uxy; const double* Uyx; const double* Uyy;
    /* sources: PrecomputedSources(wind_input, dissipation) */
    int32_t wind_kind;
    double wind_speed, wind_direction;   /* ORA_WIND_UNIFORM */
    ora_holland holland;                 /* ORA_WIND_HOLLAND */
    const double* wind_U10;              /* ORA_WIND_FIELD: (Nx,Ny) */
    const double* wind_theta;
    double beta_max, z_alpha, p_in, alpha0, rho_air, rho_water, von_karman, gravity;
    int32_t has_dissipation;
    double C_ds, B_r, ds_p, sigma_power, ds_gravity;
    /* PseudomomentumVelocities (current_coupling.jl:41-118): the Doppler velocity is recomputed from the
     * action before every tendency; Ux..Uyy above are then unused */
    int32_t pm_mode;
    int32_t pm_per_cell;                 /* 1: (Nx,Ny,Nk,Nk) overlap tables */
    const double* pm_overlap;            /* ora_pm_overlap_tables layout */
    const double* pm_kx;                 /* (Nk,Np) first-moment measures */
    const double* pm_ky;
    /* propagation_smoothing = SpatialAveraging(alpha_s, alpha_n) after every RK3 step
     * (propagation_smoothing.jl:20-199, time_step.jl:168) */
    int32_t gse;
    int32_t periodic_x, periodic_y;
    double gse_alpha_s, gse_alpha_n;
    /* per-cell widths Δx(i) (Nx) and heights Δy(j) (Ny) of the total action; NULL: dx, dy */
    const double* xspacings;
    const double* yspacings;
    /* SourceTermSet terms, applied after the bundle above (both may be present) */
    int32_t n_terms;
    const ora_term* terms;
} ora_model;

/* ---- Q kernel (src/Coupling/q_kernel.jl) ---- */
double ora_q_value(double kappa, double z, double depth, double small_mu);
double ora_q_cdf(double kappa, double z, double depth, double small_mu);
double ora_q_cell_integral(double kappa, double z1, double z2, double depth, double small_mu);
double ora_q_cdf_kappa_derivative(double kappa, double z, double depth, double small_mu);
double ora_q_cell_integral_kappa_derivative(double kappa, double z1, double z2, double depth, double small_mu);
double ora_q_cdf_kernel(double kappa, double z, double depth, double small_mu);
double ora_q_cell_integral_kernel(double kappa, double z1, double z2, double depth, double small_mu);
double ora_q_cell_integral_kappa_derivative_kernel(double kappa, double z1, double z2, double depth, double small_mu);

/* ---- Doppler velocity and its gradients ---- */
void ora_doppler_velocity(int64_t Nx, int64_t Ny, int64_t Nz, int64_t Nk,
                          const double* u, const double* v,
                          const double* depth_field, double depth_scalar,
                          const double* kappa, const double* zfaces, double small_mu,
                          int32_t derivative, double* Ux, double* Uy);
void ora_current_gradients(int64_t Nx, int64_t Ny, int64_t Nk,
                           const double* Ux, const double* Uy, double dx_inv, double dy_inv,
                           double* Uxx, double* Uxy, double* Uyx, double* Uyy);

/* ---- pseudomomentum self-coupling (src/Coupling/pseudomomentum.jl) ---- */
void ora_first_moment_measures(int64_t Nk, int64_t Np, const double* kf, const double* pf, double* kx,
                               double* ky);
void ora_pm_overlap_tables(int64_t Nx, int64_t Ny, int64_t Nk, const double* kappa, int64_t Nz,
                           const double* zf, const double* depth_field, double depth_scalar, double small_mu,
                           double* overlap, double* doverlap);
void ora_pm_doppler_velocity(int64_t Nx, int64_t Ny, int64_t Nk, int64_t Np, const double* N, int32_t per_cell,
                             const double* overlap, const double* doverlap, const double* kx, const double* ky,
                             double* Ux, double* Uy, double* dUx, double* dUy);
void ora_pm_cells(int64_t Nx, int64_t Ny, int64_t Nk, int64_t Np, const double* N, int64_t Nz, const double* zf,
                  const double* depth_field, double depth_scalar, const double* kappa, const double* kx,
                  const double* ky, double small_mu, int32_t cell_average, double* px, double* py);

/* ---- spectral grid and group velocity ---- */
void ora_lower_bounded_faces(int64_t N, const double* centers, double lower, double* faces);
void ora_uniform_periodic_faces(int64_t N, const double* centers, double* faces);
void ora_polar_weights(int64_t Nk, int64_t Np, const double* kf, const double* pf, double* w);
void ora_group_velocity_deep(int64_t Nk, int64_t Np, const double* kf, const double* pf,
                             const double* w, double gravity, double* cg_x, double* cg_y);
void ora_group_velocity_finite(int64_t Nx, int64_t Ny, int64_t Nk, int64_t Np,
                               const double* kappa, const double* phi,
                               const double* depth_field, double depth_scalar, double gravity,
                               double* cg_x, double* cg_y);

/* ---- winds and drag ---- */
double ora_friction_velocity_linear(double U10);
void ora_holland_velocity(const ora_holland* w, double x, double y, double t, double* vx, double* vy);
void ora_storm_center(const ora_holland* w, double t, double* cx, double* cy);
void ora_wind_fields(const ora_model* M, double t, double* U10, double* theta, double* ustar);

/* ---- tendencies, sources, RK3 ---- */
void ora_tendency(const ora_model* M, const double* N, double t, int32_t with_sources, double* G);
void ora_stress_factor(const ora_model* M, const double* N, double t, double* factor);
void ora_rk3_step(const ora_model* M, double* N, double dt, int64_t nsteps, double* t);
/* SpatialAveraging applied once to N (x fastest) with the step's dt (propagation_smoothing.jl:60-199). */
void ora_spatial_averaging(const ora_model* M, double* N, double dt);
/* SpatialAveraging of a slab whose rows sit at rows y_offset + 1 .. y_offset + Ny of a larger grid. */
void ora_spatial_averaging_at(const ora_model* M, double* N, double dt, int64_t y_offset);

/* ---- diagnostics (src/Diagnostics) ---- */
void ora_diagnostics(const ora_model* M, const double* N,
                     double* m0, double* hs, double* krms, double* mean_dir, double* total_action);

int ora_num_threads(void);
void ora_set_num_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
