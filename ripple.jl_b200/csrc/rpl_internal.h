// rpl_internal.h -- handle layout and kernel launchers shared by the librpl.so translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/rpl.h"

namespace rpl {

// Device-side view of the model handed to every stage kernel (by value).
struct StageParams {
    int64_t Nx, Ny, Nk, Np;
    double dx_inv, dy_inv, dk_inv, dp_inv;  // 1/first spacing (wave_current_refraction.jl:200-203)
    double dt;
    double a, b;                            // stage combine: out = max(0, a*N0 + b*max(0, N + dt*G))
    int stage;                              // 1, 2, 3
    int transport;
    int cg_per_cell;                        // 1: cg magnitude per (i,j,m) times direction table
    // tables (FP64)
    const double* kappa;                    // Nk
    const double* phi;                      // Np
    const double* weights;                  // (Nk,Np) spectral cell measures
    const double* cosp;                     // Np
    const double* sinp;                     // Np
    const double* cg_x;                     // (Nk,Np) tables, or direction cosines when cg_per_cell
    const double* cg_y;
    const double* cg_mag;                   // (Nx,Ny,Nk) when cg_per_cell
    const double* Ux;                       // (Nx,Ny,Nk)
    const double* Uy;
    const double* Uxx;
    const double* Uxy;
    const double* Uyx;
    const double* Uyy;
    const double* coef;                     // per (i,j,m) device order: 8 doubles (see rpl_layout.cu)
    const float4* trig32;                   // Np: (cos^2, cos*sin, sin^2, 0) of each direction, FP32
    const float2* cg32;                     // (Nk,Np): the cg_x, cg_y table entries rounded to FP32
    const float2* cs32;                     // Np: (cos, sin) of each direction, FP32
    const float* w32;                       // (Nk,Np): spectral cell measures, FP32
    const float* cell32;                    // (Nx*Ny) records of 8 floats: wind constants (rpl_src32.cuh)
    const float* bin32;                     // Nk records of 8 floats: per-kappa source constants
    const float* lrate;                     // learned source: (cells x Nk*Np) network outputs, bin m + Nk n
    const unsigned int* lflag;              // learned source: per cell, nonzero = use the plain sources
    float lscale;                           // learned source: rate = lscale * sinh(network output)
    int learned;                            // 1: sources from the learned network (with per-cell fallback)
    // sources
    int has_wind, stress_cap, has_diss;
    const double* wind_U10;                 // (Nx,Ny)
    const double* wind_theta;
    const double* wind_ustar;
    const double* stress_factor;            // (Nx,Ny)
    double rho_ratio, beta_max, z_alpha, p_in, alpha0, von_karman, wind_g;
    double C_ds, B_r, ds_p, sigma_power, ds_g;
    float wind_K32, von_karman32, z_alpha32;  // FP32 copies: rho_ratio beta_max / kappa_vk^2, kappa_vk, z_alpha
    unsigned int* err;                      // device error word
    const void* lin_rates;                  // SourceTermSet rates per cell-bin (state layout and type) or null
    int64_t j_lo, j_hi;                     // rows the stage updates (all: 0, Ny); other rows are not written
};

// Arguments of one FP32 tile-kernel stage launch over one model (rpl_tile32.cu): the buffers and the
// FP32 view of StageParams that the tile body reads. Plain words only (copied to shared memory by the
// ensemble kernel).
struct TileArgs {
    const float* Nin;
    const float* N0;
    float* Nout;
    const double* coef;
    const float4* trig32;
    const float2* cg32;
    const float2* cs32;
    const float* cell32;
    const float* bin32;
    unsigned int* err;
    int Nx, Ny, Nk, Np, stage, cg_per_cell, has_wind, stress_cap, has_diss, pad0;
    float dx_inv, dy_inv, dk_inv, dp_inv, dt, a, b;
    float wind_K32, von_karman32, z_alpha32, p_in, ds_p;
    float lscale;
    const float* lrate;
    const unsigned int* lflag;
    int learned, pass_b_quads;   // pass_b_quads: pass B of SRC 0/3 stages with four kappa bins per lane
    const float* lin_rates;  // SourceTermSet rates per cell-bin (state layout) or null
    int j_lo, j_hi;          // rows the stage updates
    float* sxy;              // two-pass refraction stage: x+y flux sums per cell-bin (state layout), or null
    // y-walk pass A (rpl_xyw.cu), or null: FP32 planes of U_x, U_y and the c_g magnitude per (i,j,m),
    // and the per-region upwind ratios
    const float* ux32;
    const float* uy32;
    const float* cgc32;
    const unsigned int* rmax;
};

// Tile shapes (kappa-pair lanes per cell L, tile TX x TY) compiled into the ensemble kernel; every
// shape has TX*TY*L = ENSEMBLE_THREADS threads. The autotuner picks one per size class.
struct TileShape {
    int L, TX, TY;
};
constexpr int ENSEMBLE_THREADS = 512;
constexpr int kNumEnsembleShapes = 9;
constexpr TileShape kEnsembleShapes[kNumEnsembleShapes] = {
    {16, 8, 4}, {16, 4, 8}, {16, 16, 2},   // Nk 17..32
    {8, 8, 8},  {8, 16, 4}, {8, 4, 16},    // Nk 9..16
    {4, 16, 8}, {4, 8, 16}, {4, 32, 4}};   // Nk 4..8

struct Handle {
    rpl_desc desc{};
    std::vector<double> xnodes, ynodes, kappa, kappa_faces, phi, phi_faces, depth_field, weights;
    std::vector<double> spacings;  // Nx widths then Ny heights of the cells (total action)
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int precision = RPL_FP64;
    size_t elem = 8;
    int64_t units = 0, cells = 0;
    // state: N (current), A, B (stage buffers)
    void* N = nullptr;
    void* A = nullptr;
    void* B = nullptr;
    // tables
    double* d_kappa = nullptr;
    double* d_phi = nullptr;
    double* d_cos = nullptr;
    double* d_sin = nullptr;
    double* d_weights = nullptr;
    double* d_cgx = nullptr;
    double* d_cgy = nullptr;
    double* d_cgmag = nullptr;
    double* d_depth = nullptr;
    double* d_coupling = nullptr;  // 8 arrays of (Nx,Ny,Nk): Ux Uy dUxdk dUydk Uxx Uxy Uyx Uyy (caller order,
                                   // filled from d_U when rpl_get_coupling asks)
    double* d_U = nullptr;         // Doppler velocity in device order c*Nk + m: Ux, Uy, dUx/dkappa,
                                   // dUy/dkappa, (Nx*Ny*Nk) each (prescribed or pseudomomentum)
    double* d_coef = nullptr;      // (Nx*Ny*Nk) records of 8 doubles in device order
    float* d_tab32 = nullptr;      // FP32 copies: 4*Np trig, 2*Nk*Np group velocity, 2*Np cos/sin, Nk*Np weights
    float* d_cell32 = nullptr;     // (Nx*Ny) x 8 floats of per-cell wind constants
    float* d_bin32 = nullptr;      // Nk x 8 floats of per-kappa source constants
    float* d_sxy = nullptr;        // FP32 refraction models: x+y flux sums between the two stage passes
    float* d_vel32 = nullptr;      // y-walk pass A: FP32 planes U_x, U_y, c_g per (i,j,m) (3 x Nx*Ny*Nk)
    unsigned int* d_rmax = nullptr;  // y-walk pass A: per region, axis and bin the upwind ratio maxima
    int64_t vel_regions = 0;
    // learned source (rpl_learned.cu)
    rpl_mlp* learned = nullptr;
    void* d_lx = nullptr;          // (rows x nbins) BF16 features, rows = cells rounded up to 128
    float* d_le = nullptr;         // (rows x 4) extras
    float* d_lr = nullptr;         // (rows x nbins) network outputs
    unsigned int* d_lflag = nullptr;  // per cell: inputs outside the bounds -> plain sources
    float* d_lbounds = nullptr;    // lo[nbins + 4], hi[nbins + 4]
    int64_t lrows = 0;
    bool lclamp = false;           // clamp the network outputs to the output bounds
    double lgate = 0.0;            // > 0: a cell whose network rates have |rate| * dt above it uses the plain sources
    unsigned long long* d_lcount = nullptr;  // since rpl_set_learned_source: fallback cell-stages, cell-stages
    bool currents_set = false;
    // prescribed currents: the Q grid and the last currents stay on the device so the coupling can be
    // refreshed (rpl_update_currents*) without allocating
    int64_t q_Nz = 0;
    double q_const = 0.0, q_small_mu = 0.0;
    double* d_qz = nullptr;        // Nz+1 z faces
    double* d_qdepth = nullptr;    // (Nx,Ny) projection depth, depth fields only
    double* d_qW = nullptr;        // constant depth: Q cell weights W then Wd, (Nz, Nk) each, m fastest
    double* d_cur = nullptr;       // u then v, (Nx,Ny,Nz) each, x fastest
    void* d_qcol = nullptr;        // depth field: per-column Q weights (Nz, Nk) per column, when memory allows
    bool q_col_f32 = false;        // d_qcol holds floats (FP32 models)
    bool dU_stale = false;         // the dU/dkappa caches lag the last currents or action (computed on request)
    // PseudomomentumVelocities (rpl_pm.cu)
    bool pm = false;               // the coupling is recomputed from the action before every stage
    bool pm_ready = false;         // d_U holds the velocity of some action
    int64_t pm_cols = 0;           // overlap table pairs: 1 (constant projection depth) or Nx*Ny
    double* d_pm_overlap = nullptr;  // overlap then derivative overlap, pm_cols x Nk x Nk each
    double* d_pm_moments = nullptr;  // kx then ky first-moment measures, (Nk, Np) m fastest
    float* d_pm_overlap32 = nullptr;  // FP32 models: FP32 copy of the overlap table(s)
    float* d_pm_moments32 = nullptr;  // FP32 models: FP32 copy of the moment measures
    const void* pm_last_in = nullptr;  // the action of the last refresh (a state buffer)
    // sources
    rpl_sources src{};
    bool has_sources = false;
    std::vector<double> track_t, track_x, track_y;
    double* d_wind = nullptr;      // 4 arrays of (Nx,Ny): U10 theta ustar factor
    bool wind_field_set = false;
    // propagation_smoothing = SpatialAveraging (rpl_smooth.cu)
    bool smooth = false;
    double smooth_as = 0.5, smooth_an = 0.5, smooth_dt = -1.0;  // dt of the current per-bin stencils
    void* d_smooth = nullptr;      // FP64 cg[Nk], dcg[Nk], cos[Np], sin[Np]; per-bin 3x3 stencils; far flags
    int64_t smooth_bytes = 0;
    // snapshot export (rpl_output.cu)
    cudaStream_t snap_stream = nullptr;  // device-to-host copies of snapshots
    cudaEvent_t snap_ready = nullptr;    // the staging buffer holds the snapshot
    cudaEvent_t snap_done = nullptr;     // the staging buffer has reached the host
    void* d_snap = nullptr;              // staging buffer, caller layout
    int64_t snap_bytes = 0;
    bool snap_pending = false;
    // SourceTermSet terms (rpl_terms.cu)
    int n_terms = 0;
    rpl_source_term terms[RPL_MAX_TERMS] = {};  // field pointers refer to d_terms_fields
    void* d_lin_rates = nullptr;   // per cell-bin rate, state layout and type
    double* d_terms = nullptr;     // per term 3 bin tables (Nk*Np each) then the copied fields
    double2* d_tcol = nullptr;     // per (i,j) column and term the stage's per-cell term values (x0, x1)
    int64_t terms_bytes = 0;
    // diagnostics scratch
    double* d_diag = nullptr;      // 5 (Nx,Ny) fields + block partials
    double* d_spacing = nullptr;   // Nx cell widths then Ny cell heights
    unsigned int* d_err = nullptr;
    unsigned int* h_err = nullptr;  // pinned
    bool force_column_kernel = false;  // RPL_FORCE_COLUMN_KERNEL=1 selects the generic FP32 column kernel
    bool pass_a_tiles = false;         // RPL_PASS_A=tiles: pass A of FP32 refraction from staged tiles
    bool pass_b_pairs = false;         // RPL_PASS_B=pairs: pass B with two kappa bins per lane throughout
    double time = 0.0;
    int64_t iteration = 0;
    int64_t bytes = 0;
};

// Learned-source network internals (rpl_mlp.cu, rpl_learned.cu).
int mlp_nbins(const rpl_mlp* m);
const rpl_mlp_desc& mlp_desc(const rpl_mlp* m);
cudaError_t launch_learned_stage_prep(const Handle& h, const void* Nin, double dt, cudaStream_t s);
void free_learned(Handle* h);

// Pseudomomentum self-coupling (rpl_pm.cu): refresh the velocity and coefficient records from the
// action Nin; write the caller-order coupling arrays and their gradients into d_coupling; release.
// Refresh of the Doppler velocity from the action Nin (with_derivative: dU/dkappa too, else on request).
cudaError_t launch_pm_refresh(Handle& h, const void* Nin, cudaStream_t s, bool with_derivative);
// dU/dkappa of the last refreshed action into d_U arrays 2-3 (zeros before any refresh).
cudaError_t launch_pm_derivative(const Handle& h, cudaStream_t s);
void free_pm(Handle* h);
// Releases the prescribed-currents state of rpl_set_currents (rpl_api.cu).
void free_currents(Handle* h);
// Waits for and releases the snapshot stream, events and staging buffer (rpl_output.cu).
void free_output(Handle* h);
// SpatialAveraging of the state Nin into Nout with the step's dt; release of its tables (rpl_smooth.cu).
// SpatialAveraging Nin -> Nout for rows [j_lo, j_hi) (all: 0, Ny); y_offset: the rows' offset in a larger
// grid (a decomposition slab), at whose row indices the corner weights are computed (else 0).
cudaError_t launch_smooth(Handle& h, const void* Nin, void* Nout, double dt, int64_t j_lo, int64_t j_hi,
                          int64_t y_offset, cudaStream_t s);
void free_smooth(Handle* h);

// SourceTermSet rates of the action Nin into d_lin_rates; release of their buffers (rpl_terms.cu).
cudaError_t launch_terms(const Handle& h, const void* Nin, cudaStream_t s);
void free_terms(Handle* h);

// Sets the thread-local message rpl_last_error() returns (rpl_api.cu).
void set_last_error(const std::string& msg);

// ---- launchers (rpl_setup.cu) ----
cudaError_t launch_q_table(const Handle& h, int64_t Nz, const double* d_zf, double qdepth_const, double small_mu,
                           double* W, double* Wd, cudaStream_t s);
// Per-column Q weights of a depth field into h.d_qcol (FP32 when h.q_col_f32).
cudaError_t launch_q_column_table(const Handle& h, cudaStream_t s);
// Doppler velocity (derivative = 0) or its kappa derivative (1) of the currents d_u, d_v on the Q grid
// of rpl_set_currents, into the caller-order arrays Ux, Uy.
cudaError_t launch_doppler(const Handle& h, const double* d_u, const double* d_v, int derivative, double* Ux,
                           double* Uy, cudaStream_t s);
cudaError_t launch_gradients(const Handle& h, cudaStream_t s);
cudaError_t launch_cg_field(const Handle& h, cudaStream_t s);
cudaError_t launch_wind(const Handle& h, double t, cudaStream_t s);
cudaError_t launch_stress_factor(const Handle& h, const void* Nin, cudaStream_t s, const unsigned int* only = nullptr);
// moments = false: m0 and the total action only (Hs, kappa_rms, mean direction left unwritten).
cudaError_t launch_diagnostics(const Handle& h, const void* Nin, cudaStream_t s, bool moments = true);
cudaError_t launch_scan_nonfinite(const Handle& h, const void* buf, cudaStream_t s);

// ---- layouts (rpl_layout.cu) ----
cudaError_t launch_to_device_layout(const Handle& h, const void* src, int src_dtype, void* dst, int dst_dtype,
                                    int64_t n0, int64_t nc, int64_t m0, int64_t mc, cudaStream_t s);
cudaError_t launch_from_device_layout(const Handle& h, const void* src, int src_dtype, void* dst, int dst_dtype,
                                      int64_t n0, int64_t nc, int64_t m0, int64_t mc, cudaStream_t s);
cudaError_t launch_coef(const Handle& h, cudaStream_t s);
// Coefficient fields 0-5 (Ux, Uy and the periodic gradients) from the device-order velocity d_U.
cudaError_t launch_coef_from_U(const Handle& h, cudaStream_t s);
// d_U -> the caller-order coupling arrays 0-3 of d_coupling, then their gradients (arrays 4-7).
cudaError_t launch_export_U(const Handle& h, cudaStream_t s);

// ---- y-walk pass A of the FP32 refraction stage (rpl_xyw.cu) ----
bool xyw_supported(const Handle& h);              // 32-bit offsets within a direction slice
int xyw_lanes(int64_t Nk);                        // lanes per cell (four kappa bins each)
int64_t xyw_regions(const Handle& h);             // regions of the upwind ratio table
// FP32 velocity planes and upwind ratios from d_coef (after every coefficient refresh; no-op without
// d_vel32).
cudaError_t launch_vel32(const Handle& h, cudaStream_t s);
cudaError_t launch_xyw(const TileArgs& a, cudaStream_t s);   // writes a.sxy for rows [j_lo, j_hi)
// The same x/y pass for intrinsic transport (no currents): S = fx + fy into a.sxy.
cudaError_t launch_xy_intrinsic(const TileArgs& a, cudaStream_t s);
// The whole stage of intrinsic transport (no currents) without sources (src 0) or with the SourceTermSet
// rates (src 3, the tile body's SRC).
cudaError_t launch_xyi(const TileArgs& a, int src, cudaStream_t s);

// ---- FP32 tiled stage kernel (rpl_tile32.cu) ----
bool tile32_supported(const Handle& h);
cudaError_t launch_tile32(const Handle& h, const StageParams& p, const void* Nin, const void* N0, void* Nout,
                          cudaStream_t s);
int tile_lanes(int64_t Nk);                       // L used for Nk: 4, 8 or 16
size_t tile_smem_bytes(int L, int TX, int TY);
TileArgs make_tile_args(const Handle& h, const StageParams& p, const void* Nin, const void* N0, void* Nout);
cudaError_t prepare_ensemble_kernels();           // shared-memory attribute, once per device
size_t ensemble_smem_bytes();
int ensemble_grid(bool refract, int device);      // resident CTAs: SMs x CTAs per SM
cudaError_t launch_ensemble_stage(bool refract, const TileArgs* d_args, const int4* d_items, int nitems,
                                  unsigned int* d_counter, int grid, cudaStream_t s);

// ---- stage kernels (rpl_stage.cu) ----
StageParams make_params(const Handle& h, double dt, int stage);
cudaError_t launch_stage(const Handle& h, const StageParams& p, const void* Nin, const void* N0,
                         void* Nout, cudaStream_t s);
cudaError_t launch_tendency(const Handle& h, const StageParams& p, const void* Nin, double* G,
                            cudaStream_t s);

}  // namespace rpl
