// rpl_api.cu -- the extern "C" entry points of librpl.so (declared in include/rpl.h): argument
// validation with the reference's error rules, device buffer ownership, the SSP-RK3 driver.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "rpl_internal.h"

using rpl::Handle;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    const int code = (e == cudaErrorMemoryAllocation) ? RPL_ERR_OOM : RPL_ERR_CUDA;
    return fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define RPL_CUDA(call)                                      \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

bool finite_all(const double* p, int64_t n) {
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

// Validation rules of src/CoordinateGrids/spectral_grids.jl:176-214.
std::string check_centers(const char* name, const double* c, int64_t n, bool positive) {
    for (int64_t i = 0; i + 1 < n; ++i)
        if (!(c[i + 1] > c[i])) return std::string(name) + " centers must be strictly increasing";
    if (positive)
        for (int64_t i = 0; i < n; ++i)
            if (!(c[i] > 0.0)) return std::string(name) + " centers must be positive";
    return "";
}

std::string check_faces(const char* name, const double* c, const double* f, int64_t n) {
    for (int64_t i = 0; i < n; ++i)
        if (!(f[i + 1] > f[i])) return std::string(name) + " faces must be strictly increasing";
    for (int64_t i = 0; i < n; ++i)
        if (!(f[i] <= c[i] && c[i] <= f[i + 1]))
            return std::string(name) + " center " + std::to_string(i + 1) + " must lie inside its cell faces";
    return "";
}

template <typename T>
cudaError_t dalloc(Handle* h, T** p, size_t count) {
    const size_t bytes = count * sizeof(T);
    cudaError_t e = cudaMalloc((void**)p, bytes ? bytes : 8);
    if (e == cudaSuccess) h->bytes += (int64_t)bytes;
    return e;
}

void free_all(Handle* h) {
    rpl::free_output(h);
    rpl::free_terms(h);
    rpl::free_smooth(h);
    rpl::free_learned(h);
    rpl::free_pm(h);
    rpl::free_currents(h);
    void* ptrs[] = {h->N, h->A, h->B, h->d_kappa, h->d_phi, h->d_cos, h->d_sin, h->d_weights, h->d_cgx,
                    h->d_cgy, h->d_cgmag, h->d_depth, h->d_coupling, h->d_wind, h->d_diag, h->d_err,
                    h->d_coef, h->d_tab32, h->d_cell32, h->d_bin32, h->d_U, h->d_spacing, h->d_sxy,
                    h->d_vel32, h->d_rmax};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (h->h_err) cudaFreeHost(h->h_err);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
}

}  // namespace

// Releases the prescribed-currents state (Q grid, weight tables, the device copy of u and v).
void rpl::free_currents(Handle* h) {
    const int64_t P = h->cells, Nk = h->desc.Nk;
    if (h->d_qz) h->bytes -= (h->q_Nz + 1) * 8;
    if (h->d_qdepth) h->bytes -= P * 8;
    if (h->d_qW) h->bytes -= 2 * h->q_Nz * Nk * 8;
    if (h->d_cur) h->bytes -= 2 * P * h->q_Nz * 8;
    if (h->d_qcol) h->bytes -= P * h->q_Nz * Nk * (h->q_col_f32 ? 4 : 8);
    for (double* p : {h->d_qz, h->d_qdepth, h->d_qW, h->d_cur})
        if (p) cudaFree(p);
    if (h->d_qcol) cudaFree(h->d_qcol);
    h->d_qz = h->d_qdepth = h->d_qW = h->d_cur = nullptr;
    h->d_qcol = nullptr;
    h->q_Nz = 0;
    h->dU_stale = false;
}

namespace {

// Doppler velocity of the currents (u, v device pointers, (Nx,Ny,Nz) x fastest) on the stored Q grid,
// then its gradients and the coefficient records, in stream order. The stage kernels do not read
// dU/dkappa; it is recomputed from d_cur when rpl_get_coupling asks for it.
cudaError_t refresh_currents(Handle* h, const double* u, const double* v, cudaStream_t s) {
    const int64_t c3 = h->cells * h->desc.Nk;
    cudaError_t e = rpl::launch_doppler(*h, u, v, 0, h->d_U, h->d_U + c3, s);
    if (e == cudaSuccess) e = rpl::launch_coef_from_U(*h, s);
    if (e == cudaSuccess) h->dU_stale = true;
    return e;
}

int check_handle(rpl_handle* hh) {
    if (!hh) return fail(RPL_ERR_ARGUMENT, "null handle");
    Handle* h = reinterpret_cast<Handle*>(hh);
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    return RPL_OK;
}

// Reads and clears the kernels' error word; call after the stream drained.
int check_error_word(Handle* h) {
    RPL_CUDA(cudaMemcpyAsync(h->h_err, h->d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, h->stream));
    RPL_CUDA(cudaStreamSynchronize(h->stream));
    const unsigned w = *h->h_err;
    if (w) {
        RPL_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(unsigned int), h->stream));
        RPL_CUDA(cudaStreamSynchronize(h->stream));
        if (w & 2u) return fail(RPL_ERR_NONFINITE, "non-finite values in the action passed in");
        if (w & 4u) return fail(RPL_ERR_DEVICE, "a tensor-core GEMM of the learned source gave up waiting");
        return fail(RPL_ERR_DEVICE, "a stage kernel produced non-finite wave action (time step too large?)");
    }
    return RPL_OK;
}

// One RK3 stage over rows [j_lo, j_hi): the stage's preparation kernels (wind, stress cap or learned
// rows, pseudomomentum refresh, SourceTermSet rates; all column-local) when `prepare`, the stage kernel,
// and when `finish` what completes the stage (after stage 3: SpatialAveraging and the clock).
int launch_stage_rows(Handle* h, double dt, int stage, int64_t j_lo, int64_t j_hi, bool prepare, bool finish,
                      bool defer_smooth = false) {
    cudaStream_t s = h->stream;
    const bool sources = h->has_sources && (h->src.wind_kind != RPL_WIND_NONE);
    const void* Nin = stage == 1 ? h->N : (stage == 2 ? h->A : h->B);
    // with SpatialAveraging, stage 3 writes into A (free by then) and the averaging writes A -> N
    void* Nout = stage == 1 ? h->A : (stage == 2 ? h->B : (h->smooth ? h->A : h->N));
    if (prepare) {
        if (sources) {
            if (stage == 1) RPL_CUDA(rpl::launch_wind(*h, h->time, s));
            if (h->learned) RPL_CUDA(rpl::launch_learned_stage_prep(*h, Nin, dt, s));
            else if (h->src.stress_cap) RPL_CUDA(rpl::launch_stress_factor(*h, Nin, s));
        }
        if (h->pm) RPL_CUDA(rpl::launch_pm_refresh(*h, Nin, s, false));
        if (h->n_terms) RPL_CUDA(rpl::launch_terms(*h, Nin, s));
    }
    if (j_hi > j_lo) {
        rpl::StageParams p = rpl::make_params(*h, dt, stage);
        p.j_lo = j_lo;
        p.j_hi = j_hi;
        RPL_CUDA(rpl::launch_stage(*h, p, Nin, h->N, Nout, s));
    }
    if (finish && stage == 3) {
        if (h->smooth && !defer_smooth)
            RPL_CUDA(rpl::launch_smooth(*h, h->A, h->N, dt, 0, h->desc.Ny, 0, s));  // time_step.jl:168
        h->time += dt;
        h->iteration += 1;
    }
    return RPL_OK;
}

int launch_step(Handle* h, double dt, int stage_only) {
    const int first = stage_only ? stage_only : 1, last = stage_only ? stage_only : 3;
    for (int stage = first; stage <= last; ++stage) {
        const int st = launch_stage_rows(h, dt, stage, 0, h->desc.Ny, true, true);
        if (st) return st;
    }
    return RPL_OK;
}

int check_step_args(Handle* h, double dt) {
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(RPL_ERR_DT, "time step must be positive");
    if (h->desc.transport == RPL_TRANSPORT_REFRACTION && !h->currents_set)
        return fail(RPL_ERR_STATE, "refraction transport needs rpl_set_currents before stepping");
    if (h->has_sources && h->src.wind_kind == RPL_WIND_FIELD && !h->wind_field_set)
        return fail(RPL_ERR_STATE, "RPL_WIND_FIELD sources need rpl_set_wind_field before stepping");
    return RPL_OK;
}

}  // namespace

void rpl::set_last_error(const std::string& msg) { g_last_error = msg; }

extern "C" {

const char* rpl_last_error(void) { return g_last_error.c_str(); }

int rpl_abi_version(void) { return RPL_ABI_VERSION; }

int rpl_create(const rpl_desc* d, rpl_handle** out) {
    g_last_error.clear();
    if (!d || !out) return fail(RPL_ERR_ARGUMENT, "null descriptor or output pointer");
    *out = nullptr;
    if (d->abi_version != RPL_ABI_VERSION) return fail(RPL_ERR_ARGUMENT, "descriptor abi_version mismatch");
    if (d->precision != RPL_FP64 && d->precision != RPL_FP32) return fail(RPL_ERR_ARGUMENT, "unknown precision");
    if (d->transport < RPL_TRANSPORT_NONE || d->transport > RPL_TRANSPORT_INTRINSIC)
        return fail(RPL_ERR_ARGUMENT, "unknown transport");
    if (d->Nx < 1 || d->Ny < 1 || d->Nk < 1 || d->Np < 1)
        return fail(RPL_ERR_ARGUMENT, "grid sizes must be positive");
    if (!d->xnodes || !d->ynodes || !d->kappa || !d->kappa_faces || !d->phi || !d->phi_faces)
        return fail(RPL_ERR_ARGUMENT, "null coordinate array");
    if (!(d->dx > 0.0) || !(d->dy > 0.0) || !std::isfinite(d->dx) || !std::isfinite(d->dy))
        return fail(RPL_ERR_ARGUMENT, "grid spacings must be positive and finite");
    if (!(d->gravity > 0.0)) return fail(RPL_ERR_ARGUMENT, "gravity must be positive");
    if (!finite_all(d->kappa, d->Nk) || !finite_all(d->kappa_faces, d->Nk + 1) || !finite_all(d->phi, d->Np) ||
        !finite_all(d->phi_faces, d->Np + 1) || !finite_all(d->xnodes, d->Nx) || !finite_all(d->ynodes, d->Ny))
        return fail(RPL_ERR_NONFINITE, "non-finite grid coordinates");
    std::string msg = check_centers("κ", d->kappa, d->Nk, true);
    if (msg.empty()) msg = check_centers("φ", d->phi, d->Np, false);
    if (msg.empty()) msg = check_faces("κ", d->kappa, d->kappa_faces, d->Nk);
    if (msg.empty()) msg = check_faces("φ", d->phi, d->phi_faces, d->Np);
    if (msg.empty() && d->kappa_faces[0] < 0.0) msg = "κ faces must be >= 0";
    if (!msg.empty()) return fail(RPL_ERR_ARGUMENT, msg);
    if ((d->xspacings == nullptr) != (d->yspacings == nullptr))
        return fail(RPL_ERR_ARGUMENT, "xspacings and yspacings must both be given or both be NULL");
    if (d->xspacings) {
        for (int64_t i = 0; i < d->Nx; ++i)
            if (!(d->xspacings[i] > 0.0) || !std::isfinite(d->xspacings[i]))
                return fail(RPL_ERR_ARGUMENT, "cell widths must be positive and finite");
        for (int64_t j = 0; j < d->Ny; ++j)
            if (!(d->yspacings[j] > 0.0) || !std::isfinite(d->yspacings[j]))
                return fail(RPL_ERR_ARGUMENT, "cell heights must be positive and finite");
    }
    if (d->transport != RPL_TRANSPORT_NONE) {
        if (!d->periodic_x || !d->periodic_y)
            return fail(RPL_ERR_UNSUPPORTED,
                        "the fused transport kernels need Periodic x and y (bounded topologies use the "
                        "reference's per-bin Oceananigans path, which this library does not provide)");
        if (d->Nx < 3 || d->Ny < 3) return fail(RPL_ERR_ARGUMENT, "WENO5 transport needs Nx, Ny >= 3");
        if (d->transport == RPL_TRANSPORT_REFRACTION && d->Np < 3)
            return fail(RPL_ERR_ARGUMENT, "spectral refraction needs at least 3 direction bins");
    }
    if (d->depth_kind == RPL_DEPTH_CONSTANT) {
        if (!(d->depth_constant > 0.0) || !std::isfinite(d->depth_constant))
            return fail(RPL_ERR_ARGUMENT, "depth must be positive");
    } else if (d->depth_kind == RPL_DEPTH_FIELD) {
        if (!d->depth_field) return fail(RPL_ERR_ARGUMENT, "null depth field");
        for (int64_t c = 0; c < d->Nx * d->Ny; ++c)
            if (!(d->depth_field[c] > 0.0) || !std::isfinite(d->depth_field[c]))
                return fail(RPL_ERR_ARGUMENT, "depth values must be positive");
    } else if (d->depth_kind != RPL_DEPTH_INFINITE) {
        return fail(RPL_ERR_ARGUMENT, "unknown depth kind");
    }

    const int64_t units = d->Nx * d->Ny * d->Nk * d->Np;
    const size_t elem = d->precision == RPL_FP64 ? 8 : 4;
    const int64_t c3 = d->Nx * d->Ny * d->Nk, P = d->Nx * d->Ny, nb = d->Nk * d->Np;
    int64_t need = 3 * units * (int64_t)elem + 16 * c3 * 8 + (d->depth_kind == RPL_DEPTH_FIELD ? (c3 + P) * 8 : 0) +
                   (4 * P + 2 * (d->Nx + d->Ny)) * 8 + 6 * P * 8 + 8 * nb * 8 +
                   (d->precision == RPL_FP32 && d->transport == RPL_TRANSPORT_REFRACTION ? units * 4 + 3 * c3 * 4 : 0) +
                   (d->precision == RPL_FP32 && d->transport == RPL_TRANSPORT_INTRINSIC ? c3 * 4 + units * 4 : 0);
    if (d->memory_limit_bytes > 0 && need > d->memory_limit_bytes)
        return fail(RPL_ERR_OOM, "model needs " + std::to_string(need) + " device bytes, above the memory limit of " +
                                     std::to_string(d->memory_limit_bytes));

    Handle* h = new (std::nothrow) Handle();
    if (!h) return fail(RPL_ERR_OOM, "host allocation failed");
    h->desc = *d;
    {
        const char* env = std::getenv("RPL_FORCE_COLUMN_KERNEL");
        h->force_column_kernel = env && env[0] == '1';
        const char* pa = std::getenv("RPL_PASS_A");
        h->pass_a_tiles = pa && std::string(pa) == "tiles";
        const char* pb = std::getenv("RPL_PASS_B");
        h->pass_b_pairs = pb && std::string(pb) == "pairs";
    }
    h->device = d->device;
    h->precision = d->precision;
    h->elem = elem;
    h->units = units;
    h->cells = P;
    h->xnodes.assign(d->xnodes, d->xnodes + d->Nx);
    h->ynodes.assign(d->ynodes, d->ynodes + d->Ny);
    h->kappa.assign(d->kappa, d->kappa + d->Nk);
    h->kappa_faces.assign(d->kappa_faces, d->kappa_faces + d->Nk + 1);
    h->phi.assign(d->phi, d->phi + d->Np);
    h->phi_faces.assign(d->phi_faces, d->phi_faces + d->Np + 1);
    h->spacings.resize(d->Nx + d->Ny);
    for (int64_t i = 0; i < d->Nx; ++i) h->spacings[i] = d->xspacings ? d->xspacings[i] : d->dx;
    for (int64_t j = 0; j < d->Ny; ++j) h->spacings[d->Nx + j] = d->yspacings ? d->yspacings[j] : d->dy;
    h->desc.xspacings = h->spacings.data();
    h->desc.yspacings = h->spacings.data() + d->Nx;
    if (d->depth_kind == RPL_DEPTH_FIELD) h->depth_field.assign(d->depth_field, d->depth_field + P);
    h->desc.xnodes = h->xnodes.data();
    h->desc.ynodes = h->ynodes.data();
    h->desc.kappa = h->kappa.data();
    h->desc.kappa_faces = h->kappa_faces.data();
    h->desc.phi = h->phi.data();
    h->desc.phi_faces = h->phi_faces.data();
    h->desc.depth_field = h->depth_field.empty() ? nullptr : h->depth_field.data();

    // Host tables (FP64): spectral weights and moment measures (polar_wavevector_grid.jl:44-47,73-115),
    // direction cosines, group velocities (transport.jl:53-139).
    const double g = d->gravity;
    std::vector<double> tabs(4 * nb), cosp(d->Np), sinp(d->Np), cgx(nb), cgy(nb);
    for (int64_t n = 0; n < d->Np; ++n) {
        cosp[n] = std::cos(h->phi[n]);
        sinp[n] = std::sin(h->phi[n]);
        for (int64_t m = 0; m < d->Nk; ++m) {
            const double k1 = h->kappa_faces[m], k2 = h->kappa_faces[m + 1];
            const double p1 = h->phi_faces[n], p2 = h->phi_faces[n + 1];
            const int64_t b = m + d->Nk * n;
            tabs[b] = ((k2 * k2 - k1 * k1) / 2.0) * (p2 - p1);
            const double r1 = (k2 * k2 * k2 - k1 * k1 * k1) / 3.0;
            tabs[nb + b] = r1 * (std::sin(p2) - std::sin(p1));
            tabs[2 * nb + b] = r1 * (std::cos(p1) - std::cos(p2));
            const double r2 = (std::pow(k2, 4.0) - std::pow(k1, 4.0)) / 4.0;
            const double dp = p2 - p1, s2 = std::sin(2.0 * p2) - std::sin(2.0 * p1);
            tabs[3 * nb + b] = r2 * (dp / 2.0 + s2 / 4.0) + r2 * (dp / 2.0 - s2 / 4.0);
            const double kap = h->kappa[m];
            const double kx = kap * std::cos(h->phi[n]), ky = kap * std::sin(h->phi[n]);
            if (d->depth_kind == RPL_DEPTH_INFINITE) {
                const double radial = (std::pow(k2, 1.5) - std::pow(k1, 1.5)) / 1.5;
                const double scale = std::sqrt(g) / (2.0 * tabs[b]);
                cgx[b] = scale * radial * (std::sin(p2) - std::sin(p1));
                cgy[b] = scale * radial * (std::cos(p1) - std::cos(p2));
            } else if (d->depth_kind == RPL_DEPTH_CONSTANT) {
                const double mu = kap * d->depth_constant;
                const double cp = std::sqrt(g * std::tanh(mu) / kap);
                const double gf = (1.0 + 2.0 * mu / std::sinh(2.0 * mu)) / 2.0;
                const double cg = gf * cp;
                cgx[b] = cg * kx / kap;
                cgy[b] = cg * ky / kap;
            } else {  // direction factors; the magnitude comes per (i,j,m) from the device
                cgx[b] = kx / kap;
                cgy[b] = ky / kap;
            }
        }
    }

    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) {
        delete h;
        return cuda_fail(e, "cudaSetDevice");
    }
#define TRY(call)                          \
    do {                                   \
        cudaError_t e_ = (call);           \
        if (e_ != cudaSuccess) {           \
            free_all(h);                   \
            delete h;                      \
            return cuda_fail(e_, #call);   \
        }                                  \
    } while (0)
    TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
    TRY(cudaMalloc(&h->N, units * elem));
    TRY(cudaMalloc(&h->A, units * elem));
    TRY(cudaMalloc(&h->B, units * elem));
    h->bytes += 3 * units * (int64_t)elem;
    TRY(dalloc(h, &h->d_kappa, d->Nk));
    TRY(dalloc(h, &h->d_phi, d->Np));
    TRY(dalloc(h, &h->d_cos, d->Np));
    TRY(dalloc(h, &h->d_sin, d->Np));
    TRY(dalloc(h, &h->d_weights, 4 * nb));
    TRY(dalloc(h, &h->d_cgx, nb));
    TRY(dalloc(h, &h->d_cgy, nb));
    TRY(dalloc(h, &h->d_wind, 4 * P + d->Nx + d->Ny));
    TRY(dalloc(h, &h->d_diag, 5 * P + 8));
    TRY(dalloc(h, &h->d_spacing, d->Nx + d->Ny));
    TRY(dalloc(h, &h->d_err, 1));
    TRY(cudaMallocHost(&h->h_err, sizeof(unsigned int)));
    cudaStream_t s = h->stream;
    TRY(cudaMemsetAsync(h->N, 0, units * elem, s));
    TRY(cudaMemsetAsync(h->d_err, 0, sizeof(unsigned int), s));
    TRY(cudaMemcpyAsync(h->d_kappa, h->kappa.data(), d->Nk * 8, cudaMemcpyHostToDevice, s));
    TRY(cudaMemcpyAsync(h->d_phi, h->phi.data(), d->Np * 8, cudaMemcpyHostToDevice, s));
    TRY(cudaMemcpyAsync(h->d_cos, cosp.data(), d->Np * 8, cudaMemcpyHostToDevice, s));
    TRY(cudaMemcpyAsync(h->d_sin, sinp.data(), d->Np * 8, cudaMemcpyHostToDevice, s));
    TRY(cudaMemcpyAsync(h->d_weights, tabs.data(), 4 * nb * 8, cudaMemcpyHostToDevice, s));
    TRY(cudaMemcpyAsync(h->d_cgx, cgx.data(), nb * 8, cudaMemcpyHostToDevice, s));
    TRY(cudaMemcpyAsync(h->d_cgy, cgy.data(), nb * 8, cudaMemcpyHostToDevice, s));
    TRY(cudaMemcpyAsync(h->d_spacing, h->spacings.data(), (d->Nx + d->Ny) * 8, cudaMemcpyHostToDevice, s));
    TRY(cudaMemsetAsync(h->d_wind, 0, 4 * P * 8, s));
    TRY(cudaMemcpyAsync(h->d_wind + 4 * P, h->xnodes.data(), d->Nx * 8, cudaMemcpyHostToDevice, s));
    TRY(cudaMemcpyAsync(h->d_wind + 4 * P + d->Nx, h->ynodes.data(), d->Ny * 8, cudaMemcpyHostToDevice, s));
    if (d->depth_kind == RPL_DEPTH_FIELD) {
        TRY(dalloc(h, &h->d_depth, P));
        TRY(dalloc(h, &h->d_cgmag, c3));
        TRY(cudaMemcpyAsync(h->d_depth, h->depth_field.data(), P * 8, cudaMemcpyHostToDevice, s));
        TRY(rpl::launch_cg_field(*h, s));
    }
    TRY(dalloc(h, &h->d_coef, 8 * c3));
    TRY(dalloc(h, &h->d_cell32, 8 * P));
    TRY(dalloc(h, &h->d_bin32, 8 * d->Nk));
    if (d->transport == RPL_TRANSPORT_REFRACTION && rpl::tile32_supported(*h) && !h->force_column_kernel)
        TRY(dalloc(h, &h->d_sxy, units));  // the two-pass refraction stage of FP32 models
    const bool intrinsic32 = d->transport == RPL_TRANSPORT_INTRINSIC && rpl::tile32_supported(*h) &&
                             !h->force_column_kernel;
    if ((h->d_sxy || intrinsic32) && rpl::xyw_supported(*h) && !h->pass_a_tiles) {
        // the y-walk x/y kernels: FP32 velocity planes (intrinsic: c_g only) and upwind ratios
        const bool refract_planes = h->d_sxy != nullptr;
        TRY(dalloc(h, &h->d_vel32, (refract_planes ? 3 : 1) * c3));
        // intrinsic stages with the bundle or learned sources run the x/y pass, then the sources: S
        if (!refract_planes) TRY(dalloc(h, &h->d_sxy, units));
        h->vel_regions = rpl::xyw_regions(*h);
        TRY(dalloc(h, &h->d_rmax, 2 * h->vel_regions * d->Nk));
    }
    TRY(rpl::launch_coef(*h, s));
    {
        std::vector<float> tab32(6 * d->Np + 3 * nb);
        for (int64_t n = 0; n < d->Np; ++n) {
            const float c = (float)cosp[n], sn = (float)sinp[n];
            tab32[4 * n] = c * c;
            tab32[4 * n + 1] = c * sn;
            tab32[4 * n + 2] = sn * sn;
            tab32[4 * n + 3] = 0.0f;
        }
        for (int64_t b = 0; b < nb; ++b) {
            tab32[4 * d->Np + 2 * b] = (float)cgx[b];
            tab32[4 * d->Np + 2 * b + 1] = (float)cgy[b];
            tab32[6 * d->Np + 2 * nb + b] = (float)tabs[b];
        }
        for (int64_t n = 0; n < d->Np; ++n) {
            tab32[4 * d->Np + 2 * nb + 2 * n] = (float)cosp[n];
            tab32[4 * d->Np + 2 * nb + 2 * n + 1] = (float)sinp[n];
        }
        TRY(dalloc(h, &h->d_tab32, tab32.size()));
        TRY(cudaMemcpyAsync(h->d_tab32, tab32.data(), tab32.size() * 4, cudaMemcpyHostToDevice, s));
        TRY(cudaStreamSynchronize(s));
    }
    TRY(cudaStreamSynchronize(s));
#undef TRY
    *out = reinterpret_cast<rpl_handle*>(h);
    return RPL_OK;
}

int rpl_destroy(rpl_handle* hh) {
    if (!hh) return RPL_OK;
    Handle* h = reinterpret_cast<Handle*>(hh);
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return RPL_OK;
}

int rpl_set_currents(rpl_handle* hh, int64_t Nz, const double* z_faces, int32_t q_depth_kind,
                     double q_depth_constant, const double* q_depth_field, const double* u, const double* v,
                     double small_mu) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    const rpl_desc& d = h->desc;
    if (Nz < 1 || !z_faces || !u || !v) return fail(RPL_ERR_ARGUMENT, "currents need Nz >= 1, z faces, u and v");
    if (!(small_mu >= 0.0)) return fail(RPL_ERR_ARGUMENT, "small_mu must be non-negative");
    for (int64_t k = 0; k < Nz; ++k)
        if (!(z_faces[k + 1] > z_faces[k])) return fail(RPL_ERR_ARGUMENT, "z faces must be strictly increasing");
    const int64_t P = d.Nx * d.Ny, n3 = P * Nz;
    if (!finite_all(z_faces, Nz + 1) || !finite_all(u, n3) || !finite_all(v, n3))
        return fail(RPL_ERR_NONFINITE, "non-finite currents or z faces");
    if (q_depth_kind == RPL_DEPTH_CONSTANT) {
        if (!(q_depth_constant > 0.0)) return fail(RPL_ERR_ARGUMENT, "depth must be positive");
    } else if (q_depth_kind == RPL_DEPTH_FIELD) {
        if (!q_depth_field) return fail(RPL_ERR_ARGUMENT, "null Q depth field");
        for (int64_t c = 0; c < P; ++c)
            if (!(q_depth_field[c] > 0.0)) return fail(RPL_ERR_ARGUMENT, "depth values must be positive");
    } else {
        return fail(RPL_ERR_ARGUMENT, "Q-transform depth must be constant or a field");
    }
    const int64_t c3 = P * d.Nk;
    const bool field = q_depth_kind == RPL_DEPTH_FIELD;
    const int64_t extra = (h->d_coupling ? 0 : 8 * c3 * 8) + (h->d_U ? 0 : 4 * c3 * 8) + (Nz + 1) * 8 +
                          (field ? P * 8 : 2 * Nz * d.Nk * 8) + 2 * n3 * 8;
    cudaStream_t s = h->stream;
    RPL_CUDA(cudaStreamSynchronize(s));
    rpl::free_pm(h);  // prescribed currents replace a pseudomomentum coupling
    rpl::free_currents(h);
    if (d.memory_limit_bytes > 0 && h->bytes + extra > d.memory_limit_bytes)
        return fail(RPL_ERR_OOM, "currents need " + std::to_string(extra) + " more device bytes, above the memory limit");
    h->currents_set = false;
    if (!h->d_coupling) RPL_CUDA(dalloc(h, &h->d_coupling, 8 * c3));
    if (!h->d_U) RPL_CUDA(dalloc(h, &h->d_U, 4 * c3));
    cudaError_t e = dalloc(h, &h->d_qz, Nz + 1);
    if (e == cudaSuccess && field) e = dalloc(h, &h->d_qdepth, P);
    if (e == cudaSuccess && !field) e = dalloc(h, &h->d_qW, 2 * Nz * d.Nk);
    if (e == cudaSuccess) e = dalloc(h, &h->d_cur, 2 * n3);
    if (e != cudaSuccess) {
        rpl::free_currents(h);
        cudaGetLastError();
        return fail(RPL_ERR_OOM, "currents: device allocation failed");
    }
    h->q_Nz = Nz;
    h->q_const = field ? 0.0 : q_depth_constant;
    h->q_small_mu = small_mu;
    e = cudaMemcpyAsync(h->d_cur, u, n3 * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_cur + n3, v, n3 * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_qz, z_faces, (Nz + 1) * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && field) e = cudaMemcpyAsync(h->d_qdepth, q_depth_field, P * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !field)
        e = rpl::launch_q_table(*h, Nz, h->d_qz, q_depth_constant, small_mu, h->d_qW, h->d_qW + Nz * d.Nk, s);
    if (e == cudaSuccess && field) {
        // per-column Q weights (FP32 for FP32 models): refreshes then stream them instead of evaluating
        // the Q kernel's exponentials again; skipped when they would exceed the memory limit or fail to
        // allocate
        h->q_col_f32 = h->precision == RPL_FP32;
        const int64_t tb = P * Nz * d.Nk * (h->q_col_f32 ? 4 : 8);
        if (!(d.memory_limit_bytes > 0 && h->bytes + tb > d.memory_limit_bytes) &&
            cudaMalloc(&h->d_qcol, tb) == cudaSuccess) {
            h->bytes += tb;
            e = rpl::launch_q_column_table(*h, s);
        } else {
            cudaGetLastError();
            h->d_qcol = nullptr;
        }
    }
    if (e == cudaSuccess) {
        h->currents_set = true;  // the coefficient records read the coupling from here on
        e = refresh_currents(h, h->d_cur, h->d_cur + n3, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        h->currents_set = false;
        rpl::free_currents(h);
        return cuda_fail(e, "rpl_set_currents");
    }
    return RPL_OK;
}

int rpl_update_currents(rpl_handle* hh, const double* u, const double* v) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!u || !v) return fail(RPL_ERR_ARGUMENT, "null u or v");
    if (!h->d_cur || h->pm) return fail(RPL_ERR_STATE, "rpl_update_currents needs rpl_set_currents first");
    const int64_t n3 = h->cells * h->q_Nz;
    cudaStream_t s = h->stream;
    RPL_CUDA(cudaMemcpyAsync(h->d_cur, u, n3 * 8, cudaMemcpyHostToDevice, s));
    RPL_CUDA(cudaMemcpyAsync(h->d_cur + n3, v, n3 * 8, cudaMemcpyHostToDevice, s));
    RPL_CUDA(refresh_currents(h, h->d_cur, h->d_cur + n3, s));
    return RPL_OK;
}

int rpl_update_currents_device(rpl_handle* hh, const double* u, const double* v) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!u || !v) return fail(RPL_ERR_ARGUMENT, "null u or v");
    if (!h->d_cur || h->pm) return fail(RPL_ERR_STATE, "rpl_update_currents_device needs rpl_set_currents first");
    // kept for the dU/dkappa caches that rpl_get_coupling computes on request
    const int64_t n3 = h->cells * h->q_Nz;
    RPL_CUDA(cudaMemcpyAsync(h->d_cur, u, n3 * 8, cudaMemcpyDeviceToDevice, h->stream));
    RPL_CUDA(cudaMemcpyAsync(h->d_cur + n3, v, n3 * 8, cudaMemcpyDeviceToDevice, h->stream));
    RPL_CUDA(refresh_currents(h, h->d_cur, h->d_cur + n3, h->stream));
    return RPL_OK;
}

int rpl_get_coupling(rpl_handle* hh, double* Ux, double* Uy, double* dUxdk, double* dUydk, double* Uxx,
                     double* Uxy, double* Uyx, double* Uyy) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h->currents_set) return fail(RPL_ERR_STATE, "no currents set");
    const int64_t c3 = h->desc.Nx * h->desc.Ny * h->desc.Nk;
    if (h->pm && h->dU_stale) {
        RPL_CUDA(rpl::launch_pm_derivative(*h, h->stream));
        h->dU_stale = false;
    }
    if (!h->pm && h->dU_stale) {
        const int64_t n3 = h->cells * h->q_Nz;
        RPL_CUDA(rpl::launch_doppler(*h, h->d_cur, h->d_cur + n3, 1, h->d_U + 2 * c3, h->d_U + 3 * c3, h->stream));
        h->dU_stale = false;
    }
    RPL_CUDA(rpl::launch_export_U(*h, h->stream));
    double* outs[8] = {Ux, Uy, dUxdk, dUydk, Uxx, Uxy, Uyx, Uyy};
    for (int k = 0; k < 8; ++k)
        if (outs[k])
            RPL_CUDA(cudaMemcpyAsync(outs[k], h->d_coupling + k * c3, c3 * 8, cudaMemcpyDeviceToHost, h->stream));
    RPL_CUDA(cudaStreamSynchronize(h->stream));
    return RPL_OK;
}

int rpl_set_sources(rpl_handle* hh, const rpl_sources* src) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!src) {
        h->has_sources = false;
        return RPL_OK;
    }
    const rpl_sources& s = *src;
    if (s.wind_kind < RPL_WIND_NONE || s.wind_kind > RPL_WIND_FIELD) return fail(RPL_ERR_ARGUMENT, "unknown wind kind");
    if (s.drag_form != 0 && s.drag_form != 1) return fail(RPL_ERR_ARGUMENT, "unknown drag form");
    if (s.wind_kind != RPL_WIND_NONE) {
        if (!(s.wind_gravity > 0.0) || !(s.rho_water > 0.0) || !(s.von_karman > 0.0))
            return fail(RPL_ERR_ARGUMENT, "wind-input gravity, water density and von Karman constant must be positive");
    }
    if (s.wind_kind == RPL_WIND_HOLLAND) {
        // winds.jl:219-222
        if (!(s.vmax >= 0.0)) return fail(RPL_ERR_ARGUMENT, "Holland hurricane vmax must be nonnegative");
        if (!(s.rmax > 0.0)) return fail(RPL_ERR_ARGUMENT, "Holland hurricane rmax must be positive");
        if (!(s.radius > s.rmax)) return fail(RPL_ERR_ARGUMENT, "Holland hurricane radius must exceed rmax");
        if (!(s.shape_parameter > 0.0))
            return fail(RPL_ERR_ARGUMENT, "Holland hurricane shape_parameter must be positive");
        if (s.rotation != 1 && s.rotation != -1) return fail(RPL_ERR_ARGUMENT, "rotation must be +1 or -1");
        if (s.n_track < 0 || !s.track_x || !s.track_y)
            return fail(RPL_ERR_ARGUMENT, "Holland wind needs a centre (track_x, track_y)");
        if (s.n_track > 0) {
            if (!s.track_t) return fail(RPL_ERR_ARGUMENT, "storm track needs times");
            for (int64_t k = 1; k < s.n_track; ++k)  // winds.jl:127-130
                if (!(s.track_t[k] > s.track_t[k - 1]))
                    return fail(RPL_ERR_ARGUMENT, "storm-track times must be strictly increasing");
        }
    }
    if (s.has_dissipation && (!(s.B_r > 0.0) || !(s.ds_gravity > 0.0)))
        return fail(RPL_ERR_ARGUMENT, "whitecapping B_r and gravity must be positive");
    h->src = s;
    h->track_t.clear();
    h->track_x.clear();
    h->track_y.clear();
    if (s.wind_kind == RPL_WIND_HOLLAND) {
        const int64_t n = s.n_track > 0 ? s.n_track : 1;
        if (s.n_track > 0) h->track_t.assign(s.track_t, s.track_t + n);
        h->track_x.assign(s.track_x, s.track_x + n);
        h->track_y.assign(s.track_y, s.track_y + n);
    }
    h->src.track_t = nullptr;
    h->src.track_x = nullptr;
    h->src.track_y = nullptr;
    h->has_sources = s.wind_kind != RPL_WIND_NONE || s.has_dissipation;
    h->wind_field_set = false;
    // per-kappa FP32 source constants (rpl_src32.cuh)
    {
        const int64_t Nk = h->desc.Nk;
        std::vector<float> bins(8 * Nk, 0.0f);
        for (int64_t m = 0; m < Nk; ++m) {
            const double k = h->kappa[m];
            if (s.wind_kind != RPL_WIND_NONE) {
                const double sw = std::sqrt(s.wind_gravity * k);
                bins[8 * m] = (float)std::log(k);
                bins[8 * m + 1] = (float)(k / sw);
                bins[8 * m + 2] = (float)sw;
            }
            if (s.has_dissipation) {
                const double sd = std::sqrt(s.ds_gravity * k);
                bins[8 * m + 3] = (float)(sd * (k * k * k) / s.B_r);
                bins[8 * m + 4] = (float)(-s.C_ds * std::pow(sd, s.sigma_power));
            }
        }
        RPL_CUDA(cudaMemcpyAsync(h->d_bin32, bins.data(), bins.size() * 4, cudaMemcpyHostToDevice, h->stream));
    }
    // factor = 1 until a stress kernel runs
    const int64_t P = h->cells;
    std::vector<double> ones(P, 1.0);
    RPL_CUDA(cudaMemcpyAsync(h->d_wind + 3 * P, ones.data(), P * 8, cudaMemcpyHostToDevice, h->stream));
    RPL_CUDA(cudaStreamSynchronize(h->stream));
    return RPL_OK;
}

int rpl_set_wind_field(rpl_handle* hh, const double* U10, const double* dir) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!U10 || !dir) return fail(RPL_ERR_ARGUMENT, "null wind field");
    if (!(h->has_sources && h->src.wind_kind == RPL_WIND_FIELD))
        return fail(RPL_ERR_STATE, "rpl_set_wind_field needs sources with RPL_WIND_FIELD");
    const int64_t P = h->cells;
    if (!finite_all(U10, P) || !finite_all(dir, P)) return fail(RPL_ERR_NONFINITE, "non-finite wind field");
    RPL_CUDA(cudaMemcpyAsync(h->d_wind, U10, P * 8, cudaMemcpyHostToDevice, h->stream));
    RPL_CUDA(cudaMemcpyAsync(h->d_wind + P, dir, P * 8, cudaMemcpyHostToDevice, h->stream));
    RPL_CUDA(cudaStreamSynchronize(h->stream));
    h->wind_field_set = true;
    return RPL_OK;
}

static int set_action_impl(Handle* h, const void* N, int32_t dtype, int32_t layout, bool device) {
    if (!N) return fail(RPL_ERR_ARGUMENT, "null action array");
    if (layout != RPL_LAYOUT_XFAST) return fail(RPL_ERR_ARGUMENT, "unknown layout");
    if (dtype != RPL_F64 && dtype != RPL_F32) return fail(RPL_ERR_ARGUMENT, "unknown dtype");
    cudaStream_t s = h->stream;
    const int64_t n = h->units;
    const size_t src_elem = dtype == RPL_F64 ? 8 : 4;
    const int state_dtype = h->precision == RPL_FP64 ? RPL_F64 : RPL_F32;
    const int64_t Nk = h->desc.Nk, Np = h->desc.Np, P = h->cells, slice = P * Nk;
    if (device) {
        RPL_CUDA(rpl::launch_to_device_layout(*h, N, dtype, h->N, state_dtype, 0, Np, 0, Nk, s));
    } else {
        // staged through buffer A (free between steps), transposed into the device layout chunk by chunk
        const int64_t cap = (int64_t)(h->units * h->elem / src_elem);  // source elements that fit in A
        if (cap >= slice) {
            const int64_t per = cap / slice;
            for (int64_t n0 = 0; n0 < Np; n0 += per) {
                const int64_t nc = std::min<int64_t>(per, Np - n0);
                RPL_CUDA(cudaMemcpyAsync(h->A, (const char*)N + n0 * slice * src_elem, nc * slice * src_elem,
                                         cudaMemcpyHostToDevice, s));
                RPL_CUDA(rpl::launch_to_device_layout(*h, h->A, dtype, h->N, state_dtype, n0, nc, 0, Nk, s));
            }
        } else {
            const int64_t rows = std::max<int64_t>(1, cap / P);
            for (int64_t n0 = 0; n0 < Np; ++n0)
                for (int64_t m0 = 0; m0 < Nk; m0 += rows) {
                    const int64_t mc = std::min<int64_t>(rows, Nk - m0);
                    RPL_CUDA(cudaMemcpyAsync(h->A, (const char*)N + (n0 * slice + m0 * P) * src_elem,
                                             mc * P * src_elem, cudaMemcpyHostToDevice, s));
                    RPL_CUDA(rpl::launch_to_device_layout(*h, h->A, dtype, h->N, state_dtype, n0, 1, m0, mc, s));
                }
        }
    }
    RPL_CUDA(rpl::launch_scan_nonfinite(*h, h->N, s));
    int st = check_error_word(h);
    if (st) {
        cudaMemsetAsync(h->N, 0, n * h->elem, s);
        cudaStreamSynchronize(s);
    }
    return st;
}

static int get_action_impl(Handle* h, void* N, int32_t dtype, int32_t layout, bool device) {
    if (!N) return fail(RPL_ERR_ARGUMENT, "null action array");
    if (layout != RPL_LAYOUT_XFAST) return fail(RPL_ERR_ARGUMENT, "unknown layout");
    if (dtype != RPL_F64 && dtype != RPL_F32) return fail(RPL_ERR_ARGUMENT, "unknown dtype");
    cudaStream_t s = h->stream;
    const int64_t n = h->units;
    const size_t dst_elem = dtype == RPL_F64 ? 8 : 4;
    const int state_dtype = h->precision == RPL_FP64 ? RPL_F64 : RPL_F32;
    (void)n;
    const int64_t Nk = h->desc.Nk, Np = h->desc.Np, P = h->cells, slice = P * Nk;
    if (device) {
        RPL_CUDA(rpl::launch_from_device_layout(*h, h->N, state_dtype, N, dtype, 0, Np, 0, Nk, s));
    } else {
        const int64_t cap = (int64_t)(h->units * h->elem / dst_elem);  // destination elements that fit in A
        if (cap >= slice) {
            const int64_t per = cap / slice;
            for (int64_t n0 = 0; n0 < Np; n0 += per) {
                const int64_t nc = std::min<int64_t>(per, Np - n0);
                RPL_CUDA(rpl::launch_from_device_layout(*h, h->N, state_dtype, h->A, dtype, n0, nc, 0, Nk, s));
                RPL_CUDA(cudaMemcpyAsync((char*)N + n0 * slice * dst_elem, h->A, nc * slice * dst_elem,
                                         cudaMemcpyDeviceToHost, s));
            }
        } else {
            const int64_t rows = std::max<int64_t>(1, cap / P);
            for (int64_t n0 = 0; n0 < Np; ++n0)
                for (int64_t m0 = 0; m0 < Nk; m0 += rows) {
                    const int64_t mc = std::min<int64_t>(rows, Nk - m0);
                    RPL_CUDA(rpl::launch_from_device_layout(*h, h->N, state_dtype, h->A, dtype, n0, 1, m0, mc, s));
                    RPL_CUDA(cudaMemcpyAsync((char*)N + (n0 * slice + m0 * P) * dst_elem, h->A, mc * P * dst_elem,
                                             cudaMemcpyDeviceToHost, s));
                }
        }
    }
    RPL_CUDA(cudaStreamSynchronize(s));
    return RPL_OK;
}

int rpl_set_action(rpl_handle* hh, const void* N, int32_t dtype, int32_t layout) {
    int st = check_handle(hh);
    if (st) return st;
    return set_action_impl(reinterpret_cast<Handle*>(hh), N, dtype, layout, false);
}

int rpl_get_action(rpl_handle* hh, void* N, int32_t dtype, int32_t layout) {
    int st = check_handle(hh);
    if (st) return st;
    return get_action_impl(reinterpret_cast<Handle*>(hh), N, dtype, layout, false);
}

int rpl_set_action_device(rpl_handle* hh, const void* N, int32_t dtype, int32_t layout) {
    int st = check_handle(hh);
    if (st) return st;
    return set_action_impl(reinterpret_cast<Handle*>(hh), N, dtype, layout, true);
}

int rpl_get_action_device(rpl_handle* hh, void* N, int32_t dtype, int32_t layout) {
    int st = check_handle(hh);
    if (st) return st;
    return get_action_impl(reinterpret_cast<Handle*>(hh), N, dtype, layout, true);
}

int rpl_set_clock(rpl_handle* hh, double time, int64_t iteration) {
    if (!hh) return fail(RPL_ERR_ARGUMENT, "null handle");
    if (!std::isfinite(time) || iteration < 0) return fail(RPL_ERR_ARGUMENT, "bad clock");
    Handle* h = reinterpret_cast<Handle*>(hh);
    h->time = time;
    h->iteration = iteration;
    return RPL_OK;
}

int rpl_get_clock(rpl_handle* hh, double* time, int64_t* iteration) {
    if (!hh) return fail(RPL_ERR_ARGUMENT, "null handle");
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (time) *time = h->time;
    if (iteration) *iteration = h->iteration;
    return RPL_OK;
}

int rpl_step_async(rpl_handle* hh, double dt, int64_t nsteps) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if ((st = check_step_args(h, dt))) return st;
    if (nsteps < 0) return fail(RPL_ERR_ARGUMENT, "nsteps must be non-negative");
    for (int64_t k = 0; k < nsteps; ++k)
        if ((st = launch_step(h, dt, 0))) return st;
    return RPL_OK;
}

int rpl_step(rpl_handle* hh, double dt, int64_t nsteps) {
    int st = rpl_step_async(hh, dt, nsteps);
    if (st) return st;
    return rpl_sync(hh);
}

int rpl_stage_async(rpl_handle* hh, double dt, int32_t stage) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if ((st = check_step_args(h, dt))) return st;
    if (stage < 1 || stage > 3) return fail(RPL_ERR_ARGUMENT, "stage must be 1, 2 or 3");
    return launch_step(h, dt, stage);
}

int rpl_stage_rows_async(rpl_handle* hh, double dt, int32_t stage, int64_t row0, int64_t nrows, int32_t flags) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if ((st = check_step_args(h, dt))) return st;
    if (stage < 1 || stage > 3) return fail(RPL_ERR_ARGUMENT, "stage must be 1, 2 or 3");
    if (row0 < 0 || nrows < 0 || row0 + nrows > h->desc.Ny) return fail(RPL_ERR_ARGUMENT, "rows out of range");
    if (flags & ~(RPL_STAGE_PREPARE | RPL_STAGE_FINISH | RPL_STAGE_DEFER_SMOOTH))
        return fail(RPL_ERR_ARGUMENT, "unknown stage flags");
    return launch_stage_rows(h, dt, stage, row0, row0 + nrows, (flags & RPL_STAGE_PREPARE) != 0,
                             (flags & RPL_STAGE_FINISH) != 0, (flags & RPL_STAGE_DEFER_SMOOTH) != 0);
}

int rpl_smooth_rows_async(rpl_handle* hh, double dt, int64_t row0, int64_t nrows, int64_t y_offset) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if ((st = check_step_args(h, dt))) return st;
    if (!h->smooth) return fail(RPL_ERR_STATE, "the model has no SpatialAveraging");
    if (row0 < 0 || nrows < 0 || row0 + nrows > h->desc.Ny) return fail(RPL_ERR_ARGUMENT, "rows out of range");
    if (nrows == 0) return RPL_OK;
    RPL_CUDA(rpl::launch_smooth(*h, h->A, h->N, dt, row0, row0 + nrows, y_offset, h->stream));
    return RPL_OK;
}

int rpl_sync(rpl_handle* hh) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    RPL_CUDA(cudaStreamSynchronize(h->stream));
    return check_error_word(h);
}

int rpl_set_stream(rpl_handle* hh, void* stream) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    RPL_CUDA(cudaStreamSynchronize(h->stream));
    if (h->own_stream) {
        cudaStreamDestroy(h->stream);
        h->own_stream = false;
    }
    if (stream) {
        h->stream = (cudaStream_t)stream;
    } else {
        RPL_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->own_stream = true;
    }
    return RPL_OK;
}

int rpl_tendency(rpl_handle* hh, double* G, int32_t layout) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!G) return fail(RPL_ERR_ARGUMENT, "null output");
    if (layout != RPL_LAYOUT_XFAST) return fail(RPL_ERR_ARGUMENT, "unknown layout");
    if ((st = check_step_args(h, 1.0))) return st;
    cudaStream_t s = h->stream;
    double *dG = nullptr, *dGx = nullptr;
    RPL_CUDA(cudaMalloc(&dG, h->units * 8));
    cudaError_t e = cudaMalloc(&dGx, h->units * 8);
    if (e == cudaSuccess && h->has_sources && h->src.wind_kind != RPL_WIND_NONE) {
        e = rpl::launch_wind(*h, h->time, s);
        if (e == cudaSuccess && h->src.stress_cap) e = rpl::launch_stress_factor(*h, h->N, s);
    }
    if (e == cudaSuccess && h->pm) e = rpl::launch_pm_refresh(*h, h->N, s, true);
    if (e == cudaSuccess && h->n_terms) e = rpl::launch_terms(*h, h->N, s);
    if (e == cudaSuccess) e = rpl::launch_tendency(*h, rpl::make_params(*h, 1.0, 1), h->N, dG, s);
    if (e == cudaSuccess)
        e = rpl::launch_from_device_layout(*h, dG, RPL_F64, dGx, RPL_F64, 0, h->desc.Np, 0, h->desc.Nk, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(G, dGx, h->units * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(dG);
    if (dGx) cudaFree(dGx);
    if (e != cudaSuccess) return cuda_fail(e, "rpl_tendency");
    return RPL_OK;
}

int rpl_diagnostics(rpl_handle* hh, double* m0, double* hs, double* krms, double* mean_dir, double* total) {
    int st = check_handle(hh);
    if (st) return st;
    Handle* h = reinterpret_cast<Handle*>(hh);
    cudaStream_t s = h->stream;
    const int64_t P = h->cells;
    RPL_CUDA(rpl::launch_diagnostics(*h, h->N, s, hs || krms || mean_dir));
    double* outs[4] = {m0, hs, krms, mean_dir};
    for (int k = 0; k < 4; ++k)
        if (outs[k]) RPL_CUDA(cudaMemcpyAsync(outs[k], h->d_diag + k * P, P * 8, cudaMemcpyDeviceToHost, s));
    if (total) RPL_CUDA(cudaMemcpyAsync(total, h->d_diag + 4 * P, 8, cudaMemcpyDeviceToHost, s));
    RPL_CUDA(cudaStreamSynchronize(s));
    return RPL_OK;
}

int rpl_device_bytes(rpl_handle* hh, int64_t* bytes) {
    if (!hh || !bytes) return fail(RPL_ERR_ARGUMENT, "null argument");
    *bytes = reinterpret_cast<Handle*>(hh)->bytes;
    return RPL_OK;
}

}  // extern "C"
