// rpl_terms.cu -- SourceTermSet terms whose tendency is linear in the action (rpl_set_source_terms):
// ExponentialWindInput, WaveAgeWindInput, WhitecappingDissipation, MeanSpectrumWhitecapping.
//
// Before every stage (and for rpl_tendency) terms_kernel turns the stage's action into one rate per
// cell-bin, R(i,j,m,n) = sum over terms of +rate (wind input, split_growth_rate) or -rate (dissipation,
// split_damping_rate) (src/Sources/Sources.jl:430-434,443-449), written in the state's layout and type;
// the stage kernels then add R * N to the tendency. With up to 4 terms, terms_cols_kernel and
// terms_bins_kernel (below) split the work by column and by bin; otherwise terms_kernel does both passes
// in one warp per (i,j) column, lanes over kappa bins:
//   pass 1 sums the column's integrals in FP64: m0 = sum N w over every bin (local_zeroth_moment,
//     Sources.jl:1471-1480) and, per MeanSpectrumWhitecapping term, sum N w k^p, N w sigma^p and N w over
//     the bins with N > 0 and k > 0 (mean_spectrum.jl:43-82);
//   pass 2 forms each bin's rate from those per-cell values and per-bin tables built once on the host
//     (directional weights, alignments, radial-power averages, the bins' |k|).
// The per-bin tables restate Sources.jl:1394-1434 (directional cell averages of max(cos, 0)^p),
// Sources.jl:522-554 (wave-age alignment and phase speed) and finite_volume_integration.jl:24-33,86-88
// (kappa^p cell averages); the terms' formulas follow Sources.jl:492-496,522-554,588-598 and
// mean_spectrum.jl:90-111.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "rpl_internal.h"

namespace rpl {

namespace {

constexpr int TABS = 4;  // bin tables per term

struct TermsArgs {
    int64_t P, Nk, Np;
    int n;
    int kind[RPL_MAX_TERMS];
    double rate[RPL_MAX_TERMS], speed[RPL_MAX_TERMS];
    const double* rate_field[RPL_MAX_TERMS];
    const double* speed_field[RPL_MAX_TERMS];
    double p[RPL_MAX_TERMS][4];
    const double* tabs;     // TABS * Nk * Np per term
    const double* weights;  // (Nk, Np) spectral cell measures
};

// x^e for x >= 0: small integer powers by products (x^0 = 1, including 0^0 as the reference's ^;
// x^1 = x exactly), others by pow. The wave-age input's default power is 1 (Sources.jl:77-84).
__device__ __forceinline__ double pow_nonneg(double x, double e) {
    if (e == 1.0) return x;
    if (e == 0.0) return 1.0;
    if (e == 2.0) return x * x;
    if (e == 3.0) return x * x * x;
    if (e == 4.0) {
        const double x2 = x * x;
        return x2 * x2;
    }
    return pow(x, e);
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__global__ void __launch_bounds__(256) terms_kernel(const T* __restrict__ N, TermsArgs a, T* __restrict__ R) {
    // each column's per-term values (x0, x1) for the bin pass, one slot per warp: no per-thread arrays
    // indexed by the runtime term number (those would live in local memory)
    __shared__ double2 cell[256 / 32][RPL_MAX_TERMS];
    const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (c >= a.P) return;  // uniform per warp
    const int64_t Nk = a.Nk, Np = a.Np, nb = Nk * Np;
    // pass 1: m0 = sum N w over the column
    double m0 = 0.0;
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = lane; m < Nk; m += 32)
            m0 += (double)N[(n * a.P + c) * Nk + m] * a.weights[m + Nk * n];
    m0 = warp_sum(m0);
    // per-cell values of each term: (x0, x1); a mean-spectrum term sums its column integrals first
    for (int t = 0; t < a.n; ++t) {
        const double rate = a.rate_field[t] ? a.rate_field[t][c] : a.rate[t];
        double x0 = 0.0, x1 = 0.0;
        switch (a.kind[t]) {
            case RPL_TERM_EXPONENTIAL_WIND:
                x0 = rate;
                break;
            case RPL_TERM_WAVE_AGE_WIND:
                x0 = rate;
                x1 = a.speed_field[t] ? a.speed_field[t][c] : a.speed[t];
                break;
            case RPL_TERM_WHITECAPPING: {
                const double excess = fmax(m0 / a.p[t][0] - 1.0, 0.0);
                x0 = rate * pow(excess, a.p[t][1]);
                break;
            }
            default: {  // mean spectrum: x0 = -C_ds (m0 kbar^2)^2 sigmabar, x1 = kbar (0: no dissipation)
                const double* tb = a.tabs + (int64_t)t * TABS * nb;
                double sk = 0.0, ss = 0.0, sd = 0.0;
                for (int64_t n = 0; n < Np; ++n)
                    for (int64_t m = lane; m < Nk; m += 32) {
                        const double v = (double)N[(n * a.P + c) * Nk + m];
                        const int64_t b = m + Nk * n;
                        if (v > 0.0) {
                            sk += v * tb[nb + b];
                            ss += v * tb[2 * nb + b];
                            sd += v * tb[3 * nb + b];
                        }
                    }
                const double num_k = warp_sum(sk), num_s = warp_sum(ss), den = warp_sum(sd);
                const double q = a.p[t][3];
                const double kbar = den > 0.0 ? pow(num_k / den, 1.0 / q) : 0.0;
                const double sbar = den > 0.0 ? pow(num_s / den, 1.0 / q) : 0.0;
                if (m0 > 0.0 && kbar > 0.0) {
                    const double alpha = m0 * kbar * kbar;
                    x0 = -a.p[t][0] * alpha * alpha * sbar;
                    x1 = kbar;
                }
                break;
            }
        }
        if (lane == 0) cell[w][t] = make_double2(x0, x1);
    }
    __syncwarp();
    // pass 2: the rate of every bin
    for (int64_t n = 0; n < Np; ++n)
        for (int64_t m = lane; m < Nk; m += 32) {
            const int64_t b = m + Nk * n;
            double r = 0.0;
            for (int t = 0; t < a.n; ++t) {
                const double* tb = a.tabs + (int64_t)t * TABS * nb;
                const double2 x = cell[w][t];
                switch (a.kind[t]) {
                    case RPL_TERM_EXPONENTIAL_WIND:
                        r += x.x * tb[b];
                        break;
                    case RPL_TERM_WAVE_AGE_WIND: {
                        const double al = tb[b];
                        if (al > 0.0) {
                            const double excess = fmax(x.y * al * tb[nb + b] - a.p[t][0], 0.0);
                            r += x.x * pow_nonneg(excess, a.p[t][1]) * tb[2 * nb + b];
                        }
                        break;
                    }
                    case RPL_TERM_WHITECAPPING:
                        r -= x.x * tb[b];
                        break;
                    default: {
                        const double k = tb[b];
                        if (x.y > 0.0 && k > 0.0) {
                            const double ratio = k / x.y;
                            r -= x.x * (a.p[t][1] * ratio + a.p[t][2] * ratio * ratio);
                        }
                        break;
                    }
                }
            }
            R[(n * a.P + c) * Nk + m] = (T)r;
        }
}

// Two-kernel form for up to 4 terms. terms_cols_kernel (one warp per column): m0, the mean-spectrum
// integrals and every term's per-cell values (x0, x1), written to tcol[c * n + t]. terms_bins_kernel:
// one thread per (m, n) bin walking a chunk of columns with its bin's table entries in registers
// (NT terms, unrolled), the column values read once per warp (all lanes read the same record) and the
// rates stored coalesced along kappa. The per-bin arithmetic is terms_kernel's.
template <typename T>
__global__ void __launch_bounds__(256) terms_cols_kernel(const T* __restrict__ N, TermsArgs a, double2* __restrict__ tcol) {
    const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= a.P) return;  // uniform per warp
    const int64_t Nk = a.Nk, Np = a.Np, nb = Nk * Np;
    // the column pass: m0 and the integrals of the first mean-spectrum term together, four independent
    // partial sums per lane (directions n mod 4) so the loads of four directions are in flight at once
    int tm = -1;
    for (int t = a.n - 1; t >= 0; --t)
        if (a.kind[t] == RPL_TERM_MEAN_SPECTRUM) tm = t;
    const double* tbm = a.tabs + (int64_t)(tm < 0 ? 0 : tm) * TABS * nb;
    double m0p[4] = {0.0, 0.0, 0.0, 0.0}, skp[4] = {0.0, 0.0, 0.0, 0.0}, ssp[4] = {0.0, 0.0, 0.0, 0.0},
           sdp[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t m = lane; m < Nk; m += 32)
        for (int64_t n0 = 0; n0 < Np; n0 += 4) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int64_t n = n0 + q;
                if (n < Np) {
                    const double v = (double)N[(n * a.P + c) * Nk + m];
                    const int64_t b = m + Nk * n;
                    m0p[q] += v * a.weights[b];
                    if (tm >= 0 && v > 0.0) {
                        skp[q] += v * tbm[nb + b];
                        ssp[q] += v * tbm[2 * nb + b];
                        sdp[q] += v * tbm[3 * nb + b];
                    }
                }
            }
        }
    const double m0 = warp_sum((m0p[0] + m0p[1]) + (m0p[2] + m0p[3]));
    for (int t = 0; t < a.n; ++t) {
        const double rate = a.rate_field[t] ? a.rate_field[t][c] : a.rate[t];
        double x0 = 0.0, x1 = 0.0;
        switch (a.kind[t]) {
            case RPL_TERM_EXPONENTIAL_WIND:
                x0 = rate;
                break;
            case RPL_TERM_WAVE_AGE_WIND:
                x0 = rate;
                x1 = a.speed_field[t] ? a.speed_field[t][c] : a.speed[t];
                break;
            case RPL_TERM_WHITECAPPING: {
                const double excess = fmax(m0 / a.p[t][0] - 1.0, 0.0);
                x0 = rate * pow(excess, a.p[t][1]);
                break;
            }
            default: {  // mean spectrum: x0 = -C_ds (m0 kbar^2)^2 sigmabar, x1 = kbar (0: no dissipation)
                double sk, ss, sd;
                if (t == tm) {
                    sk = (skp[0] + skp[1]) + (skp[2] + skp[3]);
                    ss = (ssp[0] + ssp[1]) + (ssp[2] + ssp[3]);
                    sd = (sdp[0] + sdp[1]) + (sdp[2] + sdp[3]);
                } else {   // a further mean-spectrum term: its own pass
                    const double* tb = a.tabs + (int64_t)t * TABS * nb;
                    sk = ss = sd = 0.0;
                    for (int64_t n = 0; n < Np; ++n)
                        for (int64_t m = lane; m < Nk; m += 32) {
                            const double v = (double)N[(n * a.P + c) * Nk + m];
                            const int64_t b = m + Nk * n;
                            if (v > 0.0) {
                                sk += v * tb[nb + b];
                                ss += v * tb[2 * nb + b];
                                sd += v * tb[3 * nb + b];
                            }
                        }
                }
                const double num_k = warp_sum(sk), num_s = warp_sum(ss), den = warp_sum(sd);
                const double q = a.p[t][3];
                const double kbar = den > 0.0 ? pow(num_k / den, 1.0 / q) : 0.0;
                const double sbar = den > 0.0 ? pow(num_s / den, 1.0 / q) : 0.0;
                if (m0 > 0.0 && kbar > 0.0) {
                    const double alpha = m0 * kbar * kbar;
                    x0 = -a.p[t][0] * alpha * alpha * sbar;
                    x1 = kbar;
                }
                break;
            }
        }
        if (lane == 0) tcol[c * a.n + t] = make_double2(x0, x1);
    }
}

constexpr int TERM_COLS = 128;   // columns per thread in terms_bins_kernel (more on very large grids)

template <typename T, int NT>
__global__ void __launch_bounds__(256) terms_bins_kernel(TermsArgs a, const double2* __restrict__ tcol, T* __restrict__ R,
                                                         int64_t chunk) {
    const int64_t nb = a.Nk * a.Np;
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const int64_t Nk = a.Nk, m = b % Nk, n = b / Nk;
    const int64_t c0 = (int64_t)blockIdx.y * chunk, c1 = min(c0 + chunk, a.P);
    double t0[NT], t1[NT], t2[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const double* tb = a.tabs + (int64_t)t * TABS * nb;
        t0[t] = tb[b];
        t1[t] = tb[nb + b];
        t2[t] = tb[2 * nb + b];
    }
    for (int64_t c = c0; c < c1; ++c) {
        double r = 0.0;
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const double2 x = __ldg(tcol + c * NT + t);
            switch (a.kind[t]) {
                case RPL_TERM_EXPONENTIAL_WIND:
                    r += x.x * t0[t];
                    break;
                case RPL_TERM_WAVE_AGE_WIND: {
                    const double al = t0[t];
                    if (al > 0.0) {
                        const double excess = fmax(x.y * al * t1[t] - a.p[t][0], 0.0);
                        r += x.x * pow_nonneg(excess, a.p[t][1]) * t2[t];
                    }
                    break;
                }
                case RPL_TERM_WHITECAPPING:
                    r -= x.x * t0[t];
                    break;
                default: {
                    const double k = t0[t];
                    if (x.y > 0.0 && k > 0.0) {
                        const double ratio = k / x.y;
                        r -= x.x * (a.p[t][1] * ratio + a.p[t][2] * ratio * ratio);
                    }
                    break;
                }
            }
        }
        R[(n * a.P + c) * Nk + m] = (T)r;
    }
}

// integral of max(cos, 0)^power over [a1, a2] (power >= 0 an integer): the antiderivative of cos^power
// by its reduction formula, summed over the half periods where cos > 0
double cos_power_antiderivative(double x, int power) {
    if (power == 0) return x;
    if (power == 1) return std::sin(x);
    return std::sin(x) * std::pow(std::cos(x), power - 1) / power +
           (double)(power - 1) / power * cos_power_antiderivative(x, power - 2);
}

double positive_cos_power_integral(double a1, double a2, int power) {
    if (a2 < a1) return -positive_cos_power_integral(a2, a1, power);
    if (power == 0) return a2 - a1;
    const double period = 2.0 * M_PI;
    const int64_t lo = (int64_t)std::floor((a1 - M_PI / 2) / period) - 1;
    const int64_t hi = (int64_t)std::ceil((a2 + M_PI / 2) / period) + 1;
    double total = 0.0;
    for (int64_t q = lo; q <= hi; ++q) {
        const double shift = q * period;
        const double left = std::max(a1, shift - M_PI / 2), right = std::min(a2, shift + M_PI / 2);
        if (right > left)
            total += cos_power_antiderivative(right - shift, power) - cos_power_antiderivative(left - shift, power);
    }
    return total;
}

int fail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

bool finite_field(const double* f, int64_t n) {
    for (int64_t k = 0; k < n; ++k)
        if (!std::isfinite(f[k])) return false;
    return true;
}

std::string check_term(const rpl_source_term& t) {
    if (!std::isfinite(t.rate) || !std::isfinite(t.direction) || !std::isfinite(t.speed))
        return "source-term parameters must be finite";
    switch (t.kind) {
        case RPL_TERM_EXPONENTIAL_WIND:  // Sources.jl:1387-1392
            if (!(t.p[0] >= 0.0)) return "directional spreading power must be nonnegative";
            if (t.p[0] != std::floor(t.p[0]) || t.p[0] > 64.0)
                return "finite-volume directional spreading currently supports nonnegative integer powers";
            return "";
        case RPL_TERM_WAVE_AGE_WIND:  // Sources.jl:523-526
            if (!(t.p[0] >= 0.0)) return "wave-age wind-input threshold must be nonnegative";
            if (!(t.p[1] >= 0.0)) return "wave-age wind-input power must be nonnegative";
            if (!(t.p[2] >= 0.0)) return "wave-age wind-input spreading power must be nonnegative";
            if (!(t.gravity > 0.0)) return "wave-age wind-input gravity must be positive";
            return "";
        case RPL_TERM_WHITECAPPING:  // Sources.jl:589-590, 568-569
            if (!(t.p[0] > 0.0)) return "whitecapping saturation threshold must be positive";
            if (!(t.p[3] > 0.0)) return "whitecapping reference wavenumber must be positive";
            if (!(t.p[2] >= 0.0)) return "wavenumber power must be nonnegative";
            return "";
        case RPL_TERM_MEAN_SPECTRUM:
            if (!(t.p[3] != 0.0) || !std::isfinite(t.p[3])) return "mean-spectrum exponent p must be nonzero";
            if (!(t.gravity > 0.0)) return "mean-spectrum gravity must be positive";
            return "";
        default:
            return "unknown source-term kind";
    }
}

}  // namespace

void free_terms(Handle* h) {
    if (h->d_lin_rates) cudaFree(h->d_lin_rates);
    if (h->d_terms) cudaFree(h->d_terms);
    if (h->d_tcol) cudaFree(h->d_tcol);
    h->bytes -= h->terms_bytes;
    h->d_lin_rates = nullptr;
    h->d_terms = nullptr;
    h->d_tcol = nullptr;
    h->terms_bytes = 0;
    h->n_terms = 0;
}

cudaError_t launch_terms(const Handle& h, const void* Nin, cudaStream_t s) {
    const rpl_desc& d = h.desc;
    TermsArgs a{};
    a.P = d.Nx * d.Ny;
    a.Nk = d.Nk;
    a.Np = d.Np;
    a.n = h.n_terms;
    for (int t = 0; t < h.n_terms; ++t) {
        const rpl_source_term& q = h.terms[t];
        a.kind[t] = q.kind;
        a.rate[t] = q.rate;
        a.speed[t] = q.speed;
        a.rate_field[t] = q.rate_field;
        a.speed_field[t] = q.speed_field;
        for (int k = 0; k < 4; ++k) a.p[t][k] = q.p[k];
    }
    a.tabs = h.d_terms;
    a.weights = h.d_weights;
    const unsigned blocks = (unsigned)((a.P * 32 + 255) / 256);
    const bool fp64 = h.precision == RPL_FP64;
    if (h.d_tcol) {   // up to 4 terms: column values, then the bins
        if (fp64) terms_cols_kernel<double><<<blocks, 256, 0, s>>>((const double*)Nin, a, h.d_tcol);
        else terms_cols_kernel<float><<<blocks, 256, 0, s>>>((const float*)Nin, a, h.d_tcol);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        const int64_t chunk = std::max<int64_t>(TERM_COLS, (a.P + 65534) / 65535);   // grid.y <= 65535
        const dim3 grid((unsigned)((a.Nk * a.Np + 255) / 256), (unsigned)((a.P + chunk - 1) / chunk));
        switch (a.n) {
#define RPL_BINS(NT)                                                                                           \
    case NT:                                                                                                   \
        if (fp64) terms_bins_kernel<double, NT><<<grid, 256, 0, s>>>(a, h.d_tcol, (double*)h.d_lin_rates, chunk); \
        else terms_bins_kernel<float, NT><<<grid, 256, 0, s>>>(a, h.d_tcol, (float*)h.d_lin_rates, chunk);  \
        break;
            RPL_BINS(1)
            RPL_BINS(2)
            RPL_BINS(3)
            RPL_BINS(4)
#undef RPL_BINS
            default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
    if (fp64)
        terms_kernel<double><<<blocks, 256, 0, s>>>((const double*)Nin, a, (double*)h.d_lin_rates);
    else
        terms_kernel<float><<<blocks, 256, 0, s>>>((const float*)Nin, a, (float*)h.d_lin_rates);
    return cudaGetLastError();
}

}  // namespace rpl

extern "C" int rpl_set_source_terms(rpl_handle* hh, const rpl_source_term* terms, int32_t count) {
    using namespace rpl;
    if (!hh) return fail(RPL_ERR_ARGUMENT, "null handle");
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (count < 0 || count > RPL_MAX_TERMS)
        return fail(RPL_ERR_ARGUMENT, "between 0 and " + std::to_string(RPL_MAX_TERMS) + " source terms");
    if (count > 0 && !terms) return fail(RPL_ERR_ARGUMENT, "null source-term array");
    const rpl_desc& d = h->desc;
    const int64_t P = d.Nx * d.Ny, Nk = d.Nk, Np = d.Np, nb = Nk * Np;
    int64_t nfields = 0;
    for (int t = 0; t < count; ++t) {
        const std::string msg = check_term(terms[t]);
        if (!msg.empty()) return fail(RPL_ERR_ARGUMENT, msg);
        if (terms[t].rate_field) {
            if (!finite_field(terms[t].rate_field, P)) return fail(RPL_ERR_NONFINITE, "non-finite source rate field");
            ++nfields;
        }
        if (terms[t].kind == RPL_TERM_WAVE_AGE_WIND && terms[t].speed_field) {
            if (!finite_field(terms[t].speed_field, P)) return fail(RPL_ERR_NONFINITE, "non-finite wind speed field");
            ++nfields;
        }
    }
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return fail(RPL_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    e = cudaStreamSynchronize(h->stream);  // the previous buffers may be in use by enqueued stages
    if (e != cudaSuccess) return fail(RPL_ERR_CUDA, std::string("rpl_set_source_terms: ") + cudaGetErrorString(e));
    free_terms(h);
    if (count == 0) return RPL_OK;

    // per term TABS bin tables, then the fields
    std::vector<double> host((size_t)(count * TABS * nb + nfields * P), 0.0);
    int64_t foff = count * TABS * nb;
    rpl_source_term dev[RPL_MAX_TERMS];
    for (int t = 0; t < count; ++t) {
        const rpl_source_term& q = terms[t];
        dev[t] = q;
        double* tb = host.data() + (size_t)t * TABS * nb;
        for (int64_t n = 0; n < Np; ++n)
            for (int64_t m = 0; m < Nk; ++m) {
                const int64_t b = m + Nk * n;
                const double kap = h->kappa[m], phi = h->phi[n];
                const double kx = kap * std::cos(phi), ky = kap * std::sin(phi), k = std::hypot(kx, ky);
                const double p1 = h->phi_faces[n], p2 = h->phi_faces[n + 1];
                const double k1 = h->kappa_faces[m], k2 = h->kappa_faces[m + 1];
                const double w = (k2 * k2 - k1 * k1) / 2.0 * (p2 - p1);
                switch (q.kind) {
                    case RPL_TERM_EXPONENTIAL_WIND: {
                        const int pw = (int)q.p[0];
                        tb[b] = pw == 0 ? 1.0 : positive_cos_power_integral(p1 - q.direction, p2 - q.direction, pw) / (p2 - p1);
                        break;
                    }
                    case RPL_TERM_WAVE_AGE_WIND: {
                        const double al =
                            (kap <= 0.0 || k == 0.0) ? 0.0
                                                     : std::max((kx * std::cos(q.direction) + ky * std::sin(q.direction)) / k, 0.0);
                        tb[b] = al;
                        tb[nb + b] = kap > 0.0 ? 1.0 / std::sqrt(q.gravity / kap) : 0.0;
                        tb[2 * nb + b] = std::pow(al, q.p[2]);
                        break;
                    }
                    case RPL_TERM_WHITECAPPING: {
                        const double pw = q.p[2];
                        tb[b] = pw == 0.0 ? 1.0
                                          : ((p2 - p1) * (std::pow(k2, pw + 2.0) - std::pow(k1, pw + 2.0)) / (pw + 2.0)) /
                                                w / std::pow(q.p[3], pw);
                        break;
                    }
                    default: {
                        tb[b] = k;
                        if (k > 0.0) {
                            tb[nb + b] = w * std::pow(k, q.p[3]);
                            tb[2 * nb + b] = w * std::pow(std::sqrt(q.gravity * k), q.p[3]);
                            tb[3 * nb + b] = w;
                        }
                        break;
                    }
                }
            }
        if (q.rate_field) {
            std::copy(q.rate_field, q.rate_field + P, host.begin() + foff);
            dev[t].rate_field = reinterpret_cast<const double*>(foff);  // offset, rebased below
            foff += P;
        }
        if (q.kind == RPL_TERM_WAVE_AGE_WIND && q.speed_field) {
            std::copy(q.speed_field, q.speed_field + P, host.begin() + foff);
            dev[t].speed_field = reinterpret_cast<const double*>(foff);
            foff += P;
        } else {
            dev[t].speed_field = nullptr;
        }
    }
    const int64_t rate_bytes = h->units * (int64_t)h->elem, tab_bytes = (int64_t)host.size() * 8;
    const int64_t col_bytes = count <= 4 ? P * count * (int64_t)sizeof(double2) : 0;
    const int64_t limit = d.memory_limit_bytes;
    if (limit > 0 && h->bytes + rate_bytes + tab_bytes + col_bytes > limit)
        return fail(RPL_ERR_OOM, "source terms need " + std::to_string(rate_bytes + tab_bytes + col_bytes) +
                                     " more device bytes, above the memory limit");
    e = cudaMalloc(&h->d_lin_rates, rate_bytes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->d_terms, tab_bytes);
    if (e == cudaSuccess && col_bytes) e = cudaMalloc((void**)&h->d_tcol, col_bytes);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->d_terms, host.data(), tab_bytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        free_terms(h);
        return fail(e == cudaErrorMemoryAllocation ? RPL_ERR_OOM : RPL_ERR_CUDA,
                    std::string("rpl_set_source_terms: ") + cudaGetErrorString(e));
    }
    h->terms_bytes = rate_bytes + tab_bytes + col_bytes;
    h->bytes += h->terms_bytes;
    for (int t = 0; t < count; ++t) {
        h->terms[t] = dev[t];
        if (dev[t].rate_field) h->terms[t].rate_field = h->d_terms + reinterpret_cast<intptr_t>(dev[t].rate_field);
        if (dev[t].speed_field) h->terms[t].speed_field = h->d_terms + reinterpret_cast<intptr_t>(dev[t].speed_field);
    }
    h->n_terms = count;
    return RPL_OK;
}
