// rpl_stage.cu -- fused SSP-RK3 stage kernels: tendency (Doppler transport + refraction, or intrinsic
// transport) + sources + stage combination + max(0, .) clamp, one pass over the state per stage.
//
// Reference: src/Coupling/wave_current_refraction.jl:74-151 (tendency),
// src/Models/intrinsic_transport.jl:14-68, src/Models/tendencies.jl:28-41,82-101 (dispatch, sources),
// src/Models/time_step.jl:67-74,98-105,138-152 (stage update with clamp).
//
// Device layout of the state: kappa fastest, (i,j,m,n) at ((n*Ny + j)*Nx + i)*Nk + m.
//
// column_kernel (Nk <= 32): one warp segment of SEG lanes (SEG = Nk rounded up to a power of two)
// owns one horizontal cell (i,j) and walks the periodic phi ring n = 0 .. Np-1, lane m holding
// kappa bin m. Every face is reconstructed once where it can be:
//   kappa faces: the + face of lane m is the - face of lane m+1 (warp shuffle); the clamped kappa
//     stencil of the reference is a shuffle from the clamped lane;
//   phi faces: a 7-deep register window along the ring; the + face of step n is the - face of
//     step n+1;
//   x, y faces: both faces of the cell from one 7-point stencil, sharing its differences.
// A face is recomputed only where the two cells on its sides upwind in different directions
// (the reference upwinds each cell's two faces by that cell's own centre velocity).
// The per-(i,j,kappa) coupling record is read once per ring, i.e. once per Np cell-bins.
//
// generic_kernel (any Nk): one thread per cell-bin, same arithmetic, all neighbours from memory.
#include <cuda_runtime.h>

#include <type_traits>

#include "rpl_device.cuh"
#include "rpl_internal.h"

namespace rpl {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int BLOCK = 256;

template <typename T> __device__ __forceinline__ T rcp_w(T x);
template <> __device__ __forceinline__ float rcp_w<float>(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
template <> __device__ __forceinline__ double rcp_w<double>(double x) { return 1.0 / x; }

// Jiang-Shu WENO5 value at the face between s2 and s3 from (s0, s1, s2, s3, s4), upwind side first
// (wave_current_refraction.jl:41-55), in difference form: with d_k the first differences and D_k the
// second differences of the stencil, beta_0 = 13/12 D1^2 + (D1/2 + d2)^2, beta_1 = 13/12 D2^2 +
// ((d2+d3)/2)^2, beta_2 = 13/12 D3^2 + (D3/2 - d3)^2 (exactly the reference's indicators), and the
// candidates enter as offsets from s2.
template <typename T>
__device__ __forceinline__ T weno5d(T s0, T s1, T s2, T s3, T s4) {
    const T eps = T(RPL_WENO_EPS);
    const T d1 = s1 - s0, d2 = s2 - s1, d3 = s3 - s2, d4 = s4 - s3;
    const T D1 = d2 - d1, D2 = d3 - d2, D3 = d4 - d3;
    const T g0 = fma(T(0.5), D1, d2);
    const T g1 = T(0.5) * (d2 + d3);
    const T g2 = fma(T(0.5), D3, -d3);
    const T t0 = fma(g0, g0, fma(T(13.0 / 12.0) * D1, D1, eps));
    const T t1 = fma(g1, g1, fma(T(13.0 / 12.0) * D2, D2, eps));
    const T t2 = fma(g2, g2, fma(T(13.0 / 12.0) * D3, D3, eps));
    const T r0 = rcp_w(t0), r1 = rcp_w(t1), r2 = rcp_w(t2);
    const T a0 = (T(0.1) * r0) * r0, a1 = (T(0.6) * r1) * r1, a2 = (T(0.3) * r2) * r2;
    const T w0 = fma(T(5.0 / 6.0), d2, T(-1.0 / 3.0) * d1);
    const T w1 = fma(T(1.0 / 3.0), d3, T(1.0 / 6.0) * d2);
    const T w2 = fma(T(2.0 / 3.0), d3, T(-1.0 / 6.0) * d4);
    const T num = fma(a2, w2, fma(a1, w1, a0 * w0));
    const T den = (a0 + a1) + a2;
    return fma(num, rcp_w(den), s2);
}

// Both faces of a cell from its 7-point stencil oriented upwind -> downwind (s3 is the cell):
// lo = value at the upwind face (from s0..s4), hi = value at the downwind face (from s1..s5).
template <typename T>
__device__ __forceinline__ void weno5_pair(T s0, T s1, T s2, T s3, T s4, T s5, T& lo, T& hi) {
    const T eps = T(RPL_WENO_EPS);
    const T d1 = s1 - s0, d2 = s2 - s1, d3 = s3 - s2, d4 = s4 - s3, d5 = s5 - s4;
    const T D1 = d2 - d1, D2 = d3 - d2, D3 = d4 - d3, D4 = d5 - d4;
    const T A1 = fma(T(13.0 / 12.0) * D1, D1, eps), A2 = fma(T(13.0 / 12.0) * D2, D2, eps);
    const T A3 = fma(T(13.0 / 12.0) * D3, D3, eps), A4 = fma(T(13.0 / 12.0) * D4, D4, eps);
    {   // upwind face: stencil s0..s4 (cells centred at s1, s2, s3)
        const T g0 = fma(T(0.5), D1, d2), g1 = T(0.5) * (d2 + d3), g2 = fma(T(0.5), D3, -d3);
        const T r0 = rcp_w(fma(g0, g0, A1)), r1 = rcp_w(fma(g1, g1, A2)), r2 = rcp_w(fma(g2, g2, A3));
        const T a0 = (T(0.1) * r0) * r0, a1 = (T(0.6) * r1) * r1, a2 = (T(0.3) * r2) * r2;
        const T w0 = fma(T(5.0 / 6.0), d2, T(-1.0 / 3.0) * d1);
        const T w1 = fma(T(1.0 / 3.0), d3, T(1.0 / 6.0) * d2);
        const T w2 = fma(T(2.0 / 3.0), d3, T(-1.0 / 6.0) * d4);
        lo = fma(fma(a2, w2, fma(a1, w1, a0 * w0)), rcp_w((a0 + a1) + a2), s2);
    }
    {   // downwind face: stencil s1..s5 (cells centred at s2, s3, s4)
        const T g0 = fma(T(0.5), D2, d3), g1 = T(0.5) * (d3 + d4), g2 = fma(T(0.5), D4, -d4);
        const T r0 = rcp_w(fma(g0, g0, A2)), r1 = rcp_w(fma(g1, g1, A3)), r2 = rcp_w(fma(g2, g2, A4));
        const T a0 = (T(0.1) * r0) * r0, a1 = (T(0.6) * r1) * r1, a2 = (T(0.3) * r2) * r2;
        const T w0 = fma(T(5.0 / 6.0), d3, T(-1.0 / 3.0) * d2);
        const T w1 = fma(T(1.0 / 3.0), d4, T(1.0 / 6.0) * d3);
        const T w2 = fma(T(2.0 / 3.0), d4, T(-1.0 / 6.0) * d5);
        hi = fma(fma(a2, w2, fma(a1, w1, a0 * w0)), rcp_w((a0 + a1) + a2), s3);
    }
}

// Flux difference u*(N_{+1/2} - N_{-1/2}) of a periodic direction from the 7-point stencil
// (m3 .. p3 around the cell), upwinded by the sign of u (wave_current_refraction.jl:104-123).
template <typename T>
__device__ __forceinline__ T flux_diff(T m3, T m2, T m1, T c, T p1, T p2, T p3, T u) {
    const bool pos = u >= T(0);
    T lo, hi;
    if (pos) weno5_pair(m3, m2, m1, c, p1, p2, lo, hi);      // lo = N(-1/2), hi = N(+1/2)
    else weno5_pair(p3, p2, p1, c, m1, m2, lo, hi);          // lo = N(+1/2), hi = N(-1/2)
    return pos ? u * (hi - lo) : u * (lo - hi);
}

struct Coef {
    double Ux, Uy, Uxx, Uxy, Uyx, Uyy, cg, kap;
};

__device__ __forceinline__ Coef load_coef(const double* __restrict__ rec) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(rec));
    const double2 b = __ldg(reinterpret_cast<const double2*>(rec) + 1);
    const double2 c = __ldg(reinterpret_cast<const double2*>(rec) + 2);
    const double2 d = __ldg(reinterpret_cast<const double2*>(rec) + 3);
    return Coef{a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y};
}

// Velocities of one cell-bin. FP64 keeps the reference's evaluation order
// (wave_current_refraction.jl:94-98); FP32 uses the same products regrouped.
template <typename T>
__device__ __forceinline__ void velocities(const Coef& q, double cph, double sph, double cgx, double cgy,
                                           bool per_cell, bool refract, T& ux, T& uy, T& ck, T& cp) {
    const double gx = per_cell ? q.cg * cgx : cgx;
    const double gy = per_cell ? q.cg * cgy : cgy;
    if (!refract) {
        ux = T(gx);
        uy = T(gy);
        ck = cp = T(0);
        return;
    }
    if constexpr (std::is_same<T, double>::value) {
        ck = -q.kap * (cph * cph * q.Uxx + cph * sph * (q.Uyx + q.Uxy) + sph * sph * q.Uyy);
        cp = cph * sph * (q.Uxx - q.Uyy) + sph * sph * q.Uyx - cph * cph * q.Uxy;
        ux = gx + q.Ux;
        uy = gy + q.Uy;
    } else {
        const float c = (float)cph, s = (float)sph, k = (float)q.kap;
        const float Uxx = (float)q.Uxx, Uxy = (float)q.Uxy, Uyx = (float)q.Uyx, Uyy = (float)q.Uyy;
        ck = -k * (c * c * Uxx + c * s * (Uyx + Uxy) + s * s * Uyy);
        cp = c * s * (Uxx - Uyy) + s * s * Uyx - c * c * Uxy;
        ux = (float)gx + (float)q.Ux;
        uy = (float)gy + (float)q.Uy;
    }
}

// FP32 copy of a coefficient record, made once per ring so the per-cell-bin work stays in FP32.
struct CoefF {
    float k, Uxx, Uxy, Uyx, Uyy, Ux, Uy, cg;
};

__device__ __forceinline__ CoefF to_f32(const Coef& q) {
    return CoefF{(float)q.kap, (float)q.Uxx, (float)q.Uxy, (float)q.Uyx, (float)q.Uyy,
                 (float)q.Ux,  (float)q.Uy,  (float)q.cg};
}

// FP32 velocities from the FP32 direction and group-velocity tables (same expression order).
__device__ __forceinline__ void velocities_f32(const CoefF& q, float4 tg, float2 g, bool per_cell, bool refract,
                                               float& ux, float& uy, float& ck, float& cp) {
    const float gx = per_cell ? q.cg * g.x : g.x;
    const float gy = per_cell ? q.cg * g.y : g.y;
    if (!refract) {
        ux = gx;
        uy = gy;
        ck = cp = 0.0f;
        return;
    }
    ck = -q.k * (tg.x * q.Uxx + tg.y * (q.Uyx + q.Uxy) + tg.z * q.Uyy);
    cp = tg.y * (q.Uxx - q.Uyy) + tg.z * q.Uyx - tg.x * q.Uxy;
    ux = gx + q.Ux;
    uy = gy + q.Uy;
}

__device__ __forceinline__ int wrapi(int i, int N) { return i < 0 ? i + N : (i >= N ? i - N : i); }

// Stage epilogue: clamp, combine with N0, error word (time_step.jl:67-74,98-105).
template <typename T>
__device__ __forceinline__ T stage_out(const StageParams& p, T a, T G, T n0) {
    const T st = relu(a + T(p.dt) * G);
    return p.stage == 1 ? st : relu(T(p.a) * n0 + T(p.b) * st);
}

template <typename T, int SEG, bool REFRACT, bool TENDENCY>
__global__ void __launch_bounds__(BLOCK) column_kernel(const T* __restrict__ Nin, const T* N0, T* Nout,
                                                       double* __restrict__ Gout, StageParams p) {
    constexpr int CPW = 32 / SEG;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int m = lane & (SEG - 1);
    const int base = lane - m;
    const int Nx = (int)p.Nx, Ny = (int)p.Ny, Nk = (int)p.Nk, Np = (int)p.Np;
    const int64_t P = (int64_t)Nx * Ny, Pr = (int64_t)Nx * (p.j_hi - p.j_lo);  // Pr: cells of the updated rows
    const int64_t col = ((int64_t)blockIdx.x * (BLOCK / 32) + warp) * CPW + lane / SEG;
    const bool live = col < Pr && m < Nk;
    const int64_t cc = (col < Pr ? col : Pr - 1) + (int64_t)Nx * p.j_lo;
    const int mm = m < Nk ? m : Nk - 1;
    const int i = (int)(cc % Nx), j = (int)(cc / Nx);
    const Coef q = load_coef(p.coef + 8 * (cc * Nk + mm));
    const CoefF qf = to_f32(q);
    // offsets of the x and y neighbours (periodic)
    const int64_t xs = Nk, ys = (int64_t)Nx * Nk;
    const int64_t xo1 = (wrapi(i + 1, Nx) - i) * xs, xo2 = (wrapi(i + 2, Nx) - i) * xs, xo3 = (wrapi(i + 3, Nx) - i) * xs;
    const int64_t xn1 = (wrapi(i - 1, Nx) - i) * xs, xn2 = (wrapi(i - 2, Nx) - i) * xs, xn3 = (wrapi(i - 3, Nx) - i) * xs;
    const int64_t yo1 = (wrapi(j + 1, Ny) - j) * ys, yo2 = (wrapi(j + 2, Ny) - j) * ys, yo3 = (wrapi(j + 3, Ny) - j) * ys;
    const int64_t yn1 = (wrapi(j - 1, Ny) - j) * ys, yn2 = (wrapi(j - 2, Ny) - j) * ys, yn3 = (wrapi(j - 3, Ny) - j) * ys;
    const int64_t slice = P * Nk;
    const int64_t home = cc * Nk + mm;  // offset within a slice
    // phi window: bins n-3 .. n+3 of this lane's (i,j,m); refraction needs Np >= 3, so one wrap suffices
    T w0 = T(0), w1 = T(0), w2 = T(0), w3 = T(0), w4 = T(0), w5 = T(0), w6 = T(0);
    if constexpr (REFRACT) {
        w0 = Nin[home + slice * wrapi(-3, Np)];
        w1 = Nin[home + slice * wrapi(-2, Np)];
        w2 = Nin[home + slice * wrapi(-1, Np)];
        w3 = Nin[home];
        w4 = Nin[home + slice * wrapi(1, Np)];
        w5 = Nin[home + slice * wrapi(2, Np)];
        w6 = Nin[home + slice * wrapi(3, Np)];
    }
    const T dx_inv = T(p.dx_inv), dy_inv = T(p.dy_inv), dk_inv = T(p.dk_inv), dp_inv = T(p.dp_inv);
    const bool hp = (m - 2 >= 0) && (m + 3 <= Nk - 1);   // kappa + face has its WENO stencil
    const bool hm = (m - 3 >= 0) && (m + 2 <= Nk - 1);   // kappa - face
    T prevF = T(0);
    bool prevPos = false, havePrev = false;
    for (int n = 0; n < Np; ++n) {
        const int64_t at = home + slice * n;
        T nxt = T(0);
        if constexpr (REFRACT) nxt = Nin[home + slice * ((n + 4) % Np)];  // next window entry
        else w3 = Nin[at];
        const T c0 = w3;
        T ux, uy, ck, cp;
        if constexpr (std::is_same<T, float>::value) {
            velocities_f32(qf, __ldg(p.trig32 + n), __ldg(p.cg32 + mm + Nk * n), p.cg_per_cell, REFRACT, ux, uy,
                           ck, cp);
        } else {
            const double cph = __ldg(p.cosp + n), sph = __ldg(p.sinp + n);
            const double cgx = __ldg(p.cg_x + mm + Nk * n), cgy = __ldg(p.cg_y + mm + Nk * n);
            velocities<T>(q, cph, sph, cgx, cgy, p.cg_per_cell, REFRACT, ux, uy, ck, cp);
        }
        // x and y
        const T* row = Nin + at;
        const T fx = flux_diff(row[xn3], row[xn2], row[xn1], c0, row[xo1], row[xo2], row[xo3], ux) * dx_inv;
        const T fy = flux_diff(row[yn3], row[yn2], row[yn1], c0, row[yo1], row[yo2], row[yo3], uy) * dy_inv;
        T G;
        if constexpr (REFRACT) {
            // kappa: neighbours from the lanes of this segment, clamped at the ends
            const T km3 = __shfl_sync(FULL, c0, base + max(m - 3, 0));
            const T km2 = __shfl_sync(FULL, c0, base + max(m - 2, 0));
            const T km1 = __shfl_sync(FULL, c0, base + max(m - 1, 0));
            const T kp1 = __shfl_sync(FULL, c0, base + min(m + 1, Nk - 1));
            const T kp2 = __shfl_sync(FULL, c0, base + min(m + 2, Nk - 1));
            const T kp3 = __shfl_sync(FULL, c0, base + min(m + 3, Nk - 1));
            const bool pk = ck >= T(0);
            T Fkp;
            {
                const T w = pk ? weno5d(km2, km1, c0, kp1, kp2) : weno5d(kp3, kp2, kp1, c0, km1);
                Fkp = hp ? w : (pk ? c0 : kp1);
            }
            const T upF = __shfl_up_sync(FULL, Fkp, 1, SEG);
            const bool upPos = __shfl_up_sync(FULL, (int)pk, 1, SEG) != 0;
            T Fkm = upF;
            if (m >= 1 && upPos != pk) {
                const T w = pk ? weno5d(km3, km2, km1, c0, kp1) : weno5d(kp2, kp1, c0, km1, km2);
                Fkm = hm ? w : (pk ? km1 : c0);
            }
            const T fkp = (m == Nk - 1) ? T(0) : ck * Fkp;
            const T fkm = (m == 0) ? T(0) : ck * Fkm;
            const T fk = (fkp - fkm) * dk_inv;
            // phi: window
            const bool pp = cp >= T(0);
            const T Fpp = pp ? weno5d(w1, w2, w3, w4, w5) : weno5d(w6, w5, w4, w3, w2);
            T Fpm = prevF;
            if (!havePrev || prevPos != pp) Fpm = pp ? weno5d(w0, w1, w2, w3, w4) : weno5d(w5, w4, w3, w2, w1);
            prevF = Fpp;
            prevPos = pp;
            havePrev = true;
            const T fp = cp * (Fpp - Fpm) * dp_inv;
            G = -(fx + fy + fk + fp);
        } else {
            G = -(fx + fy);
        }
        if (p.has_wind || p.has_diss) G = G + T(source_term(p, cc, mm, n, (double)c0));
        if (p.lin_rates) G = fma(static_cast<const T*>(p.lin_rates)[at], c0, G);
        if constexpr (TENDENCY) {
            if (live) Gout[at] = (double)G;
        } else {
            const T out = stage_out(p, c0, G, p.stage == 1 ? T(0) : N0[at]);
            if (live) {
                if (!isfinite(out)) atomicOr(p.err, 1u);
                Nout[at] = out;
            }
        }
        w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6; w6 = nxt;
    }
}

// One thread per cell-bin, for any Nk.
template <typename T, bool REFRACT, bool TENDENCY>
__global__ void __launch_bounds__(BLOCK) generic_kernel(const T* __restrict__ Nin, const T* N0, T* Nout,
                                                        double* __restrict__ Gout, StageParams p) {
    const int64_t t = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
    const int Nx = (int)p.Nx, Ny = (int)p.Ny, Nk = (int)p.Nk, Np = (int)p.Np;
    const int64_t P = (int64_t)Nx * Ny, slice = P * Nk;
    if (t >= slice * Np) return;
    const int m = (int)(t % Nk);
    const int64_t cn = t / Nk;
    const int64_t c = cn % P;
    const int n = (int)(cn / P);
    const int i = (int)(c % Nx), j = (int)(c / Nx);
    if (j < p.j_lo || j >= p.j_hi) return;
    const Coef q = load_coef(p.coef + 8 * (c * Nk + m));
    const double cph = p.cosp[n], sph = p.sinp[n];
    T ux, uy, ck, cp;
    velocities<T>(q, cph, sph, p.cg_x[m + Nk * n], p.cg_y[m + Nk * n], p.cg_per_cell, REFRACT, ux, uy, ck, cp);
    const T* row = Nin + (int64_t)n * slice;
    auto X = [&](int ii) { return row[((int64_t)j * Nx + wrapi(ii, Nx)) * Nk + m]; };
    auto Y = [&](int jj) { return row[((int64_t)wrapi(jj, Ny) * Nx + i) * Nk + m]; };
    const T c0 = row[c * Nk + m];
    const T fx = flux_diff(X(i - 3), X(i - 2), X(i - 1), c0, X(i + 1), X(i + 2), X(i + 3), ux) * T(p.dx_inv);
    const T fy = flux_diff(Y(j - 3), Y(j - 2), Y(j - 1), c0, Y(j + 1), Y(j + 2), Y(j + 3), uy) * T(p.dy_inv);
    T G;
    if constexpr (REFRACT) {
        auto K = [&](int mk) { return row[c * Nk + clampi(mk, Nk)]; };
        auto F = [&](int nk) { return Nin[(int64_t)wrapi(nk, Np) * slice + c * Nk + m]; };
        const bool hp = (m - 2 >= 0) && (m + 3 <= Nk - 1), hm = (m - 3 >= 0) && (m + 2 <= Nk - 1);
        const bool pk = ck >= T(0);
        const T Fkp = hp ? (pk ? weno5d(K(m - 2), K(m - 1), c0, K(m + 1), K(m + 2))
                               : weno5d(K(m + 3), K(m + 2), K(m + 1), c0, K(m - 1)))
                         : (pk ? c0 : K(m + 1));
        const T Fkm = hm ? (pk ? weno5d(K(m - 3), K(m - 2), K(m - 1), c0, K(m + 1))
                               : weno5d(K(m + 2), K(m + 1), c0, K(m - 1), K(m - 2)))
                         : (pk ? K(m - 1) : c0);
        const T fkp = (m == Nk - 1) ? T(0) : ck * Fkp;
        const T fkm = (m == 0) ? T(0) : ck * Fkm;
        const T fk = (fkp - fkm) * T(p.dk_inv);
        const T fp = flux_diff(F(n - 3), F(n - 2), F(n - 1), c0, F(n + 1), F(n + 2), F(n + 3), cp) * T(p.dp_inv);
        G = -(fx + fy + fk + fp);
    } else {
        G = -(fx + fy);
    }
    if (p.has_wind || p.has_diss) G = G + T(source_term(p, c, m, n, (double)c0));
    if (p.lin_rates) G = fma(static_cast<const T*>(p.lin_rates)[t], c0, G);
    if constexpr (TENDENCY) {
        Gout[t] = (double)G;
    } else {
        const T out = stage_out(p, c0, G, p.stage == 1 ? T(0) : N0[t]);
        if (!isfinite(out)) atomicOr(p.err, 1u);
        Nout[t] = out;
    }
}

// No transport (horizontal_advection = nothing, no currents): G = sources only
// (tendencies.jl:230-246 with transport_tendency(::Nothing) = 0). Touches no neighbour.
template <typename T, bool TENDENCY>
__global__ void __launch_bounds__(BLOCK) source_only_kernel(const T* __restrict__ Nin, const T* N0, T* Nout,
                                                            double* __restrict__ Gout, StageParams p) {
    const int64_t t = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
    const int64_t P = p.Nx * p.Ny, slice = P * p.Nk;
    if (t >= slice * p.Np) return;
    const int m = (int)(t % p.Nk);
    const int64_t cn = t / p.Nk;
    const int64_t jr = (cn % P) / p.Nx;
    if (jr < p.j_lo || jr >= p.j_hi) return;
    const T a = Nin[t];
    T G = T(0);
    if (p.has_wind || p.has_diss) G = T(source_term(p, cn % P, m, (int)(cn / P), (double)a));
    if (p.lin_rates) G = fma(static_cast<const T*>(p.lin_rates)[t], a, G);
    if constexpr (TENDENCY) {
        Gout[t] = (double)G;
    } else {
        const T out = stage_out(p, a, G, p.stage == 1 ? T(0) : N0[t]);
        if (!isfinite(out)) atomicOr(p.err, 1u);
        Nout[t] = out;
    }
}

template <typename T, bool TEND>
cudaError_t launch_impl(const Handle& h, const StageParams& p, const void* Nin, const void* N0, void* Nout, double* G,
                        cudaStream_t s) {
    const int64_t Nk = h.desc.Nk;
    const bool refract = p.transport == RPL_TRANSPORT_REFRACTION;
    const T* in = (const T*)Nin;
    const T* n0 = (const T*)N0;
    T* out = (T*)Nout;
    if (p.transport == RPL_TRANSPORT_NONE) {
        const dim3 grid((unsigned)((h.units + BLOCK - 1) / BLOCK));
        source_only_kernel<T, TEND><<<grid, BLOCK, 0, s>>>(in, n0, out, G, p);
    } else if (Nk <= 32) {
        const int seg = Nk <= 4 ? 4 : Nk <= 8 ? 8 : Nk <= 16 ? 16 : 32;
        const int64_t cols_per_block = (BLOCK / 32) * (32 / seg);
        const int64_t Pr = h.desc.Nx * (p.j_hi - p.j_lo);
        const dim3 grid((unsigned)((Pr + cols_per_block - 1) / cols_per_block));
#define RPL_COL(SEGV)                                                                                        \
    if (seg == SEGV) {                                                                                       \
        if (refract) column_kernel<T, SEGV, true, TEND><<<grid, BLOCK, 0, s>>>(in, n0, out, G, p);          \
        else column_kernel<T, SEGV, false, TEND><<<grid, BLOCK, 0, s>>>(in, n0, out, G, p);                 \
    }
        RPL_COL(4) RPL_COL(8) RPL_COL(16) RPL_COL(32)
#undef RPL_COL
    } else {
        const dim3 grid((unsigned)((h.units + BLOCK - 1) / BLOCK));
        if (refract) generic_kernel<T, true, TEND><<<grid, BLOCK, 0, s>>>(in, n0, out, G, p);
        else generic_kernel<T, false, TEND><<<grid, BLOCK, 0, s>>>(in, n0, out, G, p);
    }
    return cudaGetLastError();
}

}  // namespace

StageParams make_params(const Handle& h, double dt, int stage) {
    StageParams p{};
    const rpl_desc& d = h.desc;
    p.Nx = d.Nx; p.Ny = d.Ny; p.Nk = d.Nk; p.Np = d.Np;
    p.dx_inv = 1.0 / d.dx;
    p.dy_inv = 1.0 / d.dy;
    p.dk_inv = 1.0 / (h.kappa_faces[1] - h.kappa_faces[0]);
    p.dp_inv = 1.0 / (h.phi_faces[1] - h.phi_faces[0]);
    p.dt = dt;
    p.stage = stage;
    p.a = stage == 2 ? 0.75 : (stage == 3 ? 1.0 / 3.0 : 0.0);
    p.b = stage == 2 ? 0.25 : (stage == 3 ? 2.0 / 3.0 : 1.0);
    p.transport = d.transport;
    p.cg_per_cell = h.d_cgmag != nullptr;
    p.kappa = h.d_kappa; p.phi = h.d_phi; p.weights = h.d_weights;
    p.cosp = h.d_cos; p.sinp = h.d_sin;
    p.cg_x = h.d_cgx; p.cg_y = h.d_cgy; p.cg_mag = h.d_cgmag;
    p.coef = h.d_coef;
    p.trig32 = reinterpret_cast<const float4*>(h.d_tab32);
    p.cg32 = reinterpret_cast<const float2*>(h.d_tab32 + 4 * d.Np);
    p.cs32 = reinterpret_cast<const float2*>(h.d_tab32 + 4 * d.Np + 2 * d.Nk * d.Np);
    p.w32 = h.d_tab32 + 6 * d.Np + 2 * d.Nk * d.Np;
    p.cell32 = h.d_cell32;
    p.bin32 = h.d_bin32;
    p.learned = h.learned != nullptr;
    p.lrate = h.d_lr;
    p.lflag = h.d_lflag;
    p.lscale = h.learned ? mlp_desc(h.learned).target_scale : 0.0f;
    p.has_wind = h.has_sources && h.src.wind_kind != RPL_WIND_NONE;
    p.stress_cap = h.has_sources && h.src.stress_cap;
    p.has_diss = h.has_sources && h.src.has_dissipation;
    if (h.d_wind) {
        const int64_t c2 = d.Nx * d.Ny;
        p.wind_U10 = h.d_wind; p.wind_theta = h.d_wind + c2; p.wind_ustar = h.d_wind + 2 * c2;
        p.stress_factor = h.d_wind + 3 * c2;
    }
    p.rho_ratio = h.src.rho_air / h.src.rho_water;
    p.beta_max = h.src.beta_max; p.z_alpha = h.src.z_alpha; p.p_in = h.src.p_in;
    p.alpha0 = h.src.alpha0; p.von_karman = h.src.von_karman; p.wind_g = h.src.wind_gravity;
    p.C_ds = h.src.C_ds; p.B_r = h.src.B_r; p.ds_p = h.src.ds_p; p.sigma_power = h.src.sigma_power;
    p.ds_g = h.src.ds_gravity;
    p.wind_K32 = p.has_wind ? (float)(p.rho_ratio * (p.beta_max / (p.von_karman * p.von_karman))) : 0.0f;
    p.von_karman32 = (float)p.von_karman;
    p.z_alpha32 = (float)p.z_alpha;
    p.err = h.d_err;
    p.lin_rates = h.n_terms ? h.d_lin_rates : nullptr;
    p.j_lo = 0;
    p.j_hi = d.Ny;
    return p;
}

cudaError_t launch_stage(const Handle& h, const StageParams& p, const void* Nin, const void* N0, void* Nout,
                         cudaStream_t s) {
    if (h.precision == RPL_FP64) return launch_impl<double, false>(h, p, Nin, N0, Nout, nullptr, s);
    // the tile kernel takes the SourceTermSet rates alone, not together with the bundle or the network
    const bool mixed = p.lin_rates && (p.has_wind || p.has_diss || p.learned);
    if (tile32_supported(h) && !h.force_column_kernel && !mixed) return launch_tile32(h, p, Nin, N0, Nout, s);
    return launch_impl<float, false>(h, p, Nin, N0, Nout, nullptr, s);
}

cudaError_t launch_tendency(const Handle& h, const StageParams& p, const void* Nin, double* G, cudaStream_t s) {
    if (h.precision == RPL_FP64) return launch_impl<double, true>(h, p, Nin, nullptr, nullptr, G, s);
    return launch_impl<float, true>(h, p, Nin, nullptr, nullptr, G, s);
}

}  // namespace rpl
