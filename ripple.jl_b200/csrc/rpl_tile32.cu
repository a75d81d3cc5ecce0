// rpl_tile32.cu -- the FP32 stage kernel of the precision form for even Nk <= 32 with Nk % 4 == 0.
//
// Same arithmetic as rpl_stage.cu (wave_current_refraction.jl:74-151, intrinsic_transport.jl:14-68,
// time_step.jl:67-105), organised for B200:
//  * a CTA owns a TX x TY tile of horizontal cells and walks the phi ring n = 0 .. Np-1; the plane of
//    bin n for the tile plus its 3-cell cross halo is staged in shared memory with cp.async, two
//    planes ahead (three buffers), so x/y/kappa stencils are shared-memory reads with immediate offsets;
//  * L = Nk_pad/2 lanes per cell, each lane holding two adjacent kappa bins as a float2, so the WENO
//    arithmetic issues as packed FP32 pairs (FFMA2/FADD2/FMUL2, sm_100);
//  * the phi stencil comes from a 7-deep register window of the lane's own pair; the + phi face of
//    step n is the - face of step n+1; the face between the lane's two kappa bins and the face above
//    them are reconstructed together, the face below comes from the lane underneath (shuffle);
//  * reciprocals: rcp.approx of t'^2 per indicator (finite for 4(eps+beta) <= 1.8e19, i.e. |N| up to
//    ~2e9) and of the weight sum: four MUFU ops per face and element;
//  * upwinding: where a warp's velocities share a sign the stencils are read in upwind order directly,
//    per-element selects otherwise; 256-thread CTAs, two per SM (the kernel is latency-bound: while one
//    CTA waits at its per-plane barrier the other issues).
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "rpl_device.cuh"
#include "rpl_internal.h"
#include "rpl_src32.cuh"
#include "rpl_weno32.cuh"

namespace rpl {

namespace {

using namespace w32;
constexpr int NB = 3;                     // plane buffers

// u * (N(+1/2) - N(-1/2)) for a periodic direction from m3..p3, upwinded per element by sign(u)
// (per-element selects of the stencil: the general case).
__device__ __forceinline__ float2 flux2_sel(float2 m3, float2 m2, float2 m1, float2 c, float2 p1, float2 p2, float2 p3,
                                            float2 u) {
    const bool px = u.x >= 0.0f, py = u.y >= 0.0f;
    float2 lo, hi;
    weno5_pair2(sel2(px, py, m3, p3), sel2(px, py, m2, p2), sel2(px, py, m1, p1), c, sel2(px, py, p1, m1),
                sel2(px, py, p2, m2), lo, hi);
    const float2 diff = sub2(hi, lo);
    return mul2(u, make_float2(px ? diff.x : -diff.x, py ? diff.y : -diff.y));
}

// The x and y fluxes of the cell (u (N(+1/2) - N(-1/2)) each, before the 1/spacing). When the x velocities
// of every lane of the warp share one sign and so do the y velocities (the common case: |c_g| exceeds the
// current almost everywhere), one branch-free body per sign pair reads the stencils in upwind order with
// no per-element selects and lets the two directions' arithmetic interleave; otherwise the per-element
// form. Both give the reference's upwinding (wave_current_refraction.jl:104-123) bit for bit.
template <bool XP, bool YP, class VF>
__device__ __forceinline__ void flux_xy_u(VF V, int RW, float2 c, float2 ux, float2 uy, float2& fx, float2& fy) {
    float2 xl, xh, yl, yh;
    if constexpr (XP) weno5_pair2(V(-3), V(-2), V(-1), c, V(1), V(2), xl, xh);
    else weno5_pair2(V(3), V(2), V(1), c, V(-1), V(-2), xl, xh);
    if constexpr (YP) weno5_pair2(V(-3 * RW), V(-2 * RW), V(-RW), c, V(RW), V(2 * RW), yl, yh);
    else weno5_pair2(V(3 * RW), V(2 * RW), V(RW), c, V(-RW), V(-2 * RW), yl, yh);
    fx = XP ? mul2(ux, sub2(xh, xl)) : mul2(ux, sub2(xl, xh));
    fy = YP ? mul2(uy, sub2(yh, yl)) : mul2(uy, sub2(yl, yh));
}

template <class VF>
__device__ __forceinline__ void flux_xy(VF V, int RW, float2 c, float2 ux, float2 uy, float2& fx, float2& fy) {
    const bool xp = __all_sync(FULL, ux.x >= 0.0f && ux.y >= 0.0f), xn = __all_sync(FULL, ux.x < 0.0f && ux.y < 0.0f);
    const bool yp = __all_sync(FULL, uy.x >= 0.0f && uy.y >= 0.0f), yn = __all_sync(FULL, uy.x < 0.0f && uy.y < 0.0f);
    if (xp && yp) flux_xy_u<true, true>(V, RW, c, ux, uy, fx, fy);
    else if (xp && yn) flux_xy_u<true, false>(V, RW, c, ux, uy, fx, fy);
    else if (xn && yp) flux_xy_u<false, true>(V, RW, c, ux, uy, fx, fy);
    else if (xn && yn) flux_xy_u<false, false>(V, RW, c, ux, uy, fx, fy);
    else {
        fx = flux2_sel(V(-3), V(-2), V(-1), c, V(1), V(2), V(3), ux);
        fy = flux2_sel(V(-3 * RW), V(-2 * RW), V(-RW), c, V(RW), V(2 * RW), V(3 * RW), uy);
    }
}

// One CTA's work: stage update of the TX x TY tile `tile` (row-major over the tiles of the grid) for all
// bins, with TX*TY*L threads. P is TileArgs seen through the kernel parameter bank (single-model kernel)
// or a shared-memory copy (ensemble kernel).
// SRC: 0 no sources, 1 the plain FP32 sources, 2 the learned source with per-cell plain fallback,
// 3 the per-cell-bin rates of SourceTermSet terms (rpl_terms.cu).
template <int L, int TX, int TY, bool REFRACT, int SRC>
__device__ __forceinline__ void tile_body(const TileArgs& p, int tile, float* smem) {
    constexpr int RW = TX + 6, RH = TY + 6;   // staged rectangle (only its cross is loaded)
    constexpr int KP = 2 * L;                 // kappa slots per staged column
    constexpr int THREADS = TX * TY * L;
    constexpr int CROSS = RW * TY + 6 * TX;   // staged columns per plane
    const float* __restrict__ Nin = p.Nin;
    const float* N0 = p.N0;
    float* Nout = p.Nout;
    const int Nx = p.Nx, Ny = p.Ny, Nk = p.Nk, Np = p.Np;
    const int64_t slice = (int64_t)Nx * Ny * Nk;
    const int tiles_x = (Nx + TX - 1) / TX;
    const int i0 = (tile % tiles_x) * TX, j0 = p.j_lo + (tile / tiles_x) * TY;  // tiles over rows [j_lo, j_hi)
    const int tid = threadIdx.x;
    const int l = tid % L;                    // lane within the cell
    const int cell = tid / L;                 // 0 .. TX*TY-1
    const int cx = cell % TX, cy = cell / TX;
    const int i = i0 + cx, j = j0 + cy;
    const bool live_cell = i < Nx && j < p.j_hi;
    const int ic = i < Nx ? i : Nx - 1, jc = j < p.j_hi ? j : p.j_hi - 1;
    const int m0 = 2 * l;                      // this lane's kappa pair (m0, m0+1)
    const bool live = live_cell && m0 < Nk;
    const int mc = m0 < Nk ? m0 : Nk - 2;
    const int64_t home = ((int64_t)jc * Nx + ic) * Nk + mc;  // offset within a slice

    // cp.async chunk descriptors (16-byte chunks of the cross columns), reused for every plane
    const int KC = Nk / 4;
    const int nchunks = CROSS * KC;
    constexpr int MAXC = (CROSS * (KP / 4) + THREADS - 1) / THREADS;
    int64_t goff[MAXC];
    int soff[MAXC];
#pragma unroll
    for (int k = 0; k < MAXC; ++k) {
        const int q = tid + k * THREADS;
        goff[k] = -1;
        soff[k] = 0;
        if (q < nchunks) {
            const int col = q / KC, part = q % KC;
            int dx, dy;
            if (col < RW * TY) {
                dy = col / RW;
                dx = col % RW - 3;
            } else {
                const int r = col - RW * TY, yi = r / TX;
                dx = r % TX;
                dy = yi < 3 ? yi - 3 : TY + yi - 3;
            }
            int gi = i0 + dx, gj = j0 + dy;
            gi = gi < 0 ? gi + Nx : (gi >= Nx ? gi - Nx : gi);
            gj = gj < 0 ? gj + Ny : (gj >= Ny ? gj - Ny : gj);
            gi = gi < 0 ? 0 : (gi >= Nx ? Nx - 1 : gi);  // tiles wider than the grid
            gj = gj < 0 ? 0 : (gj >= Ny ? Ny - 1 : gj);
            goff[k] = ((int64_t)gj * Nx + gi) * Nk + 4 * part;
            soff[k] = ((dy + 3) * RW + (dx + 3)) * KP + 4 * part;
        }
    }
    const int plane_floats = RW * RH * KP;
    auto issue = [&](int n) {
        if (n < Np) {
            float* buf = smem + (n % NB) * plane_floats;
            const float* src = Nin + slice * n;
#pragma unroll
            for (int k = 0; k < MAXC; ++k)
                if (goff[k] >= 0) {
                    const unsigned sa = (unsigned)__cvta_generic_to_shared(buf + soff[k]);
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(src + goff[k]));
                }
        }
        asm volatile("cp.async.commit_group;");
    };
    issue(0);
    issue(1);

    // coefficient records of the pair (FP64 -> FP32 once per ring)
    const double* rec0 = p.coef + 8 * (((int64_t)jc * Nx + ic) * Nk + mc);
    const double* rec1 = rec0 + 8;
    float2 kap, Uxx, Uxy, Uyx, Uyy, Ux, Uy, cgm;
    {
        kap = make_float2((float)rec0[7], (float)rec1[7]);
        Ux = make_float2((float)rec0[0], (float)rec1[0]);
        Uy = make_float2((float)rec0[1], (float)rec1[1]);
        Uxx = make_float2((float)rec0[2], (float)rec1[2]);
        Uxy = make_float2((float)rec0[3], (float)rec1[3]);
        Uyx = make_float2((float)rec0[4], (float)rec1[4]);
        Uyy = make_float2((float)rec0[5], (float)rec1[5]);
        cgm = make_float2((float)rec0[6], (float)rec1[6]);
    }
    const float2* own = reinterpret_cast<const float2*>(Nin + home);  // stride per bin: slice/2 float2
    const int64_t s2 = slice / 2;
    float2 w0 = f2(0.f), w1 = f2(0.f), w2 = f2(0.f), w3 = f2(0.f), w4 = f2(0.f), w5 = f2(0.f), w6 = f2(0.f);
    if constexpr (REFRACT) {
        auto wr = [&](int n) { return n < 0 ? n + Np : (n >= Np ? n - Np : n); };
        w0 = own[s2 * wr(-3)]; w1 = own[s2 * wr(-2)]; w2 = own[s2 * wr(-1)]; w3 = own[0];
        w4 = own[s2 * wr(1)]; w5 = own[s2 * wr(2)]; w6 = own[s2 * wr(3)];
    }
    const float dx_inv = p.dx_inv, dy_inv = p.dy_inv, dk_inv = p.dk_inv, dp_inv = p.dp_inv;
    const float dt = p.dt, ca = p.a, cb = p.b;
    // kappa faces: face a between m0|m0+1 and face b between m0+1|m0+2
    const bool ha = (m0 - 2 >= 0) && (m0 + 3 <= Nk - 1);
    const bool hb = (m0 - 1 >= 0) && (m0 + 4 <= Nk - 1);
    const bool hlo = (m0 - 3 >= 0) && (m0 + 2 <= Nk - 1);   // face below m0 (m0-1|m0)
    const int kcm3 = max(m0 - 3, 0), kcm2 = max(m0 - 2, 0), kcm1 = max(m0 - 1, 0);
    const int kcp2 = min(m0 + 2, Nk - 1), kcp3 = min(m0 + 3, Nk - 1), kcp4 = min(m0 + 4, Nk - 1);
    const int ctr = ((cy + 3) * RW + (cx + 3)) * KP;         // this cell's column in a staged plane
    float2 prevF = f2(0.f);
    bool prevx = false, prevy = false, have = false;
    // source constants of this cell and of the lane's two kappa bins
    Cell32 wc{};
    Bin32 wb0{}, wb1{};
    bool plain_src = SRC == 1;
    const float* lrow = nullptr;
    if constexpr (SRC == 1 || SRC == 2) {
        const int64_t cidx = (int64_t)jc * Nx + ic;
        wc = load_cell32(p.cell32 + 8 * cidx);
        wb0 = load_bin32(p.bin32 + 8 * mc);
        wb1 = load_bin32(p.bin32 + 8 * (mc + 1));
        if constexpr (SRC == 2) {
            plain_src = __ldg(p.lflag + cidx) != 0u;
            lrow = p.lrate + cidx * ((int64_t)Nk * Np) + mc;
        }
    }

    for (int n = 0; n < Np; ++n) {
        float2 nxt = f2(0.f);
        if constexpr (REFRACT) nxt = own[s2 * ((n + 4) % Np)];
        const float2 n0v = (p.stage == 1 || !live) ? f2(0.f)
                                                    : *reinterpret_cast<const float2*>(N0 + slice * n + home);
        asm volatile("cp.async.wait_group 1;");
        __syncthreads();
        issue(n + 2);
        const float* pl = smem + (n % NB) * plane_floats + ctr;
        // idle lanes (m0 >= Nk) read the last live pair; their results are never stored
        auto V1 = [&](int dcol) { return *reinterpret_cast<const float2*>(pl + dcol * KP + mc); };
        const float2 c = *reinterpret_cast<const float2*>(pl + mc);
        // velocities (same expression order as the FP64 path)
        const float4 tg = __ldg(p.trig32 + n);
        const float4 g = __ldg(reinterpret_cast<const float4*>(p.cg32 + mc + Nk * n));
        float2 ux = make_float2(g.x, g.z), uy = make_float2(g.y, g.w);
        if (p.cg_per_cell) {
            ux = mul2(cgm, ux);
            uy = mul2(cgm, uy);
        }
        float2 G;
        if constexpr (REFRACT) {
            ux = add2(ux, Ux);
            uy = add2(uy, Uy);
            const float2 ck = mul2(mul2(f2(-1.f), kap),
                                   add2(add2(mul2(f2(tg.x), Uxx), mul2(f2(tg.y), add2(Uyx, Uxy))), mul2(f2(tg.z), Uyy)));
            const float2 cp = sub2(add2(mul2(f2(tg.y), sub2(Uxx, Uyy)), mul2(f2(tg.z), Uyx)), mul2(f2(tg.x), Uxy));
            // x and y
            float2 fx, fy;
            flux_xy(V1, RW, c, ux, uy, fx, fy);
            fx = mul2(fx, f2(dx_inv));
            fy = mul2(fy, f2(dy_inv));
            // kappa: stencil values of this lane's column (clamped like the reference)
            const float km3 = pl[kcm3], km2 = pl[kcm2], km1 = pl[kcm1];
            const float kp2 = pl[kcp2], kp3 = pl[kcp3], kp4 = pl[kcp4];
            const float k0 = c.x, k1 = c.y;
            // face a (m0|m0+1) upwinded by cell m0, face b (m0+1|m0+2) by cell m0+1
            const bool pa = ck.x >= 0.f, pb = ck.y >= 0.f;
            float2 Fab;
            // the kappa velocity's sign depends on the cell and direction only, so a warp's faces are
            // usually all upwinded the same way: stencils in order then, per-element selects otherwise
            if (__all_sync(FULL, pa && pb)) {
                Fab = weno5_2(make_float2(km2, km1), make_float2(km1, k0), make_float2(k0, k1), make_float2(k1, kp2),
                              make_float2(kp2, kp3));
            } else if (__all_sync(FULL, !pa && !pb)) {
                Fab = weno5_2(make_float2(kp3, kp4), make_float2(kp2, kp3), make_float2(k1, kp2), make_float2(k0, k1),
                              make_float2(km1, k0));
            } else {
                const float2 sa0 = make_float2(pa ? km2 : kp3, pb ? km1 : kp4);
                const float2 sa1 = make_float2(pa ? km1 : kp2, pb ? k0 : kp3);
                const float2 sa2 = make_float2(pa ? k0 : k1, pb ? k1 : kp2);
                const float2 sa3 = make_float2(pa ? k1 : k0, pb ? kp2 : k1);
                const float2 sa4 = make_float2(pa ? kp2 : km1, pb ? kp3 : k0);
                Fab = weno5_2(sa0, sa1, sa2, sa3, sa4);
            }
            Fab.x = ha ? Fab.x : (pa ? k0 : k1);
            Fab.y = hb ? Fab.y : (pb ? k1 : kp2);
            // the - face of cell m0+1 is face a: recompute if cell m0+1 upwinds the other way
            float Fam1 = Fab.x;
            if (pa != pb) {
                const float2 t = weno5_2(make_float2(pb ? km2 : kp3, 0.f), make_float2(pb ? km1 : kp2, 0.f),
                                         make_float2(pb ? k0 : k1, 0.f), make_float2(pb ? k1 : k0, 0.f),
                                         make_float2(pb ? kp2 : km1, 0.f));
                Fam1 = ha ? t.x : (pb ? k0 : k1);
            }
            // the - face of cell m0 is face b of the lane below (cell m0-1)
            const float upF = __shfl_up_sync(FULL, Fab.y, 1, L);
            const bool upP = __shfl_up_sync(FULL, (int)pb, 1, L) != 0;
            float Flo = upF;
            if (m0 >= 1 && upP != pa) {
                const float2 t = weno5_2(make_float2(pa ? km3 : kp2, 0.f), make_float2(pa ? km2 : k1, 0.f),
                                         make_float2(pa ? km1 : k0, 0.f), make_float2(pa ? k0 : km1, 0.f),
                                         make_float2(pa ? k1 : km2, 0.f));
                Flo = hlo ? t.x : (pa ? km1 : k0);
            }
            const float fk0 = kflux(m0 == Nk - 1, m0 == 0, ck.x, Fab.x, Flo);
            const float fk1 = kflux(m0 + 1 == Nk - 1, false, ck.y, Fab.y, Fam1);
            const float2 fk = mul2(make_float2(fk0, fk1), f2(dk_inv));
            // phi: window
            const bool qx = cp.x >= 0.f, qy = cp.y >= 0.f;
            float2 Fpp;
            if (__all_sync(FULL, qx && qy)) Fpp = weno5_2(w1, w2, w3, w4, w5);   // same for the phi window
            else if (__all_sync(FULL, !qx && !qy)) Fpp = weno5_2(w6, w5, w4, w3, w2);
            else Fpp = weno5_2(sel2(qx, qy, w1, w6), sel2(qx, qy, w2, w5), sel2(qx, qy, w3, w4),
                               sel2(qx, qy, w4, w3), sel2(qx, qy, w5, w2));
            float2 Fpm = prevF;
            if (!have || prevx != qx || prevy != qy) {
                const float2 t = weno5_2(sel2(qx, qy, w0, w5), sel2(qx, qy, w1, w4), sel2(qx, qy, w2, w3),
                                         sel2(qx, qy, w3, w2), sel2(qx, qy, w4, w1));
                if (!have || prevx != qx) Fpm.x = t.x;
                if (!have || prevy != qy) Fpm.y = t.y;
            }
            prevF = Fpp;
            prevx = qx;
            prevy = qy;
            have = true;
            const float2 fp = mul2(mul2(cp, sub2(Fpp, Fpm)), f2(dp_inv));
            G = mul2(f2(-1.f), add2(add2(add2(fx, fy), fk), fp));
        } else {
            float2 fx, fy;
            flux_xy(V1, RW, c, ux, uy, fx, fy);
            fx = mul2(fx, f2(dx_inv));
            fy = mul2(fy, f2(dy_inv));
            G = mul2(f2(-1.f), add2(fx, fy));
        }
        if constexpr (SRC != 0) {
            if (plain_src) {
                const float2 cs = __ldg(p.cs32 + n);
                G.x += source32(p, wc, wb0, cs.x, cs.y, c.x);
                G.y += source32(p, wc, wb1, cs.x, cs.y, c.y);
            } else if (SRC == 2) {  // learned: N * rate, rate = lscale * sinh(network output of bin (m, n))
                const float2 y = __ldg(reinterpret_cast<const float2*>(lrow + (int64_t)n * Nk));
                G = fma2(mul2(c, f2(p.lscale)), make_float2(sinhf(y.x), sinhf(y.y)), G);
            } else {  // SourceTermSet rates of this stage, state layout
                G = fma2(*reinterpret_cast<const float2*>(p.lin_rates + slice * n + home), c, G);
            }
        }
        // stage update
        float2 st = fma2(f2(dt), G, c);
        st.x = relu(st.x);
        st.y = relu(st.y);
        float2 out = st;
        if (p.stage != 1) {
            out = fma2(f2(ca), n0v, mul2(f2(cb), st));
            out.x = relu(out.x);
            out.y = relu(out.y);
        }
        if (live) {
            if (!isfinite(out.x) || !isfinite(out.y)) atomicOr(p.err, 1u);
            *reinterpret_cast<float2*>(Nout + slice * n + home) = out;
        }
        w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6; w6 = nxt;
    }
    asm volatile("cp.async.wait_group 0;");
}

// Refraction stages of FP32 models run as two kernels with smaller register footprints than the fused
// tile body, so more warps hide the latency of the WENO5 chains (measured on seamount 1024^2 x 32 x 36:
// 12.9 ms per stage against 14.4 ms fused, bit-identical results):
//   xy_kernel (pass A): the tile body's staging of the phi planes and its x and y fluxes; writes
//     S = fx/dx + fy/dy per cell-bin (state layout);
//   kp_kernel (pass B): one thread per (cell, kappa pair) walking the phi ring with its register window,
//     the kappa stencil from the cell's other lanes (warp shuffles, the reference's clamped indices),
//     the kappa and phi fluxes, sources and the stage update: G = -(((S + fk) + fp)), the fused kernel's
//     order of additions.
template <int L, int TX, int TY>
__device__ __forceinline__ void xy_body(const TileArgs& p, int tile, float* smem) {
    float* S = p.sxy;
    constexpr int RW = TX + 6, RH = TY + 6, KP = 2 * L, THREADS = TX * TY * L, CROSS = RW * TY + 6 * TX;
    const float* __restrict__ Nin = p.Nin;
    const int Nx = p.Nx, Ny = p.Ny, Nk = p.Nk, Np = p.Np;
    const int64_t slice = (int64_t)Nx * Ny * Nk;
    const int tiles_x = (Nx + TX - 1) / TX;
    const int i0 = (tile % tiles_x) * TX, j0 = p.j_lo + (tile / tiles_x) * TY;
    const int tid = threadIdx.x, l = tid % L, cell = tid / L, cx = cell % TX, cy = cell / TX;
    const int i = i0 + cx, j = j0 + cy;
    const bool live_cell = i < Nx && j < p.j_hi;
    const int ic = i < Nx ? i : Nx - 1, jc = j < p.j_hi ? j : p.j_hi - 1;
    const int m0 = 2 * l;
    const bool live = live_cell && m0 < Nk;
    const int mc = m0 < Nk ? m0 : Nk - 2;
    const int64_t home = ((int64_t)jc * Nx + ic) * Nk + mc;
    const int KC = Nk / 4, nchunks = CROSS * KC;
    constexpr int MAXC = (CROSS * (KP / 4) + THREADS - 1) / THREADS;
    int64_t goff[MAXC];
    int soff[MAXC];
#pragma unroll
    for (int k = 0; k < MAXC; ++k) {
        const int q = tid + k * THREADS;
        goff[k] = -1;
        soff[k] = 0;
        if (q < nchunks) {
            const int col = q / KC, part = q % KC;
            int dx, dy;
            if (col < RW * TY) { dy = col / RW; dx = col % RW - 3; }
            else { const int r = col - RW * TY, yi = r / TX; dx = r % TX; dy = yi < 3 ? yi - 3 : TY + yi - 3; }
            int gi = i0 + dx, gj = j0 + dy;
            gi = gi < 0 ? gi + Nx : (gi >= Nx ? gi - Nx : gi);
            gj = gj < 0 ? gj + Ny : (gj >= Ny ? gj - Ny : gj);
            gi = gi < 0 ? 0 : (gi >= Nx ? Nx - 1 : gi);
            gj = gj < 0 ? 0 : (gj >= Ny ? Ny - 1 : gj);
            goff[k] = ((int64_t)gj * Nx + gi) * Nk + 4 * part;
            soff[k] = ((dy + 3) * RW + (dx + 3)) * KP + 4 * part;
        }
    }
    const int plane_floats = RW * RH * KP;
    auto issue = [&](int n) {
        if (n < Np) {
            float* buf = smem + (n % NB) * plane_floats;
            const float* src = Nin + slice * n;
#pragma unroll
            for (int k = 0; k < MAXC; ++k)
                if (goff[k] >= 0) {
                    const unsigned sa = (unsigned)__cvta_generic_to_shared(buf + soff[k]);
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(src + goff[k]));
                }
        }
        asm volatile("cp.async.commit_group;");
    };
    issue(0);
    issue(1);
    const double* rec0 = p.coef + 8 * (((int64_t)jc * Nx + ic) * Nk + mc);
    const double* rec1 = rec0 + 8;
    const float2 Ux = make_float2((float)rec0[0], (float)rec1[0]), Uy = make_float2((float)rec0[1], (float)rec1[1]);
    const float2 cgm = make_float2((float)rec0[6], (float)rec1[6]);
    const float dx_inv = p.dx_inv, dy_inv = p.dy_inv;
    const int ctr = ((cy + 3) * RW + (cx + 3)) * KP;
    for (int n = 0; n < Np; ++n) {
        asm volatile("cp.async.wait_group 1;");
        __syncthreads();
        issue(n + 2);
        const float* pl = smem + (n % NB) * plane_floats + ctr;
        auto V1 = [&](int dcol) { return *reinterpret_cast<const float2*>(pl + dcol * KP + mc); };
        const float2 c = *reinterpret_cast<const float2*>(pl + mc);
        const float4 g = __ldg(reinterpret_cast<const float4*>(p.cg32 + mc + Nk * n));
        float2 ux = make_float2(g.x, g.z), uy = make_float2(g.y, g.w);
        if (p.cg_per_cell) {
            ux = mul2(cgm, ux);
            uy = mul2(cgm, uy);
        }
        ux = add2(ux, Ux);
        uy = add2(uy, Uy);
        float2 fx, fy;
        flux_xy(V1, RW, c, ux, uy, fx, fy);
        fx = mul2(fx, f2(dx_inv));
        fy = mul2(fy, f2(dy_inv));
        if (live) *reinterpret_cast<float2*>(S + slice * n + home) = add2(fx, fy);
    }
    asm volatile("cp.async.wait_group 0;");
}


template <int L, int TX, int TY, int MINB>
__global__ void __launch_bounds__(TX * TY * L, MINB) xy_kernel(const TileArgs p) {
    extern __shared__ __align__(16) float smem[];
    xy_body<L, TX, TY>(p, blockIdx.x, smem);
}

// Pass B: one thread per (cell, kappa pair), CPB cells per CTA, no shared memory.
template <int L, int CPB, int MINB, int SRC>
__global__ void __launch_bounds__(CPB * L, MINB) kp_kernel(const TileArgs p) {
    const float* __restrict__ S = p.sxy;
    const float* __restrict__ Nin = p.Nin;
    const float* N0 = p.N0;
    float* Nout = p.Nout;
    const int Nx = p.Nx, Ny = p.Ny, Nk = p.Nk, Np = p.Np;
    const int64_t slice = (int64_t)Nx * Ny * Nk;
    const int64_t P = (int64_t)Nx * (p.j_hi - p.j_lo);
    const int tid = threadIdx.x, l = tid % L;
    const int64_t cidx = (int64_t)blockIdx.x * CPB + tid / L;
    const bool live_cell = cidx < P;
    const int64_t cc = (live_cell ? cidx : P - 1) + (int64_t)Nx * p.j_lo;
    const int m0 = 2 * l;
    const bool live = live_cell && m0 < Nk;
    const int mc = m0 < Nk ? m0 : Nk - 2;
    const int64_t home = cc * Nk + mc;
    const double* rec0 = p.coef + 8 * (cc * Nk + mc);
    const double* rec1 = rec0 + 8;
    const float2 kap = make_float2((float)rec0[7], (float)rec1[7]);
    const float2 Uxx = make_float2((float)rec0[2], (float)rec1[2]), Uxy = make_float2((float)rec0[3], (float)rec1[3]);
    const float2 Uyx = make_float2((float)rec0[4], (float)rec1[4]), Uyy = make_float2((float)rec0[5], (float)rec1[5]);
    // source constants of this cell and of the lane's two kappa bins (as the tile body)
    Cell32 wc{};
    Bin32 wb0{}, wb1{};
    bool plain_src = SRC == 1;
    const float* lrow = nullptr;
    if constexpr (SRC == 1 || SRC == 2) {
        wc = load_cell32(p.cell32 + 8 * cc);
        wb0 = load_bin32(p.bin32 + 8 * mc);
        wb1 = load_bin32(p.bin32 + 8 * (mc + 1));
        if constexpr (SRC == 2) {
            plain_src = __ldg(p.lflag + cc) != 0u;
            lrow = p.lrate + cc * ((int64_t)Nk * Np) + mc;
        }
    }
    const float2* own = reinterpret_cast<const float2*>(Nin + home);
    const int64_t s2 = slice / 2;
    auto wr = [&](int n) { return n < 0 ? n + Np : (n >= Np ? n - Np : n); };
    float2 w0 = own[s2 * wr(-3)], w1 = own[s2 * wr(-2)], w2 = own[s2 * wr(-1)], w3 = own[0];
    float2 w4 = own[s2 * wr(1)], w5 = own[s2 * wr(2)], w6 = own[s2 * wr(3)];
    const float dk_inv = p.dk_inv, dp_inv = p.dp_inv, dt = p.dt, ca = p.a, cb = p.b;
    const bool ha = (m0 - 2 >= 0) && (m0 + 3 <= Nk - 1);
    const bool hb = (m0 - 1 >= 0) && (m0 + 4 <= Nk - 1);
    const bool hlo = (m0 - 3 >= 0) && (m0 + 2 <= Nk - 1);
    const bool up2 = m0 + 2 <= Nk - 1, up3 = m0 + 3 <= Nk - 1, up4 = m0 + 4 <= Nk - 1;
    float2 prevF = f2(0.f);
    bool prevx = false, prevy = false, have = false;
    for (int n = 0; n < Np; ++n) {
        const float2 nxt = own[s2 * ((n + 4) % Np)];
        const float2 n0v = (p.stage == 1 || !live) ? f2(0.f) : *reinterpret_cast<const float2*>(N0 + slice * n + home);
        const float2 sxy = *reinterpret_cast<const float2*>(S + slice * n + home);
        const float2 c = w3;
        const float4 tg = __ldg(p.trig32 + n);
        const float2 ck = mul2(mul2(f2(-1.f), kap),
                               add2(add2(mul2(f2(tg.x), Uxx), mul2(f2(tg.y), add2(Uyx, Uxy))), mul2(f2(tg.z), Uyy)));
        const float2 cp = sub2(add2(mul2(f2(tg.y), sub2(Uxx, Uyy)), mul2(f2(tg.z), Uyx)), mul2(f2(tg.x), Uxy));
        // kappa stencil of the lane's pair (the reference's clamped indices) from the neighbouring lanes
        const float a_ = __shfl_sync(FULL, c.x, l - 1, L), b_ = __shfl_sync(FULL, c.y, l - 1, L);
        const float d_ = __shfl_sync(FULL, c.y, l - 2, L);
        const float e_ = __shfl_sync(FULL, c.x, l + 1, L), f_ = __shfl_sync(FULL, c.y, l + 1, L);
        const float g_ = __shfl_sync(FULL, c.x, l + 2, L);
        const float k0 = c.x, k1 = c.y;
        const float km1 = l >= 1 ? b_ : k0, km2 = l >= 1 ? a_ : k0, km3 = l >= 2 ? d_ : (l == 1 ? a_ : k0);
        const float kp2 = up2 ? e_ : k1, kp3 = up3 ? f_ : k1, kp4 = up4 ? g_ : (up3 ? f_ : k1);
        const bool pa = ck.x >= 0.f, pb = ck.y >= 0.f;
        float2 Fab;
        if (__all_sync(FULL, pa && pb)) {
            Fab = weno5_2(make_float2(km2, km1), make_float2(km1, k0), make_float2(k0, k1), make_float2(k1, kp2),
                          make_float2(kp2, kp3));
        } else if (__all_sync(FULL, !pa && !pb)) {
            Fab = weno5_2(make_float2(kp3, kp4), make_float2(kp2, kp3), make_float2(k1, kp2), make_float2(k0, k1),
                          make_float2(km1, k0));
        } else {
            const float2 sa0 = make_float2(pa ? km2 : kp3, pb ? km1 : kp4);
            const float2 sa1 = make_float2(pa ? km1 : kp2, pb ? k0 : kp3);
            const float2 sa2 = make_float2(pa ? k0 : k1, pb ? k1 : kp2);
            const float2 sa3 = make_float2(pa ? k1 : k0, pb ? kp2 : k1);
            const float2 sa4 = make_float2(pa ? kp2 : km1, pb ? kp3 : k0);
            Fab = weno5_2(sa0, sa1, sa2, sa3, sa4);
        }
        Fab.x = ha ? Fab.x : (pa ? k0 : k1);
        Fab.y = hb ? Fab.y : (pb ? k1 : kp2);
        float Fam1 = Fab.x;
        if (pa != pb) {
            const float2 t = weno5_2(make_float2(pb ? km2 : kp3, 0.f), make_float2(pb ? km1 : kp2, 0.f),
                                     make_float2(pb ? k0 : k1, 0.f), make_float2(pb ? k1 : k0, 0.f),
                                     make_float2(pb ? kp2 : km1, 0.f));
            Fam1 = ha ? t.x : (pb ? k0 : k1);
        }
        const float upF = __shfl_up_sync(FULL, Fab.y, 1, L);
        const bool upP = __shfl_up_sync(FULL, (int)pb, 1, L) != 0;
        float Flo = upF;
        if (m0 >= 1 && upP != pa) {
            const float2 t = weno5_2(make_float2(pa ? km3 : kp2, 0.f), make_float2(pa ? km2 : k1, 0.f),
                                     make_float2(pa ? km1 : k0, 0.f), make_float2(pa ? k0 : km1, 0.f),
                                     make_float2(pa ? k1 : km2, 0.f));
            Flo = hlo ? t.x : (pa ? km1 : k0);
        }
        const float fk0 = kflux(m0 == Nk - 1, m0 == 0, ck.x, Fab.x, Flo);
        const float fk1 = kflux(m0 + 1 == Nk - 1, false, ck.y, Fab.y, Fam1);
        const float2 fk = mul2(make_float2(fk0, fk1), f2(dk_inv));
        const bool qx = cp.x >= 0.f, qy = cp.y >= 0.f;
        float2 Fpp;
        if (__all_sync(FULL, qx && qy)) Fpp = weno5_2(w1, w2, w3, w4, w5);
        else if (__all_sync(FULL, !qx && !qy)) Fpp = weno5_2(w6, w5, w4, w3, w2);
        else Fpp = weno5_2(sel2(qx, qy, w1, w6), sel2(qx, qy, w2, w5), sel2(qx, qy, w3, w4), sel2(qx, qy, w4, w3),
                           sel2(qx, qy, w5, w2));
        float2 Fpm = prevF;
        if (!have || prevx != qx || prevy != qy) {
            const float2 t = weno5_2(sel2(qx, qy, w0, w5), sel2(qx, qy, w1, w4), sel2(qx, qy, w2, w3),
                                     sel2(qx, qy, w3, w2), sel2(qx, qy, w4, w1));
            if (!have || prevx != qx) Fpm.x = t.x;
            if (!have || prevy != qy) Fpm.y = t.y;
        }
        prevF = Fpp;
        prevx = qx;
        prevy = qy;
        have = true;
        const float2 fp = mul2(mul2(cp, sub2(Fpp, Fpm)), f2(dp_inv));
        float2 G = mul2(f2(-1.f), add2(add2(sxy, fk), fp));
        if constexpr (SRC != 0) {
            if (plain_src) {
                const float2 cs = __ldg(p.cs32 + n);
                G.x += source32(p, wc, wb0, cs.x, cs.y, c.x);
                G.y += source32(p, wc, wb1, cs.x, cs.y, c.y);
            } else if (SRC == 2) {  // learned: N * rate, rate = lscale * sinh(network output of bin (m, n))
                const float2 y = __ldg(reinterpret_cast<const float2*>(lrow + (int64_t)n * Nk));
                G = fma2(mul2(c, f2(p.lscale)), make_float2(sinhf(y.x), sinhf(y.y)), G);
            } else {  // SourceTermSet rates of this stage, state layout
                G = fma2(*reinterpret_cast<const float2*>(p.lin_rates + slice * n + home), c, G);
            }
        }
        float2 st = fma2(f2(dt), G, c);
        st.x = relu(st.x);
        st.y = relu(st.y);
        float2 out = st;
        if (p.stage != 1) {
            out = fma2(f2(ca), n0v, mul2(f2(cb), st));
            out.x = relu(out.x);
            out.y = relu(out.y);
        }
        if (live) {
            if (!isfinite(out.x) || !isfinite(out.y)) atomicOr(p.err, 1u);
            *reinterpret_cast<float2*>(Nout + slice * n + home) = out;
        }
        w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6; w6 = nxt;
    }
}

// Pass B with four kappa bins per lane (two packed pairs), for stages without the bundle or learned
// sources (SRC 0 and 3): the pair kernel's arithmetic element for element, with per-lane overhead
// (shuffles, window bookkeeping, addressing) shared by four bins. The kappa stencil m0-3 .. m0+6 comes
// from the lanes below and above (three shuffles each, the reference's clamped indices: Nk % 4 == 0, so
// only the lowest and the highest live lane clamp).
template <int L, int CPB, int MINB, int SRC>
__global__ void __launch_bounds__(CPB * L, MINB) kq_kernel(const TileArgs p) {
    static_assert(SRC == 0 || SRC == 3, "bundle and learned sources use the pair kernel");
    const float* __restrict__ S = p.sxy;
    const float* __restrict__ Nin = p.Nin;
    const float* N0 = p.N0;
    float* Nout = p.Nout;
    const int Nx = p.Nx, Ny = p.Ny, Nk = p.Nk, Np = p.Np;
    const int64_t slice = (int64_t)Nx * Ny * Nk;
    const int64_t P = (int64_t)Nx * (p.j_hi - p.j_lo);
    const int tid = threadIdx.x, l = tid % L;
    const int64_t cidx = (int64_t)blockIdx.x * CPB + tid / L;
    const bool live_cell = cidx < P;
    const int64_t cc = (live_cell ? cidx : P - 1) + (int64_t)Nx * p.j_lo;
    const int m0 = 4 * l;
    const bool live = live_cell && m0 < Nk;
    const int mc = m0 < Nk ? m0 : Nk - 4;
    const int64_t home = cc * Nk + mc;
    const double* r0 = p.coef + 8 * home;
    auto cq = [&](int f) {
        return Q{make_float2((float)r0[f], (float)r0[8 + f]), make_float2((float)r0[16 + f], (float)r0[24 + f])};
    };
    const Q kap = cq(7), Uxx = cq(2), Uxy = cq(3), Uyx = cq(4), Uyy = cq(5);
    const float* own = Nin + home;
    auto wr = [&](int n) { return n < 0 ? n + Np : (n >= Np ? n - Np : n); };
    Q w0 = ldq(own + slice * wr(-3)), w1 = ldq(own + slice * wr(-2)), w2 = ldq(own + slice * wr(-1));
    Q w3 = ldq(own), w4 = ldq(own + slice * wr(1)), w5 = ldq(own + slice * wr(2)), w6 = ldq(own + slice * wr(3));
    const float dk_inv = p.dk_inv, dp_inv = p.dp_inv, dt = p.dt, ca = p.a, cb = p.b;
    auto full = [&](int q) { return q - 2 >= 0 && q + 3 <= Nk - 1; };   // face q|q+1 has its 5-point stencil
    const bool hlo = full(m0 - 1), ha = full(m0), hb = full(m0 + 1), hc = full(m0 + 2), hd = full(m0 + 3);
    const bool up = m0 + 4 <= Nk - 1;   // bins above the quad exist (else clamped to the last bin)
    Q prevF = qz();
    bool pvx = false, pvy = false, pvz = false, pvw = false, have = false;
    for (int n = 0; n < Np; ++n) {
        const int64_t off = slice * n + home;
        const Q nxt = ldq(own + slice * ((n + 4) % Np));
        const Q n0v = (p.stage == 1 || !live) ? qz() : ldq(N0 + off);
        const Q sxy = ldq(S + off);
        const Q c = w3;
        const float4 tg = __ldg(p.trig32 + n);
        auto ckf = [&](float2 kp_, float2 xx, float2 xy, float2 yx, float2 yy) {
            return mul2(mul2(f2(-1.f), kp_),
                        add2(add2(mul2(f2(tg.x), xx), mul2(f2(tg.y), add2(yx, xy))), mul2(f2(tg.z), yy)));
        };
        auto cpf = [&](float2 xx, float2 xy, float2 yx, float2 yy) {
            return sub2(add2(mul2(f2(tg.y), sub2(xx, yy)), mul2(f2(tg.z), yx)), mul2(f2(tg.x), xy));
        };
        const Q ck = {ckf(kap.a, Uxx.a, Uxy.a, Uyx.a, Uyy.a), ckf(kap.b, Uxx.b, Uxy.b, Uyx.b, Uyy.b)};
        const Q cp = {cpf(Uxx.a, Uxy.a, Uyx.a, Uyy.a), cpf(Uxx.b, Uxy.b, Uyx.b, Uyy.b)};
        const float k0 = c.a.x, k1 = c.a.y, k2 = c.b.x, k3 = c.b.y;
        const float s_m3 = __shfl_sync(FULL, k1, l - 1, L), s_m2 = __shfl_sync(FULL, k2, l - 1, L);
        const float s_m1 = __shfl_sync(FULL, k3, l - 1, L);
        const float s_p4 = __shfl_sync(FULL, k0, l + 1, L), s_p5 = __shfl_sync(FULL, k1, l + 1, L);
        const float s_p6 = __shfl_sync(FULL, k2, l + 1, L);
        const float km3 = l >= 1 ? s_m3 : k0, km2 = l >= 1 ? s_m2 : k0, km1 = l >= 1 ? s_m1 : k0;
        const float kp4 = up ? s_p4 : k3, kp5 = up ? s_p5 : k3, kp6 = up ? s_p6 : k3;
        // upper faces a..d of bins m0..m0+3, each upwinded by its own bin
        const bool pa = ck.a.x >= 0.f, pb = ck.a.y >= 0.f, pc = ck.b.x >= 0.f, pd = ck.b.y >= 0.f;
        float2 Fab, Fcd;
        if (__all_sync(FULL, pa && pb && pc && pd)) {
            Fab = weno5_2(make_float2(km2, km1), make_float2(km1, k0), make_float2(k0, k1), make_float2(k1, k2),
                          make_float2(k2, k3));
            Fcd = weno5_2(make_float2(k0, k1), make_float2(k1, k2), make_float2(k2, k3), make_float2(k3, kp4),
                          make_float2(kp4, kp5));
        } else if (__all_sync(FULL, !pa && !pb && !pc && !pd)) {
            Fab = weno5_2(make_float2(k3, kp4), make_float2(k2, k3), make_float2(k1, k2), make_float2(k0, k1),
                          make_float2(km1, k0));
            Fcd = weno5_2(make_float2(kp5, kp6), make_float2(kp4, kp5), make_float2(k3, kp4), make_float2(k2, k3),
                          make_float2(k1, k2));
        } else {
            Fab = weno5_2(make_float2(pa ? km2 : k3, pb ? km1 : kp4), make_float2(pa ? km1 : k2, pb ? k0 : k3),
                          make_float2(pa ? k0 : k1, pb ? k1 : k2), make_float2(pa ? k1 : k0, pb ? k2 : k1),
                          make_float2(pa ? k2 : km1, pb ? k3 : k0));
            Fcd = weno5_2(make_float2(pc ? k0 : kp5, pd ? k1 : kp6), make_float2(pc ? k1 : kp4, pd ? k2 : kp5),
                          make_float2(pc ? k2 : k3, pd ? k3 : kp4), make_float2(pc ? k3 : k2, pd ? kp4 : k3),
                          make_float2(pc ? kp4 : k1, pd ? kp5 : k2));
        }
        const float Fa = ha ? Fab.x : (pa ? k0 : k1), Fb = hb ? Fab.y : (pb ? k1 : k2);
        const float Fc = hc ? Fcd.x : (pc ? k2 : k3), Fd = hd ? Fcd.y : (pd ? k3 : kp4);
        // lower faces: of m0 the lane below's face d (upwinded by bin m0-1), of m0+1..m0+3 the faces
        // a..c; recomputed in the bin's own orientation where the two bins' signs differ
        const float upF = __shfl_up_sync(FULL, Fd, 1, L);
        const bool upP = __shfl_up_sync(FULL, (int)pd, 1, L) != 0;
        const bool mA0 = m0 >= 1 && upP != pa, mA1 = pa != pb, mB0 = pb != pc, mB1 = pc != pd;
        float loA0 = upF, loA1 = Fa, loB0 = Fb, loB1 = Fc;
        if (mA0 || mA1) {
            const float2 t = weno5_2(make_float2(pa ? km3 : k2, pb ? km2 : k3), make_float2(pa ? km2 : k1, pb ? km1 : k2),
                                     make_float2(pa ? km1 : k0, pb ? k0 : k1), make_float2(pa ? k0 : km1, pb ? k1 : k0),
                                     make_float2(pa ? k1 : km2, pb ? k2 : km1));
            if (mA0) loA0 = hlo ? t.x : (pa ? km1 : k0);
            if (mA1) loA1 = ha ? t.y : (pb ? k0 : k1);
        }
        if (mB0 || mB1) {
            const float2 t = weno5_2(make_float2(pc ? km1 : kp4, pd ? k0 : kp5), make_float2(pc ? k0 : k3, pd ? k1 : kp4),
                                     make_float2(pc ? k1 : k2, pd ? k2 : k3), make_float2(pc ? k2 : k1, pd ? k3 : k2),
                                     make_float2(pc ? k3 : k0, pd ? kp4 : k1));
            if (mB0) loB0 = hb ? t.x : (pc ? k1 : k2);
            if (mB1) loB1 = hc ? t.y : (pd ? k2 : k3);
        }
        const Q fk = {mul2(make_float2(kflux(m0 == Nk - 1, m0 == 0, ck.a.x, Fa, loA0),
                                       kflux(m0 + 1 == Nk - 1, false, ck.a.y, Fb, loA1)), f2(dk_inv)),
                      mul2(make_float2(kflux(m0 + 2 == Nk - 1, false, ck.b.x, Fc, loB0),
                                       kflux(m0 + 3 == Nk - 1, false, ck.b.y, Fd, loB1)), f2(dk_inv))};
        // phi faces: the upper from the window, the lower carried from the previous step unless the sign changed
        const bool qx = cp.a.x >= 0.f, qy = cp.a.y >= 0.f, qz_ = cp.b.x >= 0.f, qw = cp.b.y >= 0.f;
        Q Fpp;
        if (__all_sync(FULL, qx && qy && qz_ && qw)) Fpp = qweno(w1, w2, w3, w4, w5);
        else if (__all_sync(FULL, !qx && !qy && !qz_ && !qw)) Fpp = qweno(w6, w5, w4, w3, w2);
        else
            Fpp = {weno5_2(sel2(qx, qy, w1.a, w6.a), sel2(qx, qy, w2.a, w5.a), sel2(qx, qy, w3.a, w4.a),
                           sel2(qx, qy, w4.a, w3.a), sel2(qx, qy, w5.a, w2.a)),
                   weno5_2(sel2(qz_, qw, w1.b, w6.b), sel2(qz_, qw, w2.b, w5.b), sel2(qz_, qw, w3.b, w4.b),
                           sel2(qz_, qw, w4.b, w3.b), sel2(qz_, qw, w5.b, w2.b))};
        Q Fpm = prevF;
        if (!have || pvx != qx || pvy != qy) {
            const float2 t = weno5_2(sel2(qx, qy, w0.a, w5.a), sel2(qx, qy, w1.a, w4.a), sel2(qx, qy, w2.a, w3.a),
                                     sel2(qx, qy, w3.a, w2.a), sel2(qx, qy, w4.a, w1.a));
            if (!have || pvx != qx) Fpm.a.x = t.x;
            if (!have || pvy != qy) Fpm.a.y = t.y;
        }
        if (!have || pvz != qz_ || pvw != qw) {
            const float2 t = weno5_2(sel2(qz_, qw, w0.b, w5.b), sel2(qz_, qw, w1.b, w4.b), sel2(qz_, qw, w2.b, w3.b),
                                     sel2(qz_, qw, w3.b, w2.b), sel2(qz_, qw, w4.b, w1.b));
            if (!have || pvz != qz_) Fpm.b.x = t.x;
            if (!have || pvw != qw) Fpm.b.y = t.y;
        }
        prevF = Fpp;
        pvx = qx;
        pvy = qy;
        pvz = qz_;
        pvw = qw;
        have = true;
        const Q fp = {mul2(mul2(cp.a, sub2(Fpp.a, Fpm.a)), f2(dp_inv)), mul2(mul2(cp.b, sub2(Fpp.b, Fpm.b)), f2(dp_inv))};
        Q G = {mul2(f2(-1.f), add2(add2(sxy.a, fk.a), fp.a)), mul2(f2(-1.f), add2(add2(sxy.b, fk.b), fp.b))};
        if constexpr (SRC == 3) {   // SourceTermSet rates of this stage, state layout
            const Q r = ldq(p.lin_rates + off);
            G = {fma2(r.a, c.a, G.a), fma2(r.b, c.b, G.b)};
        }
        auto upd = [&](float2 g, float2 cv, float2 nv) {
            float2 st = fma2(f2(dt), g, cv);
            st.x = relu(st.x);
            st.y = relu(st.y);
            float2 out = st;
            if (p.stage != 1) {
                out = fma2(f2(ca), nv, mul2(f2(cb), st));
                out.x = relu(out.x);
                out.y = relu(out.y);
            }
            return out;
        };
        const Q out = {upd(G.a, c.a, n0v.a), upd(G.b, c.b, n0v.b)};
        if (live) {
            if (!isfinite(out.a.x) || !isfinite(out.a.y) || !isfinite(out.b.x) || !isfinite(out.b.y)) atomicOr(p.err, 1u);
            stq(Nout + off, out);
        }
        w0 = w1;
        w1 = w2;
        w2 = w3;
        w3 = w4;
        w4 = w5;
        w5 = w6;
        w6 = nxt;
    }
}

// Second pass of an intrinsic stage with the bundle (SRC 1) or the learned (SRC 2) sources, after the
// y-walk x/y pass stored S = fx + fy: one thread per (cell, kappa pair) walking the phi ring with the
// cell's wind constants and its bins' constants loaded once; G = -S, the sources and the stage update
// as the tile body (G = -(fx + fy) there).
template <int L, int CPB, int MINB, int SRC>
__global__ void __launch_bounds__(CPB * L, MINB) ks_kernel(const TileArgs p) {
    static_assert(SRC == 1 || SRC == 2, "bundle or learned sources");
    const float* __restrict__ S = p.sxy;
    const float* __restrict__ Nin = p.Nin;
    const float* N0 = p.N0;
    float* Nout = p.Nout;
    const int Nx = p.Nx, Ny = p.Ny, Nk = p.Nk, Np = p.Np;
    const int64_t slice = (int64_t)Nx * Ny * Nk;
    const int64_t P = (int64_t)Nx * (p.j_hi - p.j_lo);
    const int tid = threadIdx.x, l = tid % L;
    const int64_t cidx = (int64_t)blockIdx.x * CPB + tid / L;
    const bool live_cell = cidx < P;
    const int64_t cc = (live_cell ? cidx : P - 1) + (int64_t)Nx * p.j_lo;
    const int m0 = 2 * l;
    const bool live = live_cell && m0 < Nk;
    const int mc = m0 < Nk ? m0 : Nk - 2;
    const int64_t home = cc * Nk + mc;
    const Cell32 wc = load_cell32(p.cell32 + 8 * cc);
    const Bin32 wb0 = load_bin32(p.bin32 + 8 * mc), wb1 = load_bin32(p.bin32 + 8 * (mc + 1));
    bool plain_src = SRC == 1;
    const float* lrow = nullptr;
    if constexpr (SRC == 2) {
        plain_src = __ldg(p.lflag + cc) != 0u;
        lrow = p.lrate + cc * ((int64_t)Nk * Np) + mc;
    }
    const float dt = p.dt, ca = p.a, cb = p.b;
    for (int n = 0; n < Np; ++n) {
        const int64_t off = slice * n + home;
        const float2 c = *reinterpret_cast<const float2*>(Nin + off);
        const float2 sxy = *reinterpret_cast<const float2*>(S + off);
        const float2 n0v = (p.stage == 1 || !live) ? f2(0.f) : *reinterpret_cast<const float2*>(N0 + off);
        float2 G = mul2(f2(-1.f), sxy);
        if (plain_src) {
            const float2 cs = __ldg(p.cs32 + n);
            G.x += source32(p, wc, wb0, cs.x, cs.y, c.x);
            G.y += source32(p, wc, wb1, cs.x, cs.y, c.y);
        } else if constexpr (SRC == 2) {  // learned: N * rate, rate = lscale * sinh(network output of bin (m, n))
            const float2 y = __ldg(reinterpret_cast<const float2*>(lrow + (int64_t)n * Nk));
            G = fma2(mul2(c, f2(p.lscale)), make_float2(sinhf(y.x), sinhf(y.y)), G);
        }
        float2 st = fma2(f2(dt), G, c);
        st.x = relu(st.x);
        st.y = relu(st.y);
        float2 out = st;
        if (p.stage != 1) {
            out = fma2(f2(ca), n0v, mul2(f2(cb), st));
            out.x = relu(out.x);
            out.y = relu(out.y);
        }
        if (live) {
            if (!isfinite(out.x) || !isfinite(out.y)) atomicOr(p.err, 1u);
            *reinterpret_cast<float2*>(Nout + off) = out;
        }
    }
}

// Single-model kernel: one CTA per TX x TY tile, MINB CTAs resident per SM.
template <int L, int TX, int TY, int MINB, bool REFRACT, int SRC>
__global__ void __launch_bounds__(TX * TY * L, MINB) tile_kernel(const TileArgs p) {
    extern __shared__ __align__(16) float smem[];
    tile_body<L, TX, TY, REFRACT, SRC>(p, blockIdx.x, smem);
}

// Tile shape of the single-model kernel per lane count: 256 threads and two CTAs per SM (while one CTA
// waits at its per-plane barrier the other issues). Measured on seamount 1024^2 x 32 x 36 (stage 2):
// 4 x 4 tiles 14.4 ms against 15.6 ms for one 512-thread CTA per SM with 8 x 4 tiles; 8 x 2 and 2 x 8
// tiles, 128-thread CTAs four per SM, and three 256-thread CTAs per SM (96 registers, spilling) were
// slower.
template <int L> struct Shape;
template <> struct Shape<16> { static constexpr int TX = 4, TY = 4, MINB = 2; };
template <> struct Shape<8> { static constexpr int TX = 8, TY = 4, MINB = 2; };
template <> struct Shape<4> { static constexpr int TX = 8, TY = 8, MINB = 2; };

// Ensemble kernel: a persistent grid of ENSEMBLE_THREADS-thread CTAs takes work items (member, tile,
// tile shape) from one atomic counter until the list is exhausted; no CTA ever waits for another.
// The member's arguments are copied to shared memory per item.
template <bool REFRACT>
__global__ void __launch_bounds__(ENSEMBLE_THREADS, 1)
    ensemble_kernel(const TileArgs* __restrict__ args, const int4* __restrict__ items, int nitems,
                    unsigned int* counter) {
    extern __shared__ __align__(16) float smem[];
    __shared__ TileArgs s_args;
    __shared__ int s_item;
    constexpr int WORDS = (int)(sizeof(TileArgs) / 4);
    static_assert(sizeof(TileArgs) % 4 == 0 && WORDS <= ENSEMBLE_THREADS, "TileArgs copy");
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const int4 w = __ldg(items + it);
        if (threadIdx.x < WORDS)
            reinterpret_cast<int*>(&s_args)[threadIdx.x] = __ldg(reinterpret_cast<const int*>(args + w.x) + threadIdx.x);
        __syncthreads();
        switch (w.z) {
            case 0: tile_body<kEnsembleShapes[0].L, kEnsembleShapes[0].TX, kEnsembleShapes[0].TY, REFRACT, 0>(s_args, w.y, smem); break;
            case 1: tile_body<kEnsembleShapes[1].L, kEnsembleShapes[1].TX, kEnsembleShapes[1].TY, REFRACT, 0>(s_args, w.y, smem); break;
            case 2: tile_body<kEnsembleShapes[2].L, kEnsembleShapes[2].TX, kEnsembleShapes[2].TY, REFRACT, 0>(s_args, w.y, smem); break;
            case 3: tile_body<kEnsembleShapes[3].L, kEnsembleShapes[3].TX, kEnsembleShapes[3].TY, REFRACT, 0>(s_args, w.y, smem); break;
            case 4: tile_body<kEnsembleShapes[4].L, kEnsembleShapes[4].TX, kEnsembleShapes[4].TY, REFRACT, 0>(s_args, w.y, smem); break;
            case 5: tile_body<kEnsembleShapes[5].L, kEnsembleShapes[5].TX, kEnsembleShapes[5].TY, REFRACT, 0>(s_args, w.y, smem); break;
            case 6: tile_body<kEnsembleShapes[6].L, kEnsembleShapes[6].TX, kEnsembleShapes[6].TY, REFRACT, 0>(s_args, w.y, smem); break;
            case 7: tile_body<kEnsembleShapes[7].L, kEnsembleShapes[7].TX, kEnsembleShapes[7].TY, REFRACT, 0>(s_args, w.y, smem); break;
            default: tile_body<kEnsembleShapes[8].L, kEnsembleShapes[8].TX, kEnsembleShapes[8].TY, REFRACT, 0>(s_args, w.y, smem); break;
        }
        __syncthreads();  // the staged planes, s_args and s_item are reused by the next item
    }
}

template <int L, bool REFRACT, int SRC>
cudaError_t launch_variant(const TileArgs& a, int tiles, cudaStream_t s) {
    constexpr int TX = Shape<L>::TX, TY = Shape<L>::TY;
    const size_t smem = tile_smem_bytes(L, TX, TY);
    auto k = tile_kernel<L, TX, TY, Shape<L>::MINB, REFRACT, SRC>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<tiles, TX * TY * L, smem, s>>>(a);
    return cudaGetLastError();
}

// Two-pass refraction stage: pass A over the shape's tiles, then pass B over 256-thread CTAs, three CTAs
// per SM each (24 warps at <= 80 registers).
template <int L, int SRC>
cudaError_t launch_split(const TileArgs& a, cudaStream_t s) {
    constexpr int TX = Shape<L>::TX, TY = Shape<L>::TY, CPB = 256 / L;
    const int tiles = ((a.Nx + TX - 1) / TX) * ((a.j_hi - a.j_lo + TY - 1) / TY);
    cudaError_t e;
    if (a.ux32) {   // the y-walk form (rpl_xyw.cu): one reconstruction per face
        e = launch_xyw(a, s);
    } else {
        const size_t smem = tile_smem_bytes(L, TX, TY);
        auto ka = xy_kernel<L, TX, TY, 3>;
        cudaFuncSetAttribute(ka, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        ka<<<tiles, TX * TY * L, smem, s>>>(a);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    const int64_t cells = (int64_t)a.Nx * (a.j_hi - a.j_lo);
    if constexpr (SRC == 0 || SRC == 3) {
        if (a.pass_b_quads) {   // four kappa bins per lane: 128-thread CTAs, four per SM
            constexpr int L4 = L / 2, QPB = 128 / L4;
            kq_kernel<L4, QPB, 4, SRC><<<(unsigned)((cells + QPB - 1) / QPB), QPB * L4, 0, s>>>(a);
            return cudaGetLastError();
        }
    }
    // the per-cell source constants of the bundle and the learned source need registers: two CTAs per SM
    constexpr int BMINB = (SRC == 1 || SRC == 2) ? 2 : 3;
    kp_kernel<L, CPB, BMINB, SRC><<<(unsigned)((cells + CPB - 1) / CPB), CPB * L, 0, s>>>(a);
    return cudaGetLastError();
}

template <int L>
cudaError_t launch_L(const Handle& h, const StageParams& p, const TileArgs& a, cudaStream_t s) {
    constexpr int TX = Shape<L>::TX, TY = Shape<L>::TY;
    const int tiles = (int)(((h.desc.Nx + TX - 1) / TX) * ((p.j_hi - p.j_lo + TY - 1) / TY));
    const bool refract = p.transport == RPL_TRANSPORT_REFRACTION;
    const int src = p.learned ? 2 : ((p.has_wind || p.has_diss) ? 1 : (p.lin_rates ? 3 : 0));
    if (refract && a.sxy) {
        if (src == 3) return launch_split<L, 3>(a, s);
        if (src == 2) return launch_split<L, 2>(a, s);
        return src ? launch_split<L, 1>(a, s) : launch_split<L, 0>(a, s);
    }
    if (refract) {
        if (src == 3) return launch_variant<L, true, 3>(a, tiles, s);
        if (src == 2) return launch_variant<L, true, 2>(a, tiles, s);
        return src ? launch_variant<L, true, 1>(a, tiles, s) : launch_variant<L, true, 0>(a, tiles, s);
    }
    // the y-walk form (rpl_xyw.cu, one reconstruction per face): one pass without the bundle or learned
    // sources; with them the x/y pass stores S and ks_kernel adds the sources per cell (their per-cell
    // constants loaded once per phi ring) and updates
    if (a.rmax && (src == 0 || src == 3)) return launch_xyi(a, src, s);
    if (a.rmax && a.sxy && (src == 1 || src == 2)) {
        cudaError_t e = launch_xy_intrinsic(a, s);
        if (e != cudaSuccess) return e;
        constexpr int CPB = 256 / L;
        const int64_t cells = (int64_t)a.Nx * (a.j_hi - a.j_lo);
        const unsigned blocks = (unsigned)((cells + CPB - 1) / CPB);
        if (src == 1) ks_kernel<L, CPB, 2, 1><<<blocks, CPB * L, 0, s>>>(a);
        else ks_kernel<L, CPB, 2, 2><<<blocks, CPB * L, 0, s>>>(a);
        return cudaGetLastError();
    }
    if (src == 3) return launch_variant<L, false, 3>(a, tiles, s);
    if (src == 2) return launch_variant<L, false, 2>(a, tiles, s);
    return src ? launch_variant<L, false, 1>(a, tiles, s) : launch_variant<L, false, 0>(a, tiles, s);
}

}  // namespace

size_t tile_smem_bytes(int L, int TX, int TY) { return (size_t)NB * (TX + 6) * (TY + 6) * 2 * L * sizeof(float); }

size_t ensemble_smem_bytes() {
    size_t m = 0;
    for (const TileShape& t : kEnsembleShapes) m = std::max(m, tile_smem_bytes(t.L, t.TX, t.TY));
    return m;
}

TileArgs make_tile_args(const Handle& h, const StageParams& p, const void* Nin, const void* N0, void* Nout) {
    TileArgs a{};
    a.Nin = (const float*)Nin;
    a.N0 = (const float*)N0;
    a.Nout = (float*)Nout;
    a.coef = p.coef;
    a.trig32 = p.trig32;
    a.cg32 = p.cg32;
    a.cs32 = p.cs32;
    a.cell32 = p.cell32;
    a.bin32 = p.bin32;
    a.err = p.err;
    a.Nx = (int)h.desc.Nx;
    a.Ny = (int)h.desc.Ny;
    a.Nk = (int)h.desc.Nk;
    a.Np = (int)h.desc.Np;
    a.stage = p.stage;
    a.cg_per_cell = p.cg_per_cell;
    a.has_wind = p.has_wind;
    a.stress_cap = p.stress_cap;
    a.has_diss = p.has_diss;
    a.dx_inv = (float)p.dx_inv;
    a.dy_inv = (float)p.dy_inv;
    a.dk_inv = (float)p.dk_inv;
    a.dp_inv = (float)p.dp_inv;
    a.dt = (float)p.dt;
    a.a = (float)p.a;
    a.b = (float)p.b;
    a.wind_K32 = p.wind_K32;
    a.von_karman32 = p.von_karman32;
    a.z_alpha32 = p.z_alpha32;
    a.p_in = (float)p.p_in;
    a.ds_p = (float)p.ds_p;
    a.learned = p.learned;
    a.lrate = p.lrate;
    a.lflag = p.lflag;
    a.lscale = p.lscale;
    a.lin_rates = static_cast<const float*>(p.lin_rates);
    a.j_lo = (int)p.j_lo;
    a.j_hi = (int)p.j_hi;
    a.sxy = h.d_sxy;
    a.pass_b_quads = !h.pass_b_pairs;
    if (h.d_vel32) {
        const int64_t c3 = h.desc.Nx * h.desc.Ny * h.desc.Nk;
        if (h.desc.transport == RPL_TRANSPORT_REFRACTION) {
            a.ux32 = h.d_vel32;
            a.uy32 = h.d_vel32 + c3;
            a.cgc32 = h.d_vel32 + 2 * c3;
        } else {
            a.cgc32 = h.d_vel32;   // intrinsic transport: the c_g plane only
        }
        a.rmax = h.d_rmax;
    }
    return a;
}

bool tile32_supported(const Handle& h) {
    const rpl_desc& d = h.desc;
    return h.precision == RPL_FP32 && d.transport != RPL_TRANSPORT_NONE && d.Nk % 4 == 0 && d.Nk >= 4 &&
           d.Nk <= 32 && (d.transport != RPL_TRANSPORT_REFRACTION || d.Np >= 3) && d.Nx >= 3 && d.Ny >= 3;
}

int tile_lanes(int64_t Nk) { return Nk <= 8 ? 4 : (Nk <= 16 ? 8 : 16); }

cudaError_t launch_tile32(const Handle& h, const StageParams& p, const void* Nin, const void* N0, void* Nout,
                          cudaStream_t s) {
    const TileArgs a = make_tile_args(h, p, Nin, N0, Nout);
    switch (tile_lanes(h.desc.Nk)) {
        case 4: return launch_L<4>(h, p, a, s);
        case 8: return launch_L<8>(h, p, a, s);
        default: return launch_L<16>(h, p, a, s);
    }
}

cudaError_t prepare_ensemble_kernels() {
    const int smem = (int)ensemble_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(ensemble_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(ensemble_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    return e;
}

int ensemble_grid(bool refract, int device) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int smem = (int)ensemble_smem_bytes();
    if (refract) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ensemble_kernel<true>, ENSEMBLE_THREADS, smem);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ensemble_kernel<false>, ENSEMBLE_THREADS, smem);
    return std::max(1, sms) * std::max(1, per_sm);
}

cudaError_t launch_ensemble_stage(bool refract, const TileArgs* d_args, const int4* d_items, int nitems,
                                  unsigned int* d_counter, int grid, cudaStream_t s) {
    const size_t smem = ensemble_smem_bytes();
    if (refract) ensemble_kernel<true><<<grid, ENSEMBLE_THREADS, smem, s>>>(d_args, d_items, nitems, d_counter);
    else ensemble_kernel<false><<<grid, ENSEMBLE_THREADS, smem, s>>>(d_args, d_items, nitems, d_counter);
    return cudaGetLastError();
}

}  // namespace rpl
