// rpl_xyw.cu -- pass A of the FP32 refraction stage as a y-walk: the x and y fluxes
// u (N(+1/2) - N(-1/2)) / spacing of every cell-bin (wave_current_refraction.jl:104-123), written as
// S = fx + fy in the state layout for pass B (kp_kernel, rpl_tile32.cu).
//
// Layout of the work: a CTA owns one direction bin n, CX consecutive cells in x (the first of them only
// supplies a face: CX-1 cells are written) and a segment of SEG rows, with L lanes per cell and four
// adjacent kappa bins per lane (two packed FP32 pairs). Its threads walk the rows j of the segment:
//  * every face is reconstructed once. The x face between cells s and s+1 is computed by the lane of
//    cell s and handed to cell s+1 through shared memory one row later; the y face j+1/2 of a column
//    is the upper face of row j and the lower face of row j+1 in the same thread;
//  * the y stencil (rows j-3 .. j+3) and the x stencil of row j come from a shared ring of 8 staged
//    rows. A row is written twice (slot s and s+8), so the seven rows around j sit at constant
//    offsets from one slot; row j+3 is written before the step's barrier into the slot of row j-5,
//    which no thread reads after step k-2 (the slowest thread is past the previous barrier);
//  * upwinding: the reference upwinds each cell's two faces by the sign of the cell-centre velocity.
//    Where a CTA's x (or y) velocities share one sign, each face needs one reconstruction and the
//    body has no per-element selects. The FP32 velocity of bin (m, n) is u = c g(m,n) + U (c the
//    per-cell c_g magnitude when the depth varies, else 1 with c_g in the table g), so it has the sign
//    of g(m,n) wherever |g(m,n)| > |U| / c. vel32_kernel stores, per region of cells and kappa bin, the
//    maximum of |U| / c enlarged by 1e-5; a CTA whose every bin passes |g| (1 - 1e-5) > that maximum,
//    with one sign, runs the uniform body, every other CTA the general body (both candidates where
//    needed, per-element selects). The margins cover the FP32 roundings of the product, the division
//    and the test. Both bodies give the fused tile kernel's face values bit for bit.
//  * the same body, with no currents and the stage update in place of the store of S, is the whole
//    stage of intrinsic transport without the bundle or learned sources (launch_xyi), in place of the
//    fused tile kernel.
#include <cuda_runtime.h>

#include <type_traits>

#include "rpl_internal.h"
#include "rpl_weno32.cuh"

namespace rpl {

namespace {

using namespace w32;

constexpr int XSEG = 128;            // rows per CTA segment (and per region of the ratio table)
constexpr int XTHREADS = 256;        // threads per CTA: CX = XTHREADS / L cells
enum { POS = 0, NEG = 1, MIX = 2 };

// bit 0: some element >= 0; bit 1: some element < 0
__device__ __forceinline__ int code2(float2 u) {
    return ((u.x >= 0.f || u.y >= 0.f) ? 1 : 0) | ((u.x < 0.f || u.y < 0.f) ? 2 : 0);
}
__device__ __forceinline__ int codeq(Q u) { return code2(u.a) | code2(u.b); }
__device__ __forceinline__ float2 selp(float2 u, float2 a, float2 b) {  // per element: u >= 0 ? a : b
    return make_float2(u.x >= 0.f ? a.x : b.x, u.y >= 0.f ? a.y : b.y);
}
__device__ __forceinline__ Q selq(Q u, Q x, Q y) { return {selp(u.a, x.a, y.a), selp(u.b, x.b, y.b)}; }

template <int L>
struct Lay {
    static constexpr int CX = XTHREADS / L, XW = CX + 5, KP = 4 * L, ROW = XW * KP;
    static constexpr int ring = 16 * ROW, fs = 2 * CX * L * 8, sg = 2 * (CX + 1) * L;
    static constexpr size_t bytes = (size_t)(ring + fs + sg) * 4;
};

// FSRC < 0: pass A of a refraction stage (currents, S = fx + fy stored). FSRC 0 or 3: the whole stage of
// intrinsic transport (no currents, no kappa or phi terms): G = -(fx + fy) in the tile body's order, with
// FSRC 3 the SourceTermSet rates, and the stage update, written to Nout. (The bundle and the learned
// sources stay in the tile kernel, which walks the phi ring at a fixed cell and loads their per-cell
// constants once: measured on the 768^2 hurricane, 24.4 against 30.3 ms per step.)
// FSRC -2: pass A of an intrinsic stage with the bundle or learned sources (no currents, S stored; the
// sources and the update follow in ks_kernel, rpl_tile32.cu).
template <int L, int XM, int YM, int FSRC>
__device__ __forceinline__ void xyw_body(const TileArgs& p, float* smem, int n, int tx, int js, int je) {
    static_assert(FSRC == -2 || FSRC == -1 || FSRC == 0 || FSRC == 3,
                  "pass A, or an intrinsic stage without bundle sources");
    constexpr bool FUSED = FSRC >= 0, CURR = FSRC == -1;   // CURR: currents (refraction)
    using Y = Lay<L>;
    constexpr int CX = Y::CX, KP = Y::KP, ROW = Y::ROW;
    const int Nx = p.Nx, Ny = p.Ny, Nk = p.Nk;
    const int64_t slice = (int64_t)Nx * Ny * Nk;
    const int tid = threadIdx.x, l = tid % L, slot = tid / L;
    const int cnt = je - js;
    const int ibase = tx * (CX - 1) - 1;                       // x of slot 0
    const int my_i = ((ibase + slot) % Nx + Nx) % Nx;
    const bool own = slot >= 1 && ibase + slot < Nx;
    const int m0 = 4 * l;
    const bool klive = m0 < Nk;
    const int mc = klive ? m0 : Nk - 4;                        // idle lanes read the last live quad
    const bool out_ok = own && klive;
    // halo columns: 2 on the left, 3 on the right, loaded by the first 5*L threads
    const bool hal = tid < 5 * L;
    const int hs = tid / L < 2 ? tid / L - 2 : CX + tid / L - 2;
    const int hi_x = hal ? ((ibase + hs) % Nx + Nx) % Nx : 0;
    float* ring = smem;
    float* fsm = smem + Y::ring;
    int* sg = reinterpret_cast<int*>(smem + Y::ring + Y::fs);
    const int rs = Nx * Nk;                                    // row stride within a direction slice
    const float* base = p.Nin + slice * n;
    float* Sn = FUSED ? p.Nout + slice * n : p.sxy + slice * n;   // S (pass A) or the stage's output
    const float* N0n = p.N0 + slice * n;
    const int colm = my_i * Nk + mc, hcol = hi_x * Nk + mc;
    const float4 g0 = __ldg(reinterpret_cast<const float4*>(p.cg32 + mc + Nk * n));
    const float4 g1 = __ldg(reinterpret_cast<const float4*>(p.cg32 + mc + 2 + Nk * n));
    const Q gx = {make_float2(g0.x, g0.z), make_float2(g1.x, g1.z)};
    const Q gy = {make_float2(g0.y, g0.w), make_float2(g1.y, g1.w)};
    const bool cgp = p.cg_per_cell != 0;
    auto modr = [&](int r) { return (r % Ny + Ny) % Ny; };
    auto ld = [&](int r, int col) { return ldq(base + r * rs + col); };
    const int own_off = (slot + 2) * KP + 4 * l, hal_off = (hs + 2) * KP + 4 * l;
    auto put = [&](int s, int off, Q q) {
        stq(ring + s * ROW + off, q);
        stq(ring + (s + 8) * ROW + off, q);
    };
    // prologue: rows js-3 .. js+2 of the own column, rows js .. js+2 of the halo columns (ring slots 0..5)
    for (int d = -3; d <= 2; ++d) put(d + 3, own_off, ld(modr(js + d), colm));
    if (hal)
        for (int d = 0; d <= 2; ++d) put(d + 3, hal_off, ld(modr(js + d), hcol));
    Q nw = ld(modr(js + 3), colm), hv = hal ? ld(modr(js + 3), hcol) : qz();
    Q vx, vy, vc = {f2(1.f), f2(1.f)};
    auto vload = [&](int r) {
        const int e = r * rs + colm;
        if constexpr (CURR) {
            vx = ldgq(p.ux32 + e);
            vy = ldgq(p.uy32 + e);
        }
        if (cgp) vc = ldgq(p.cgc32 + e);
    };
    // velocities in the fused kernel's order: (c_g * direction table) + U (intrinsic: no U)
    auto velo = [&](Q& ux, Q& uy) {
        ux = gx;
        uy = gy;
        if (cgp) {
            ux = qmul(vc, ux);
            uy = qmul(vc, uy);
        }
        if constexpr (CURR) {
            ux = qadd(ux, vx);
            uy = qadd(uy, vy);
        }
    };
    // fused stage: the inputs of the row being finished, loaded one row ahead (after that row's faces)
    Q pn0 = qz(), plr = qz();
    auto pend = [&](int j) {
        const int off = j * rs + colm;
        if (p.stage != 1) pn0 = ldq(N0n + off);
        if constexpr (FSRC == 3) plr = ldq(p.lin_rates + slice * n + off);
    };
    vload(modr(js));
    Q ux0, uy0;
    velo(ux0, uy0);
    Q uy1 = qz();
    vload(modr(js + 1));
    if (XM == MIX && slot == 0) {
        sg[CX * L + l] = 0;
        sg[(2 * CX + 1) * L + l] = 0;
    }
    __syncthreads();
    const float* q = ring + own_off;
    Q pLy = qz(), pRy = qz();   // the two candidates of the lower y face of the current row
    {
        auto R = [&](int d) { return ldq(q + d * ROW); };     // row js-3+d
        if constexpr (YM == POS) pLy = qweno(R(0), R(1), R(2), R(3), R(4));
        else if constexpr (YM == NEG) pRy = qweno(R(5), R(4), R(3), R(2), R(1));
        else {
            const int need = own ? codeq(uy0) : 0;
            if (__any_sync(FULL, need & 1)) pLy = qweno(R(0), R(1), R(2), R(3), R(4));
            if (__any_sync(FULL, need & 2)) pRy = qweno(R(5), R(4), R(3), R(2), R(1));
        }
    }
    int rl = modr(js + 4), rv = modr(js + 2);
    int sw = 6, sq = 0;                                         // ring slots of rows j+3 and j-3
    const float dxi = p.dx_inv, dyi = p.dy_inv;
    Q Fx_prev = qz(), fy_prev = qz(), ux_prev = qz();
    int outoff = js * rs + colm;
    auto step = [&](int k, auto bufc) {
        constexpr int buf = decltype(bufc)::value;
        const bool row = k < cnt;
        Q ux1 = qz();
        if (row) {
            put(sw, own_off, nw);
            if (hal) put(sw, hal_off, hv);
            if constexpr (XM == MIX) sg[(buf * (CX + 1) + slot) * L + l] = own ? codeq(ux0) : 0;
            velo(ux1, uy1);
            nw = ld(rl, colm);
            if (hal) hv = ld(rl, hcol);
            vload(rv);
        }
        __syncthreads();
        // the previous row: its lower x face from the left neighbour's candidates, then S
        if (k > 0 && slot >= 1) {
            Q Flo;
            if constexpr (XM == MIX) {
                const float* f = fsm + (((1 - buf) * CX + slot - 1) * L + l) * 8;
                Flo = selq(ux_prev, ldq(f), ldq(f + 4));
            } else {
                Flo = ldq(fsm + (((1 - buf) * CX + slot - 1) * L + l) * 4);
            }
            const Q fx = qmuls(qmul(ux_prev, qsub(Fx_prev, Flo)), dxi);
            if constexpr (!FUSED) {
                if (out_ok) stq(Sn + outoff - rs, qadd(fx, fy_prev));
            } else {
                const Q cv = ldq(q + (sq + 2) * ROW);          // the finished row's action
                Q G = {mul2(f2(-1.f), add2(fx.a, fy_prev.a)), mul2(f2(-1.f), add2(fx.b, fy_prev.b))};
                if constexpr (FSRC == 3) {   // SourceTermSet rates of this stage, state layout
                    G.a = fma2(plr.a, cv.a, G.a);
                    G.b = fma2(plr.b, cv.b, G.b);
                }
                auto upd = [&](float2 g, float2 c0, float2 nv) {
                    float2 st = fma2(f2(p.dt), g, c0);
                    st.x = relu(st.x);
                    st.y = relu(st.y);
                    float2 out = st;
                    if (p.stage != 1) {
                        out = fma2(f2(p.a), nv, mul2(f2(p.b), st));
                        out.x = relu(out.x);
                        out.y = relu(out.y);
                    }
                    return out;
                };
                const Q o = {upd(G.a, cv.a, pn0.a), upd(G.b, cv.b, pn0.b)};
                if (out_ok) {
                    if (!isfinite(o.a.x) || !isfinite(o.a.y) || !isfinite(o.b.x) || !isfinite(o.b.y))
                        atomicOr(p.err, 1u);
                    stq(Sn + outoff - rs, o);
                }
            }
        }
        if (!row) return false;
        if constexpr (FUSED) pend(js + k);
        const float* qq = q + sq * ROW;
        auto R = [&](int d) { return ldq(qq + d * ROW); };     // own column, row j-3+d
        const Q c = R(3);
        {
            const float* xr = qq + 3 * ROW - 2 * KP;             // row j
            auto X = [&](int d) { return ldq(xr + (d + 2) * KP); };   // cell slot+d
            if constexpr (XM == POS) {
                const Q F = qweno(X(-2), X(-1), c, X(1), X(2));
                stq(fsm + ((buf * CX + slot) * L + l) * 4, F);
                Fx_prev = F;
            } else if constexpr (XM == NEG) {
                const Q F = qweno(X(3), X(2), X(1), c, X(-1));
                stq(fsm + ((buf * CX + slot) * L + l) * 4, F);
                Fx_prev = F;
            } else {
                const int need = (own ? codeq(ux0) : 0) | sg[(buf * (CX + 1) + slot + 1) * L + l];
                Q Lx = qz(), Rx = qz();
                if (__any_sync(FULL, need & 1)) Lx = qweno(X(-2), X(-1), c, X(1), X(2));
                if (__any_sync(FULL, need & 2)) Rx = qweno(X(3), X(2), X(1), c, X(-1));
                stq(fsm + ((buf * CX + slot) * L + l) * 8, Lx);
                stq(fsm + ((buf * CX + slot) * L + l) * 8 + 4, Rx);
                Fx_prev = selq(ux0, Lx, Rx);
            }
            ux_prev = ux0;
        }
        {
            Q Fhi, Flo;
            if constexpr (YM == POS) {
                Fhi = qweno(R(1), R(2), c, R(4), R(5));
                Flo = pLy;
                pLy = Fhi;
            } else if constexpr (YM == NEG) {
                Fhi = qweno(R(6), R(5), R(4), c, R(2));
                Flo = pRy;
                pRy = Fhi;
            } else {
                const int need = own ? (codeq(uy0) | (k + 1 < cnt ? codeq(uy1) : 0)) : 0;
                Q Ly = qz(), Ry = qz();
                if (__any_sync(FULL, need & 1)) Ly = qweno(R(1), R(2), c, R(4), R(5));
                if (__any_sync(FULL, need & 2)) Ry = qweno(R(6), R(5), R(4), c, R(2));
                Fhi = selq(uy0, Ly, Ry);
                Flo = selq(uy0, pLy, pRy);
                pLy = Ly;
                pRy = Ry;
            }
            fy_prev = qmuls(qmul(uy0, qsub(Fhi, Flo)), dyi);
        }
        ux0 = ux1;
        uy0 = uy1;
        rl = rl + 1 == Ny ? 0 : rl + 1;
        rv = rv + 1 == Ny ? 0 : rv + 1;
        sw = sw + 1 == 8 ? 0 : sw + 1;
        sq = sq + 1 == 8 ? 0 : sq + 1;
        outoff += rs;
        return true;
    };
    for (int k = 0;; k += 2) {
        if (!step(k, std::integral_constant<int, 0>{})) break;
        if (!step(k + 1, std::integral_constant<int, 1>{})) break;
    }
}

__device__ __forceinline__ float4 ld_ratio4(const unsigned* p) {
    const uint4 u = __ldg(reinterpret_cast<const uint4*>(p));
    return make_float4(__uint_as_float(u.x), __uint_as_float(u.y), __uint_as_float(u.z), __uint_as_float(u.w));
}

// One CTA per (direction, x tile, row segment), direction fastest so the CTAs of one region run together.
template <int L, int FSRC>
__global__ void __launch_bounds__(XTHREADS, 2) xyw_kernel(const TileArgs p, int seg0) {
    extern __shared__ __align__(16) float smem[];
    constexpr int CX = Lay<L>::CX;
    const int tiles_x = (p.Nx + CX - 2) / (CX - 1);
    int b = blockIdx.x;
    const int n = b % p.Np;
    b /= p.Np;
    const int tx = b % tiles_x, seg = seg0 + b / tiles_x;
    const int js = max(p.j_lo, seg * XSEG), je = min(p.j_hi, (seg + 1) * XSEG);
    // the uniform test of the thread's four bins against the region's ratios (idle lanes pass)
    const int Nk = p.Nk, m0 = 4 * (threadIdx.x % L), mc = m0 < Nk ? m0 : Nk - 4;
    const int64_t region = (int64_t)seg * tiles_x + tx;
    const float4 rx = ld_ratio4(p.rmax + (2 * region) * Nk + mc);
    const float4 ry = ld_ratio4(p.rmax + (2 * region + 1) * Nk + mc);
    const float4 g0 = __ldg(reinterpret_cast<const float4*>(p.cg32 + mc + Nk * n));
    const float4 g1 = __ldg(reinterpret_cast<const float4*>(p.cg32 + mc + 2 + Nk * n));
    constexpr float SH = 1.0f - 1e-5f;
    auto clear = [](float g, float r) { return fabsf(g) * SH > r; };
    const bool live = m0 < Nk;
    const bool cx = clear(g0.x, rx.x) && clear(g0.z, rx.y) && clear(g1.x, rx.z) && clear(g1.z, rx.w);
    const bool cy = clear(g0.y, ry.x) && clear(g0.w, ry.y) && clear(g1.y, ry.z) && clear(g1.w, ry.w);
    const bool xp = g0.x > 0.f && g0.z > 0.f && g1.x > 0.f && g1.z > 0.f;
    const bool xn = g0.x < 0.f && g0.z < 0.f && g1.x < 0.f && g1.z < 0.f;
    const bool yp = g0.y > 0.f && g0.w > 0.f && g1.y > 0.f && g1.w > 0.f;
    const bool yn = g0.y < 0.f && g0.w < 0.f && g1.y < 0.f && g1.w < 0.f;
    const int allxp = __syncthreads_and(!live || (cx && xp)), allxn = __syncthreads_and(!live || (cx && xn));
    const int allyp = __syncthreads_and(!live || (cy && yp)), allyn = __syncthreads_and(!live || (cy && yn));
    const int xm = allxp ? POS : (allxn ? NEG : MIX);
    const int ym = allyp ? POS : (allyn ? NEG : MIX);
    // the four sign-uniform bodies, else the general one (either axis mixed: 2-5% of the CTAs)
    if (xm == MIX || ym == MIX) xyw_body<L, MIX, MIX, FSRC>(p, smem, n, tx, js, je);
    else if (xm == POS) {
        if (ym == POS) xyw_body<L, POS, POS, FSRC>(p, smem, n, tx, js, je);
        else xyw_body<L, POS, NEG, FSRC>(p, smem, n, tx, js, je);
    } else {
        if (ym == POS) xyw_body<L, NEG, POS, FSRC>(p, smem, n, tx, js, je);
        else xyw_body<L, NEG, NEG, FSRC>(p, smem, n, tx, js, je);
    }
}

// FP32 velocity planes (U_x, U_y, c_g magnitude per (i,j,m), device order) from the coefficient records,
// and per region (x tile of per_tile cells, XSEG rows) and bin m the maxima of |U_x| / c and |U_y| / c
// (c the per-cell c_g magnitude, or 1 when c_g is folded into the direction table), enlarged by 1e-5,
// at rmax[(2 region + axis) Nk + m] as bit patterns (non-negative floats order like them). One thread per
// (bin, column, segment) walks the segment's rows.
__global__ void vel32_kernel(int Nx, int Ny, int Nk, int per_tile, int tiles_x, const double* __restrict__ coef,
                             int cg_per_cell, float* ux32, float* uy32, float* cgc32, unsigned* rmax) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int nseg = (Ny + XSEG - 1) / XSEG;
    if (t >= (int64_t)Nk * Nx * nseg) return;
    const int m = (int)(t % Nk), i = (int)((t / Nk) % Nx), seg = (int)(t / ((int64_t)Nk * Nx));
    float rx = 0.f, ry = 0.f;
    const float inf = __int_as_float(0x7f800000);
    for (int j = seg * XSEG; j < min(Ny, (seg + 1) * XSEG); ++j) {
        const int64_t e = ((int64_t)j * Nx + i) * Nk + m;
        const double* r = coef + 8 * e;
        const float ux = (float)r[0], uy = (float)r[1], cm = (float)r[6];
        if (ux32) {
            ux32[e] = ux;
            uy32[e] = uy;
        }
        cgc32[e] = cm;
        const float c = cg_per_cell ? cm : 1.0f;
        rx = fmaxf(rx, c > 0.f ? fabsf(ux) / c * (1.0f + 1e-5f) : inf);
        ry = fmaxf(ry, c > 0.f ? fabsf(uy) / c * (1.0f + 1e-5f) : inf);
    }
    const int64_t region = (int64_t)seg * tiles_x + i / per_tile;
    atomicMax(rmax + (2 * region) * Nk + m, __float_as_uint(rx));
    atomicMax(rmax + (2 * region + 1) * Nk + m, __float_as_uint(ry));
}

template <int L, int FSRC>
cudaError_t launch_xyw_L(const TileArgs& a, cudaStream_t s) {
    constexpr int CX = Lay<L>::CX;
    const size_t smem = Lay<L>::bytes;
    const int tiles_x = (a.Nx + CX - 2) / (CX - 1);
    const int seg0 = a.j_lo / XSEG, seg1 = (a.j_hi - 1) / XSEG;
    const int64_t blocks = (int64_t)a.Np * tiles_x * (seg1 - seg0 + 1);
    auto k = xyw_kernel<L, FSRC>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<(unsigned)blocks, XTHREADS, smem, s>>>(a, seg0);
    return cudaGetLastError();
}

}  // namespace

int xyw_lanes(int64_t Nk) { return Nk <= 4 ? 1 : (Nk <= 8 ? 2 : (Nk <= 16 ? 4 : 8)); }

int64_t xyw_regions(const Handle& h) {
    const int per_tile = XTHREADS / xyw_lanes(h.desc.Nk) - 1;
    return ((h.desc.Nx + per_tile - 1) / per_tile) * ((h.desc.Ny + XSEG - 1) / XSEG);
}

bool xyw_supported(const Handle& h) {
    const rpl_desc& d = h.desc;
    // offsets within one direction slice are 32-bit
    return d.Nx * d.Ny * d.Nk < (int64_t)1 << 31 && d.Nx >= 3 && d.Ny >= 3;
}

cudaError_t launch_vel32(const Handle& h, cudaStream_t s) {
    if (!h.d_vel32) return cudaSuccess;
    const rpl_desc& d = h.desc;
    const int64_t c3 = d.Nx * d.Ny * d.Nk;
    const int per_tile = XTHREADS / xyw_lanes(d.Nk) - 1;
    const int tiles_x = (int)((d.Nx + per_tile - 1) / per_tile);
    cudaError_t e = cudaMemsetAsync(h.d_rmax, 0, 2 * h.vel_regions * d.Nk * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    const int64_t threads = d.Nk * d.Nx * ((d.Ny + XSEG - 1) / XSEG);
    // refraction: U_x, U_y and c_g planes; intrinsic transport (no currents): the c_g plane only
    const bool refract = d.transport == RPL_TRANSPORT_REFRACTION;
    float* ux = refract ? h.d_vel32 : nullptr;
    float* uy = refract ? h.d_vel32 + c3 : nullptr;
    float* cg = refract ? h.d_vel32 + 2 * c3 : h.d_vel32;
    vel32_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>((int)d.Nx, (int)d.Ny, (int)d.Nk, per_tile, tiles_x,
                                                                h.d_coef, h.d_cgmag != nullptr, ux, uy, cg,
                                                                h.d_rmax);
    return cudaGetLastError();
}

template <int FSRC>
cudaError_t launch_lanes(const TileArgs& a, cudaStream_t s) {
    switch (xyw_lanes(a.Nk)) {
        case 1: return launch_xyw_L<1, FSRC>(a, s);
        case 2: return launch_xyw_L<2, FSRC>(a, s);
        case 4: return launch_xyw_L<4, FSRC>(a, s);
        default: return launch_xyw_L<8, FSRC>(a, s);
    }
}

cudaError_t launch_xyw(const TileArgs& a, cudaStream_t s) { return launch_lanes<-1>(a, s); }

cudaError_t launch_xy_intrinsic(const TileArgs& a, cudaStream_t s) { return launch_lanes<-2>(a, s); }

cudaError_t launch_xyi(const TileArgs& a, int src, cudaStream_t s) {
    if (src != 0 && src != 3) return cudaErrorInvalidValue;
    return src == 0 ? launch_lanes<0>(a, s) : launch_lanes<3>(a, s);
}

}  // namespace rpl
