// Tracer advection with flux-corrected transport on the device:
//   ATMOS_DYN_Tstep_tracer_fvm_heve  scale_atmos_dyn_tstep_tracer_fvm_heve.F90:72-240
//   ATMOS_DYN_fct / get_fact_fct     scale_atmos_dyn_common.F90:1922-2734
//   UD1 low-order fluxes             scale_atmos_dyn_fvm_flux_ud1.F90:135-294
//
// A stage without FCT is one kernel (every cell forms its six face fluxes and
// updates). With FCT the limiter needs the low-order solution and the
// limiting factors of the neighbours, so the stage splits at the halo fill of
// R+/R- (the reference's mid-limiter COMM_vars8, :2558-2561). Its fused form:
//   k_fct_limit   a CTA owns 8 columns (4 in FP32) x 32 levels and marches
//                 along j over a strip of rows; QTRC0 rows come into a ring in
//                 shared memory by bulk tensor copies (TMA, two rows ahead,
//                 bounded mbarrier waits). Per row it forms the low-order
//                 solution phi_lo of the tile and a halo of one in shared
//                 memory, the high- and low-order fluxes of every face of the
//                 tile and their differences (the anti-diffusive fluxes: z by
//                 warp shuffle, both x faces by each column's warp, y carried
//                 from the row before), and from them P+/P-, the along-stream
//                 or 7-point bounds Q+/Q- and R+/R-. Only R+/R- and a copy of
//                 R(QTRC0) for k_fct_update leave the kernel.
//   k_fct_update  forms each face's high- and low-order fluxes again, limits
//                 their difference with R+/R- and updates the tracer.
// The three-kernel form (k_fct_lo: phi_lo and the anti-diffusive fluxes to
// HBM; k_fct_r: R+/R-; k_fct_apply) runs where QTRC0 admits no tensor map or
// no status word is given. Both forms evaluate every value with the same
// operations in the same order: on the FP64 path they give identical bits.
//
// R is the type of the flux and limiter arithmetic and of the flux-like arrays:
// double on the plain path (bit-identical to the oracle), float on the
// mixed-precision path, where the tracer values, the densities and the update
// of the tracer stay FP64 and every FP64 operand enters the fluxes and the
// limiter converted with R(...) at its use (the identity for R = double). The
// limiter's zero tests compare with the FP64 epsilon on both paths (a normal
// FP32 number): they ask whether a velocity or an anti-diffusive change is zero
// at the resolution of the FP64 state, and FP32's own epsilon would switch off
// the limiting of every change below 1.2e-7 that the FP64 path limits.
#include "hevi_kernels.cuh"
#include "tma_util.cuh"

namespace hevi {

// EPSILON(0.0_DP) of the reference's zero tests, in the arithmetic type
template <typename R> __device__ __forceinline__ R eps_of() { return R(EPS); }

// stage density, tinteg_tracer_rk3.F90:140-147 / :168-175
template <typename R>
__device__ __forceinline__ double dens_of(const TracerArgsT<R> &a, size_t c)
{
    const double d = ld(a.DENS + c);
    if (a.dens_mode == 0) return d;
    const double d0 = ld(a.DENS0 + c);
    return a.dens_mode == 1 ? d0 + (d - d0) / 3.0 : d0 + (d - d0) * 0.5;
}

// the num_diff term of a high-order flux; with terrain GSQRT times it, at the
// staggering of the face (fluxZ/X/Y_XYZ: I_XYW, I_UYZ, I_XVZ)
template <typename R>
__device__ __forceinline__ R ndq_at(const TracerArgsT<R> &a, size_t N3, int dir, size_t c)
{
    const R nd = a.ndq ? ld(a.ndq + (size_t)dir * N3 + c) : R(0.0);
    if (!a.GS) return nd;
    const int slice = dir == 0 ? 1 : dir == 1 ? 4 : 5; // I_XYW, I_UYZ, I_XVZ (0-based)
    return R(ld(a.GS + (size_t)slice * N3 + c) * (double)nd);
}
// x * MAPF(i,j,1) * MAPF(i,j,2) / GSQRT(k,i,j,I_XYZ) with terrain, x on flat terrain
// (the metric factor of every flux divergence, tstep_tracer_fvm_heve.F90:188-236,
// common.F90:2051-2120)
template <typename R>
__device__ __forceinline__ R mfac(const Grid &g, const TracerArgsT<R> &a, R x, int i, int j, size_t c)
{
    if (!a.GS) return x;
    const size_t p = (size_t)(i - 1) + (size_t)g.IA * (size_t)(j - 1);
    return R((double)x * ld(a.MAPF + p) * ld(a.MAPF + p + (size_t)g.IA * g.JA) / ld(a.GS + c));
}

// high-order z flux at the face above level m (fluxZ_XYZ, ud3.F90:157-247, ud5.F90:194-321)
template <int S, typename R>
__device__ R hflux_z(const Grid &g, const TracerArgsT<R> &a, size_t N3, size_t col, int m)
{
    if (m < g.KS || m > g.KE - 1) return R(0.0);
    const double *q = a.QTRC + col - 1;
    const R vel = ld(a.mflx + col + m - 1);
    const R v = zface<S>(vel, m, g.KS, g.KE, [&](int l) { return R(ld(q + l)); });
    return vel * v + ndq_at(a, N3, 0, col + m - 1);
}
// high-order flux at the face between c and c+s (fluxX/Y_XYZ, ud3.F90:251-353); dir 1 = x, 2 = y
template <int S, typename R>
__device__ __forceinline__ R hflux_h(const TracerArgsT<R> &a, size_t N3, int dir, size_t c, long s)
{
    const R vel = ld(a.mflx + (size_t)dir * N3 + c);
    const double *q = a.QTRC + c;
    constexpr bool W6 = wide_scheme(S);
    return vel * ip6<S>(vel, W6 ? R(ld(q - 2 * s)) : R(0.0), R(ld(q - s)), R(ld(q)), R(ld(q + s)), R(ld(q + 2 * s)),
                        W6 ? R(ld(q + 3 * s)) : R(0.0))
           + ndq_at(a, N3, dir, c);
}
// donor-cell flux of mass flux vel between the values lo (below / west /
// south) and hi (ud1.F90:155-165)
template <typename R>
__device__ __forceinline__ R lflux_v(R vel, R lo, R hi)
{
    return vel * (R(0.5) * (hi + lo) - fsign(R(0.5), vel) * (hi - lo));
}
// donor-cell flux at the face between c and c+s
template <typename R>
__device__ __forceinline__ R lflux(const TracerArgsT<R> &a, size_t N3, int dir, size_t c, long s)
{
    return lflux_v(ld(a.mflx + (size_t)dir * N3 + c), R(ld(a.QTRC0 + c)), R(ld(a.QTRC0 + c + s)));
}

// ---- stage without FCT, tstep_tracer_fvm_heve.F90:214-236 -------------------
// CTAs per SM of the two warp-per-column tracer kernels, which are bound by
// load latency: 16 (32 registers) for k_tracer_plain and 12 (40 registers)
// for k_fct_update, against 48 and 64 registers unbounded (512x512x128, UD3:
// 6.69 -> 5.92 ms per FP64 tracer step, 5.19 -> 4.68 ms mixed; 16 CTAs for
// k_fct_update spill 400 B and took 7.80 ms)
#ifndef HEVI_TR_MINB
#define HEVI_TR_MINB 16
#endif
#ifndef HEVI_UPD_MINB
#define HEVI_UPD_MINB 12
#endif
#define HEVI_TR_BOUNDS __launch_bounds__(128, HEVI_TR_MINB)
#define HEVI_UPD_BOUNDS __launch_bounds__(128, HEVI_UPD_MINB)
template <int S, typename R>
__global__ void HEVI_TR_BOUNDS k_tracer_plain(const Grid g, const TracerArgsT<R> a)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const size_t col = idx3(g, 1, i, j);
    const R rcdx = R(ld(g.RCDX + i - 1)), rcdy = R(ld(g.RCDY + j - 1));
    // the z flux through the face above a level; the face below is the previous
    // lane's (lane 0: the previous pass's lane 31; zero below KS)
    R carry = R(0.0);
    for (int k0 = g.KS; k0 <= g.KE; k0 += 32) {
        const int k = k0 + threadIdx.x;
        const bool ok = k <= g.KE;
        const size_t c = col + k - 1;
        const R hz = ok ? hflux_z<S>(g, a, N3, col, k) : R(0.0);
        R hzm = __shfl_up_sync(0xffffffffu, hz, 1);
        if (threadIdx.x == 0) hzm = carry;
        carry = __shfl_sync(0xffffffffu, hz, 31);
        if (!ok) continue;
        const R hx = hflux_h<S>(a, N3, 1, c, sI), hxm = hflux_h<S>(a, N3, 1, c - sI, sI);
        const R hy = hflux_h<S>(a, N3, 2, c, sJ), hym = hflux_h<S>(a, N3, 2, c - sJ, sJ);
        const R div = (hz - hzm) * R(ld(g.RCDZ + k - 1)) + (hx - hxm) * rcdx + (hy - hym) * rcdy;
        a.QTRCo[c] = (ld(a.QTRC0 + c) * ld(a.DENS0 + c) + a.dtl * (double)(mfac(g, a, -div, i, j, c) + ld(a.RHOQ_t + c)))
                     / dens_of(a, c);
    }
}

// ---- FCT part 1: low-order solution and raw anti-diffusive fluxes (common.F90:1990-2073) ----
template <int S, typename R>
__global__ void __launch_bounds__(128) k_fct_lo(const Grid g, const TracerArgsT<R> a)
{
    // columns i in IS-1..IE+1, j in JS-1..JE+1
    const int i = g.IS - 1 + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS - 1 + blockIdx.y;
    if (i > g.IE + 1) return;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const size_t col = idx3(g, 1, i, j);
    const bool inter = (i >= g.IS && i <= g.IE && j >= g.JS && j <= g.JE);
    const R rcdx = R(ld(g.RCDX + i - 1)), rcdy = R(ld(g.RCDY + j - 1));
    for (int k = g.KS + threadIdx.x; k <= g.KE; k += 32) {
        const size_t c = col + k - 1;
        const R lz = (k <= g.KE - 1) ? lflux(a, N3, 0, c, 1) : R(0.0);
        const R lzm = (k >= g.KS + 1) ? lflux(a, N3, 0, c - 1, 1) : R(0.0);
        const R lx = lflux(a, N3, 1, c, sI), lxm = lflux(a, N3, 1, c - sI, sI);
        const R ly = lflux(a, N3, 2, c, sJ), lym = lflux(a, N3, 2, c - sJ, sJ);
        a.phi_lo[c] = R((ld(a.QTRC0 + c) * ld(a.DENS0 + c)
                         + a.dtl * (double)mfac(g, a, -((lz - lzm) * R(ld(g.RCDZ + k - 1)) + (lx - lxm) * rcdx + (ly - lym) * rcdy),
                                                i, j, c))
                        / ld(a.DENS + c));
        if (inter) {
            R *aZ = a.anti, *aX = a.anti + N3, *aY = a.anti + 2 * N3;
            aZ[c] = (k <= g.KE - 1) ? hflux_z<S>(g, a, N3, col, k) - lz : R(0.0);
            if (k == g.KS) aZ[c - 1] = R(0.0);
            aX[c] = hflux_h<S>(a, N3, 1, c, sI) - lx;
            aY[c] = hflux_h<S>(a, N3, 2, c, sJ) - ly;
            if (i == g.IS) aX[c - sI] = hflux_h<S>(a, N3, 1, c - sI, sI) - lxm;
            if (j == g.JS) aY[c - sJ] = hflux_h<S>(a, N3, 2, c - sJ, sJ) - lym;
        }
    }
}

// get_fact_fct, common.F90:2676-2734; f[a][b+1][c+1] = fact(a,b,c)
template <typename R>
__device__ __forceinline__ void fact_fct(R f[2][3][3], R rw, R ru, R rv)
{
    const R h = R(0.5), one = R(1.0), eps = eps_of<R>();
    const R ugev = fsign(h, fabs(ru) - fabs(rv)) + h;
    const R ugew = fsign(h, fabs(ru) - fabs(rw)) + h;
    const R vgew = fsign(h, fabs(rv) - fabs(rw)) + h;
    const R uzero = fsign(h, fabs(ru) - eps) - h;
    const R vzero = fsign(h, fabs(rv) - eps) - h;
    const R wzero = fsign(h, fabs(rw) - eps) - h;
    const R sign_uv = fsign(h, ru * rv) + h;
    const R sign_uw = fsign(h, ru * rw) + h;
    const R sign_vw = fsign(h, rv * rw) + h;
    const R wu = fabs(rw / (ru + uzero) * (one + uzero));
    const R vu = fabs(rv / (ru + uzero) * (one + uzero));
    const R uv = fabs(ru / (rv + vzero) * (one + vzero));
    const R wv = fabs(rw / (rv + vzero) * (one + vzero));
    const R uw = fabs(ru / (rw + wzero) * (one + wzero));
    const R vw = fabs(rv / (rw + wzero) * (one + wzero));
    const R umax = ugev * ugew * (one + uzero);
    const R vmax = (one - ugev) * vgew;
    const R wmax = one - ugev * ugew - vmax;
    const R tri = umax * vu * wu + vmax * uv * wv + wmax * uw * vw;
    const R xz = ugew * wu * (one - vu) + (one - ugew) * uw * (one - vw);
    const R yz = vgew * wv * (one - uv) + (one - vgew) * vw * (one - uw);
    const R xy = ugev * vu * (one - wu) + (one - ugev) * uv * (one - wv);
#define FF(x, y, z) f[x][(y) + 1][(z) + 1]
    FF(0, 0, 0) = -ugev * ugew * uzero;
    FF(1, 0, 0) = wmax * (one - uw) * (one - vw);
    FF(0, 1, 0) = umax * (one - vu) * (one - wu);
    FF(0, 0, 1) = vmax * (one - uv) * (one - wv);
    FF(1, 1, 1) = sign_uv * sign_uw * tri;
    FF(1, -1, 1) = (one - sign_uv) * (one - sign_uw) * tri;
    FF(1, 1, -1) = (one - sign_uv) * sign_uw * tri;
    FF(1, -1, -1) = sign_uv * (one - sign_uw) * tri;
    FF(1, 1, 0) = sign_uw * (one - vmax) * xz;
    FF(1, -1, 0) = (one - sign_uw) * (one - vmax) * xz;
    FF(1, 0, 1) = sign_vw * (one - umax) * yz;
    FF(1, 0, -1) = (one - sign_vw) * (one - umax) * yz;
    FF(0, 1, 1) = sign_uv * (one - wmax) * xy;
    FF(0, 1, -1) = (one - sign_uv) * (one - wmax) * xy;
#undef FF
}

// ---- FCT part 2: limiting factors R+ and R- (common.F90:2079-2553) ----------
template <typename R>
__global__ void __launch_bounds__(128, 4) k_fct_r(const Grid g, const TracerArgsT<R> a)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const size_t col = idx3(g, 1, i, j);
    const R *aZ = a.anti, *aX = a.anti + N3, *aY = a.anti + 2 * N3;
    const R *mZ = a.mflx, *mX = a.mflx + N3, *mY = a.mflx + 2 * N3;
    const R rdx = R(ld(g.RCDX + i - 1)), rdy = R(ld(g.RCDY + j - 1));
    const R zero = R(0.0), one = R(1.0), h = R(0.5), eps = eps_of<R>(), dtl = R(a.dtl);
    const int KS = g.KS, KE = g.KE;
    for (int k = KS + threadIdx.x; k <= KE; k += 32) {
        const size_t c = col + k - 1;
        const R rdz = R(ld(g.RCDZ + k - 1));
        // net incoming / outgoing anti-diffusive change :2077-2120
        const R pz = rmax(zero, ld(aZ + c - 1)) - rmin(zero, ld(aZ + c));
        const R px = rmax(zero, ld(aX + c - sI)) - rmin(zero, ld(aX + c));
        const R py = rmax(zero, ld(aY + c - sJ)) - rmin(zero, ld(aY + c));
        const R pjpls = mfac(g, a, dtl * (pz * rdz + px * rdx + py * rdy), i, j, c);
        const R mz = rmax(zero, ld(aZ + c)) - rmin(zero, ld(aZ + c - 1));
        const R mx = rmax(zero, ld(aX + c)) - rmin(zero, ld(aX + c - sI));
        const R my = rmax(zero, ld(aY + c)) - rmin(zero, ld(aY + c - sJ));
        const R pjmns = mfac(g, a, dtl * (mz * rdz + mx * rdx + my * rdy), i, j, c);

        const double *PI = a.QTRC0 + c;
        const R *PL = a.phi_lo + c;
        R qmax, qmin;
        if (a.along_stream) {
            // along-stream bound :2126-2369; ka / kb are the levels of the upstream
            // and downstream (1,*,*) points (clamped at KS and KE as the reference does)
            R rw;
            long ka, kb;
            if (k == KS) { rw = ld(mZ + c) * rdz; ka = 1; kb = 0; }
            else if (k == KE) { rw = ld(mZ + c - 1) * rdz; ka = 0; kb = -1; }
            else { rw = (ld(mZ + c) + ld(mZ + c - 1)) * rdz; ka = 1; kb = -1; }
            const R ru = (ld(mX + c) + ld(mX + c - sI)) * rdx;
            const R rv = (ld(mY + c) + ld(mY + c - sJ)) * rdy;
            R f[2][3][3];
            fact_fct(f, rw, ru, rv);
#define FA(x, y, z) f[x][(y) + 1][(z) + 1]
#define V(P, o) R(ld(P + (o)))
#define QA(P) (FA(1, 1, 1) * V(P, ka + sI + sJ) + FA(0, 1, 1) * V(P, sI + sJ) + FA(1, 0, 1) * V(P, ka + sJ)    \
               + FA(0, 0, 1) * V(P, sJ) + FA(1, -1, 1) * V(P, ka - sI + sJ) + FA(1, 1, 0) * V(P, ka + sI)      \
               + FA(0, 1, 0) * V(P, sI) + FA(1, 0, 0) * V(P, ka) + FA(1, -1, 0) * V(P, ka - sI)                 \
               + FA(1, 1, -1) * V(P, ka + sI - sJ) + FA(0, 1, -1) * V(P, sI - sJ) + FA(1, 0, -1) * V(P, ka - sJ) \
               + FA(1, -1, -1) * V(P, ka - sI - sJ) + FA(0, 0, 0) * V(P, 0))
#define QB(P) (FA(1, 1, 1) * V(P, kb - sI - sJ) + FA(0, 1, 1) * V(P, -sI - sJ) + FA(1, 0, 1) * V(P, kb - sJ)    \
               + FA(0, 0, 1) * V(P, -sJ) + FA(1, -1, 1) * V(P, kb + sI - sJ) + FA(1, 1, 0) * V(P, kb - sI)      \
               + FA(0, 1, 0) * V(P, -sI) + FA(1, 0, 0) * V(P, kb) + FA(1, -1, 0) * V(P, kb + sI)                 \
               + FA(1, 1, -1) * V(P, kb - sI + sJ) + FA(0, 1, -1) * V(P, -sI - sJ) + FA(1, 0, -1) * V(P, kb - sJ) \
               + FA(1, -1, -1) * V(P, kb + sI + sJ) + FA(0, 0, 0) * V(P, 0))
            const R qa_in = QA(PI), qb_in = QB(PI), qa_lo = QA(PL), qb_lo = QB(PL);
#undef QA
#undef QB
#undef V
#undef FA
            const R pin = R(ld(PI)), plo = ld(PL);
            qmax = rmax(rmax(rmax(rmax(rmax(pin, qa_in), qb_in), plo), qa_lo), qb_lo);
            qmin = rmin(rmin(rmin(rmin(rmin(pin, qa_in), qb_in), plo), qa_lo), qb_lo);
        } else {
            // 7-point bound :2370-2515
            const R pin = R(ld(PI)), plo = ld(PL);
            qmax = rmax(pin, plo);
            qmin = rmin(pin, plo);
            const long nb[6] = {1, -1, sI, -sI, sJ, -sJ};
            for (int n = 0; n < 6; ++n) {
                if ((k == KS && nb[n] == -1) || (k == KE && nb[n] == 1)) continue;
                const R x = R(ld(PI + nb[n])), y = ld(PL + nb[n]);
                qmax = rmax(rmax(qmax, x), y);
                qmin = rmin(rmin(qmin, x), y);
            }
        }
        const R dn = R(ld(a.DENS + c)), plo = ld(PL);
        const R qjpls = (qmax - plo) * dn;
        const R qjmns = (plo - qmin) * dn;
        R zerosw = h - fsign(h, pjpls - eps);
        a.rjp[c] = rmin(one, qjpls * (one - zerosw) / (pjpls - zerosw));
        zerosw = h - fsign(h, pjmns - eps);
        a.rjm[c] = rmin(one, qjmns * (one - zerosw) / (pjmns - zerosw));
    }
}

// limited anti-diffusive flux at the face between c and c+s (common.F90:2563-2660)
template <typename R>
__device__ __forceinline__ R limit(const TracerArgsT<R> &a, R anti, size_t c, long s)
{
    const R dirsw = R(0.5) + fsign(R(0.5), anti);
    return anti * (R(1.0) - rmin(ld(a.rjp + c + s), ld(a.rjm + c)) * (dirsw)
                   - rmin(ld(a.rjp + c), ld(a.rjm + c + s)) * (R(1.0) - dirsw));
}

// ---- FCT part 3: limit and update (tstep_tracer_fvm_heve.F90:188-210) ------
template <int S, typename R>
__global__ void __launch_bounds__(128) k_fct_apply(const Grid g, const TracerArgsT<R> a)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const size_t col = idx3(g, 1, i, j);
    const R *aZ = a.anti, *aX = a.anti + N3, *aY = a.anti + 2 * N3;
    const R rcdx = R(ld(g.RCDX + i - 1)), rcdy = R(ld(g.RCDY + j - 1));
    for (int k = g.KS + threadIdx.x; k <= g.KE; k += 32) {
        const size_t c = col + k - 1;
        const R az = (k <= g.KE - 1) ? limit(a, ld(aZ + c), c, 1) : R(0.0);
        const R azm = (k >= g.KS + 1) ? limit(a, ld(aZ + c - 1), c - 1, 1) : R(0.0);
        const R ax = limit(a, ld(aX + c), c, sI), axm = limit(a, ld(aX + c - sI), c - sI, sI);
        const R ay = limit(a, ld(aY + c), c, sJ), aym = limit(a, ld(aY + c - sJ), c - sJ, sJ);
        const R hz = hflux_z<S>(g, a, N3, col, k), hzm = hflux_z<S>(g, a, N3, col, k - 1);
        const R hx = hflux_h<S>(a, N3, 1, c, sI), hxm = hflux_h<S>(a, N3, 1, c - sI, sI);
        const R hy = hflux_h<S>(a, N3, 2, c, sJ), hym = hflux_h<S>(a, N3, 2, c - sJ, sJ);
        const R div = (hz - az - hzm + azm) * R(ld(g.RCDZ + k - 1)) + (hx - ax - hxm + axm) * rcdx
                      + (hy - ay - hym + aym) * rcdy;
        a.QTRCo[c] = (ld(a.QTRC0 + c) * ld(a.DENS0 + c) + a.dtl * (double)(mfac(g, a, -div, i, j, c) + ld(a.RHOQ_t + c)))
                     / ld(a.DENS + c);
    }
}

// =============================================================================
// fused form: k_fct_limit, k_fct_update
// =============================================================================
namespace fct {
#ifndef HEVI_FCT_JB
#define HEVI_FCT_JB 16
#endif
// tile width and CTAs per SM (measured on 512x512x128, UD3, along-stream):
// FP64 8 columns, 4 CTAs (64 registers); FP32 4 columns, 8 CTAs
#ifndef HEVI_FCT_FW
#ifdef HEVI_FLOAT_TU
#define HEVI_FCT_FW 4
#define HEVI_FCT_MINB 8
#else
#define HEVI_FCT_FW 8
#define HEVI_FCT_MINB 4
#endif
#endif
constexpr int FW = HEVI_FCT_FW;  // tile columns along i, one warp each
constexpr int KC = 32;           // levels of a CTA, one per lane
constexpr int BK = 38;           // staged levels of a QTRC0 row (a 16-byte multiple) from L0-2 or one below
constexpr int BW = FW + 4;       // staged columns: i0-2 .. i0+FW+1
constexpr int SLOT = (BK * BW + 15) / 16 * 16; // doubles per staged row, padded to 128 bytes
constexpr int NS = 6;            // staged rows in the ring
constexpr int PK = KC + 2;       // phi_lo levels: L0-1 .. L0+KC
constexpr int PW = FW + 2;       // phi_lo columns: i0-1 .. i0+FW
constexpr int NP = 4;            // phi_lo rows in the ring
constexpr int JB = HEVI_FCT_JB;  // rows of a CTA's strip
constexpr unsigned ROW_BYTES = BK * BW * sizeof(double);
template <typename R> constexpr size_t smem_bytes()
{
    return (size_t)NS * SLOT * sizeof(double) + NS * sizeof(uint64_t) + (size_t)NP * PW * PK * sizeof(R);
}
}  // namespace fct

// the along-stream weighted sums qa and qb of one field around a cell
// (common.F90:2143-2170; the same terms at KS and KE with ka, kb clamped);
// v(dk, di, dj) is the field at (k+dk, i+di, j+dj). qb reads (k, i-1, j-1)
// for fact(0,1,-1) and (k-1, i, j-1) for fact(1,0,-1) as the reference does.
template <typename R, class V>
__device__ __forceinline__ R qa_sum(const R (&f)[2][3][3], int ka, const V &v)
{
#define FA(x, y, z) f[x][(y) + 1][(z) + 1]
    return FA(1, 1, 1) * v(ka, 1, 1) + FA(0, 1, 1) * v(0, 1, 1) + FA(1, 0, 1) * v(ka, 0, 1) + FA(0, 0, 1) * v(0, 0, 1)
           + FA(1, -1, 1) * v(ka, -1, 1) + FA(1, 1, 0) * v(ka, 1, 0) + FA(0, 1, 0) * v(0, 1, 0)
           + FA(1, 0, 0) * v(ka, 0, 0) + FA(1, -1, 0) * v(ka, -1, 0) + FA(1, 1, -1) * v(ka, 1, -1)
           + FA(0, 1, -1) * v(0, 1, -1) + FA(1, 0, -1) * v(ka, 0, -1) + FA(1, -1, -1) * v(ka, -1, -1)
           + FA(0, 0, 0) * v(0, 0, 0);
}
template <typename R, class V>
__device__ __forceinline__ R qb_sum(const R (&f)[2][3][3], int kb, const V &v)
{
    return FA(1, 1, 1) * v(kb, -1, -1) + FA(0, 1, 1) * v(0, -1, -1) + FA(1, 0, 1) * v(kb, 0, -1)
           + FA(0, 0, 1) * v(0, 0, -1) + FA(1, -1, 1) * v(kb, 1, -1) + FA(1, 1, 0) * v(kb, -1, 0)
           + FA(0, 1, 0) * v(0, -1, 0) + FA(1, 0, 0) * v(kb, 0, 0) + FA(1, -1, 0) * v(kb, 1, 0)
           + FA(1, 1, -1) * v(kb, -1, 1) + FA(0, 1, -1) * v(0, -1, -1) + FA(1, 0, -1) * v(kb, 0, -1)
           + FA(1, -1, -1) * v(kb, 1, 1) + FA(0, 0, 0) * v(0, 0, 0);
#undef FA
}

// R+/R- of the cells of a strip (common.F90:1990-2553 without the halo fill),
// and R(QTRC0) of the cells and their lateral halo ring into the phi_lo
// scratch for k_fct_update (phi_lo itself stays in shared memory).
// Block (32, FW): lane = level L0+lane, warp w = column i0+w; the CTA marches
// over rows jb0 .. jb0+nrow-1. Iteration t forms phi_lo of row r = jb0-1+t and,
// from t = 2, R+/R- of row o = r-1, with one CTA barrier per iteration (after
// phi_lo; each warp forms both x faces of its column). QTRC0 row jb0-2+rr
// sits in ring slot rr % NS (mbarrier rr % NS, phase rr / NS); rows rr = 0..3
// are copied before the march, row t+3 is waited for before the barrier of
// iteration t and row t+4 is copied after it, so a slot is refilled only after
// the iteration that last read it has ended everywhere, and a phi_lo slot is
// rewritten only after the barrier that follows its last reads.
template <int S, typename R>
__global__ void __launch_bounds__(32 * fct::FW, HEVI_FCT_MINB)
    k_fct_limit(const Grid g, const TracerArgsT<R> a, const __grid_constant__ CUtensorMap map)
{
    using namespace fct;
    using namespace tma;
    extern __shared__ __align__(1024) double fsm[];
    double *spi = fsm;                                               // QTRC0 rows [slot][i][k]
    uint64_t *bar = reinterpret_cast<uint64_t *>(spi + NS * SLOT);   // one mbarrier per slot
    R *spl = reinterpret_cast<R *>(bar + NS);                        // phi_lo rows [slot][i][k]
    // staging status, double-buffered: with one barrier per iteration, thread 0
    // writes iteration t+1's word while others may still read iteration t's
    __shared__ int s_ok[2];
    const int lane = threadIdx.x, w = threadIdx.y, tid = w * 32 + lane;
    const int nti = (g.IMAX + FW - 1) / FW;
    const int i0 = g.IS + ((int)blockIdx.x % nti) * FW, L0 = g.KS + ((int)blockIdx.x / nti) * KC;
    const int jb0 = g.JS + (int)blockIdx.y * JB;
    const int nrow = min(JB, g.JE - jb0 + 1);
    const int rlast = nrow + 3;        // last ring row: QTRC0 rows jb0-2 .. jb0+nrow+1
    const int kx = (L0 - 3) & ~1;      // 0-based first staged level (level L0-2 or one below): even, a 16-byte start
    const int KS = g.KS, KE = g.KE;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const R *mZ = a.mflx, *mX = a.mflx + N3, *mY = a.mflx + 2 * N3;

    auto issue = [&](int rr) { // thread 0
        uint64_t *b = bar + rr % NS;
        mbar_expect_tx(b, ROW_BYTES);
        tma_load_3d(spi + (rr % NS) * SLOT, &map, kx, i0 - 3, jb0 - 3 + rr, b);
    };
    auto wait_row = [&](int rr) { return mbar_wait(bar + rr % NS, (unsigned)(rr / NS) & 1u); };
    // staged QTRC0 and phi_lo at level kk, column ii of row j
    auto PI = [&](int j, int kk, int ii) -> double {
        return spi[((j - jb0 + 2) % NS) * SLOT + (ii - i0 + 2) * BK + (kk - 1 - kx)];
    };
    auto PL = [&](int j, int kk, int ii) -> R { return spl[((j - jb0 + 1) % NP) * (PW * PK) + (ii - i0 + 1) * PK + (kk - L0 + 1)]; };

    if (tid == 0) {
        for (int q = 0; q < NS; ++q) mbar_init(bar + q, 1);
        fence_mbar_init();
        for (int rr = 0; rr < 4; ++rr) issue(rr);
        const bool ok = wait_row(0) && wait_row(1) && wait_row(2);
        if (!ok)
            for (int rr = 0; rr < 4; ++rr) (void)wait_row(rr); // bounded: the copies still in flight
        s_ok[1] = ok ? 1 : 0;
    }
    __syncthreads();
    if (!s_ok[1]) {
        if (tid == 0) atomicOr(a.status, ST_TMA_TIMEOUT);
        return; // block-uniform
    }
    for (int rr = 0; rr < 3; ++rr) (void)mbar_try(bar + rr, 0u); // completed phases: the copies are visible here

    const int i = i0 + w, k = L0 + lane;
    const bool cell = i <= g.IE && k <= KE;
    const R zero = R(0.0), one = R(1.0), h = R(0.5), eps = eps_of<R>(), dtl = R(a.dtl);
    const R rdx = cell ? R(ld(g.RCDX + i - 1)) : zero;
    const R rdz = cell ? R(ld(g.RCDZ + k - 1)) : zero;
    R ay_prev = zero; // anti-diffusive y flux through the face j+1/2 of the row before

    for (int t = 0; t <= nrow + 1; ++t) {
        const int r = jb0 - 1 + t;
        // (a) phi_lo of row r on the tile and a halo of one (common.F90:1990-2073)
        {
            R *pl = spl + (t % NP) * (PW * PK);
            const R rcdy = R(ld(g.RCDY + r - 1));
            for (int p = tid; p < PW * PK; p += 32 * FW) {
                const int ii = i0 - 1 + p / PK, kk = L0 - 1 + p % PK;
                if (ii > g.IE + 1 || kk < KS || kk > KE) continue;
                const size_t c = idx3(g, kk, ii, r);
                const R q = R(PI(r, kk, ii));
                const R lz = kk <= KE - 1 ? lflux_v(ld(mZ + c), q, R(PI(r, kk + 1, ii))) : zero;
                const R lzm = kk >= KS + 1 ? lflux_v(ld(mZ + c - 1), R(PI(r, kk - 1, ii)), q) : zero;
                const R lx = lflux_v(ld(mX + c), q, R(PI(r, kk, ii + 1)));
                const R lxm = lflux_v(ld(mX + c - sI), R(PI(r, kk, ii - 1)), q);
                const R ly = lflux_v(ld(mY + c), q, R(PI(r + 1, kk, ii)));
                const R lym = lflux_v(ld(mY + c - sJ), R(PI(r - 1, kk, ii)), q);
                pl[p] = R((PI(r, kk, ii) * ld(a.DENS0 + c)
                           + a.dtl * (double)mfac(g, a, -((lz - lzm) * R(ld(g.RCDZ + kk - 1)) + (lx - lxm) * R(ld(g.RCDX + ii - 1))
                                                          + (ly - lym) * rcdy),
                                                  ii, r, c))
                          / ld(a.DENS + c));
            }
        }
        if (tid == 0 && t + 3 <= rlast) {
            const bool ok = wait_row(t + 3);
            if (!ok) (void)wait_row(t + 3); // bounded: the copy still in flight
            s_ok[t & 1] = ok ? 1 : 0;
        } else if (tid == 0) {
            s_ok[t & 1] = 1;
        }
        __syncthreads(); // phi_lo of row r in place; every read of iteration t-1 done
        if (!s_ok[t & 1]) {
            if (tid == 0) atomicOr(a.status, ST_TMA_TIMEOUT);
            return; // block-uniform
        }
        if (t + 3 <= rlast) (void)mbar_try(bar + (t + 3) % NS, (unsigned)((t + 3) / NS) & 1u);
        if (tid == 0 && t + 4 <= rlast) {
            fence_proxy_async();
            issue(t + 4);
        }
        // (b) anti-diffusive fluxes of the faces of row o's cells (common.F90:2050-2073)
        const int o = r - 1;
        const bool out = t >= 2; // block-uniform
        const size_t c = idx3(g, min(k, KE), min(i, g.IE), o);
        const size_t col = c - (size_t)(min(k, KE) - 1);
        R az = zero, azm = zero, ax = zero, ay = zero, aym = zero, axm = zero;
        if (out) {
            if (cell && k <= KE - 1)
                az = hflux_z<S>(g, a, N3, col, k) - lflux_v(ld(mZ + c), R(PI(o, k, i)), R(PI(o, k + 1, i)));
            azm = __shfl_up_sync(0xffffffffu, az, 1);
            if (lane == 0)
                azm = (cell && L0 > KS)
                          ? hflux_z<S>(g, a, N3, col, L0 - 1) - lflux_v(ld(mZ + c - 1), R(PI(o, L0 - 1, i)), R(PI(o, L0, i)))
                          : zero;
            if (cell) {
                // R(QTRC0) for k_fct_update: this cell and the halo ring its faces reach
                a.phi_lo[c] = R(PI(o, k, i));
                if (i == g.IS) a.phi_lo[c - sI] = R(PI(o, k, i - 1));
                if (i == g.IE) a.phi_lo[c + sI] = R(PI(o, k, i + 1));
                if (o == g.JS) a.phi_lo[c - sJ] = R(PI(o - 1, k, i));
                if (o == g.JE) a.phi_lo[c + sJ] = R(PI(o + 1, k, i));
                ax = hflux_h<S>(a, N3, 1, c, sI) - lflux_v(ld(mX + c), R(PI(o, k, i)), R(PI(o, k, i + 1)));
                axm = hflux_h<S>(a, N3, 1, c - sI, sI) - lflux_v(ld(mX + c - sI), R(PI(o, k, i - 1)), R(PI(o, k, i)));
                ay = hflux_h<S>(a, N3, 2, c, sJ) - lflux_v(ld(mY + c), R(PI(o, k, i)), R(PI(o + 1, k, i)));
                aym = t == 2 ? hflux_h<S>(a, N3, 2, c - sJ, sJ) - lflux_v(ld(mY + c - sJ), R(PI(o - 1, k, i)), R(PI(o, k, i)))
                             : ay_prev;
                ay_prev = ay;
            }
        }
        if (!out || !cell) continue;

        // (c) P+/P-, the bounds Q+/Q- and R+/R- of cell (k, i, o) (common.F90:2077-2553)
        const R pz = rmax(zero, azm) - rmin(zero, az);
        const R px = rmax(zero, axm) - rmin(zero, ax);
        const R py = rmax(zero, aym) - rmin(zero, ay);
        const R rdy = R(ld(g.RCDY + o - 1));
        const R pjpls = mfac(g, a, dtl * (pz * rdz + px * rdx + py * rdy), i, o, c);
        const R mz = rmax(zero, az) - rmin(zero, azm);
        const R mx = rmax(zero, ax) - rmin(zero, axm);
        const R my = rmax(zero, ay) - rmin(zero, aym);
        const R pjmns = mfac(g, a, dtl * (mz * rdz + mx * rdx + my * rdy), i, o, c);
        const auto vin = [&](int dk, int di, int dj) { return R(PI(o + dj, k + dk, i + di)); };
        const auto vlo = [&](int dk, int di, int dj) { return PL(o + dj, k + dk, i + di); };
        const R pin = vin(0, 0, 0), plo = vlo(0, 0, 0);
        R qmax, qmin;
        if (a.along_stream) {
            R rw;
            int ka, kb;
            if (k == KS) { rw = ld(mZ + c) * rdz; ka = 1; kb = 0; }
            else if (k == KE) { rw = ld(mZ + c - 1) * rdz; ka = 0; kb = -1; }
            else { rw = (ld(mZ + c) + ld(mZ + c - 1)) * rdz; ka = 1; kb = -1; }
            const R ru = (ld(mX + c) + ld(mX + c - sI)) * rdx;
            const R rv = (ld(mY + c) + ld(mY + c - sJ)) * rdy;
            R f[2][3][3];
            fact_fct(f, rw, ru, rv);
            const R qa_in = qa_sum(f, ka, vin), qb_in = qb_sum(f, kb, vin);
            const R qa_lo = qa_sum(f, ka, vlo), qb_lo = qb_sum(f, kb, vlo);
            qmax = rmax(rmax(rmax(rmax(rmax(pin, qa_in), qb_in), plo), qa_lo), qb_lo);
            qmin = rmin(rmin(rmin(rmin(rmin(pin, qa_in), qb_in), plo), qa_lo), qb_lo);
        } else {
            qmax = rmax(pin, plo);
            qmin = rmin(pin, plo);
            const int nb[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
#pragma unroll
            for (int n = 0; n < 6; ++n) {
                if ((k == KS && nb[n][0] == -1) || (k == KE && nb[n][0] == 1)) continue;
                const R x = vin(nb[n][0], nb[n][1], nb[n][2]), y = vlo(nb[n][0], nb[n][1], nb[n][2]);
                qmax = rmax(rmax(qmax, x), y);
                qmin = rmin(rmin(qmin, x), y);
            }
        }
        const R dn = R(ld(a.DENS + c));
        const R qjpls = (qmax - plo) * dn;
        const R qjmns = (plo - qmin) * dn;
        R zerosw = h - fsign(h, pjpls - eps);
        a.rjp[c] = rmin(one, qjpls * (one - zerosw) / (pjpls - zerosw));
        zerosw = h - fsign(h, pjmns - eps);
        a.rjm[c] = rmin(one, qjmns * (one - zerosw) / (pjmns - zerosw));
    }
}

// limit and update (tstep_tracer_fvm_heve.F90:188-210) with the anti-diffusive
// fluxes formed again from the high- and low-order fluxes; the z fluxes of
// the face below a level come from the previous lane (lane 0: the previous
// pass's lane 31; zero below KS). The low-order fluxes read R(QTRC0) from the
// copy k_fct_limit left in the phi_lo scratch, not QTRC0 itself: QTRCo may be
// QTRC0 (the RK3 integrator updates the tracer in place), and a neighbour's
// value there may already be the new one. Each cell's own QTRC0 is read
// before its own write.
template <int S, typename R>
__global__ void HEVI_UPD_BOUNDS k_fct_update(const Grid g, const TracerArgsT<R> a)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const size_t col = idx3(g, 1, i, j);
    const R rcdx = R(ld(g.RCDX + i - 1)), rcdy = R(ld(g.RCDY + j - 1));
    const R *q0 = a.phi_lo; // R(QTRC0)
    // donor-cell flux at the face between c and c+s
    auto lf = [&](int dir, size_t c, long s) {
        return lflux_v(ld(a.mflx + (size_t)dir * N3 + c), ld(q0 + c), ld(q0 + c + s));
    };
    R carry_h = R(0.0), carry_a = R(0.0);
    for (int k0 = g.KS; k0 <= g.KE; k0 += 32) {
        const int k = k0 + threadIdx.x;
        const bool ok = k <= g.KE;
        const size_t c = col + k - 1;
        R hz = R(0.0), az = R(0.0);
        if (ok) {
            hz = hflux_z<S>(g, a, N3, col, k);
            if (k <= g.KE - 1) az = limit(a, hz - lf(0, c, 1), c, 1);
        }
        R hzm = __shfl_up_sync(0xffffffffu, hz, 1), azm = __shfl_up_sync(0xffffffffu, az, 1);
        if (threadIdx.x == 0) {
            hzm = carry_h;
            azm = carry_a;
        }
        carry_h = __shfl_sync(0xffffffffu, hz, 31);
        carry_a = __shfl_sync(0xffffffffu, az, 31);
        if (!ok) continue;
        const R hx = hflux_h<S>(a, N3, 1, c, sI), hxm = hflux_h<S>(a, N3, 1, c - sI, sI);
        const R hy = hflux_h<S>(a, N3, 2, c, sJ), hym = hflux_h<S>(a, N3, 2, c - sJ, sJ);
        const R ax = limit(a, hx - lf(1, c, sI), c, sI);
        const R axm = limit(a, hxm - lf(1, c - sI, sI), c - sI, sI);
        const R ay = limit(a, hy - lf(2, c, sJ), c, sJ);
        const R aym = limit(a, hym - lf(2, c - sJ, sJ), c - sJ, sJ);
        const R div = (hz - az - hzm + azm) * R(ld(g.RCDZ + k - 1)) + (hx - ax - hxm + axm) * rcdx
                      + (hy - ay - hym + aym) * rcdy;
        a.QTRCo[c] = (ld(a.QTRC0 + c) * ld(a.DENS0 + c) + a.dtl * (double)(mfac(g, a, -div, i, j, c) + ld(a.RHOQ_t + c)))
                     / ld(a.DENS + c);
    }
}

// the halo of R+/R- between the limiter's kernels: the exchange hook of a
// decomposed domain, else the periodic fill (one launch)
template <typename R>
static cudaError_t fill_r(const Grid &g, const TracerArgsT<R> &a, cudaStream_t st, const HaloFill *fill, int &nk)
{
    R *rr[2] = {a.rjp, a.rjm};
    if (fill) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (fill->fn(fill->ctx, reinterpret_cast<void *const *>(rr), 2, (int)sizeof(R))) return cudaErrorUnknown;
    } else {
        periodic_halo(g, Members{}, rr, 2, st);
        ++nk;
    }
    return cudaSuccess;
}

// the fused form of a limited stage; cudaErrorNotSupported (nothing launched)
// without a status word or where QTRC0 admits no tensor map (even KA, a
// 16-byte aligned base)
template <int S, typename R>
static cudaError_t fct_fused(const Grid &g, const TracerArgsT<R> &a, cudaStream_t st, const HaloFill *fill, int &nk)
{
    CUtensorMap map;
    if (!a.status || !tma::encode(&map, a.QTRC0, g, fct::BK, fct::BW, 1)) return cudaErrorNotSupported;
    const dim3 gf((unsigned)(((g.IMAX + fct::FW - 1) / fct::FW) * ((g.KMAX + fct::KC - 1) / fct::KC)),
                  (unsigned)((g.JMAX + fct::JB - 1) / fct::JB));
    auto kl = k_fct_limit<S, R>;
    cudaError_t e = tma::open_smem(kl, fct::smem_bytes<R>());
    if (e != cudaSuccess) return e;
    kl<<<gf, dim3(32, fct::FW), fct::smem_bytes<R>(), st>>>(g, a, map);
    ++nk;
    e = fill_r(g, a, st, fill, nk);
    if (e != cudaSuccess) return e;
    k_fct_update<S, R><<<dim3((g.IMAX + 3) / 4, g.JMAX), dim3(32, 4), 0, st>>>(g, a);
    ++nk;
    return cudaGetLastError();
}

template <int S, typename R>
static cudaError_t tracer_stage(const Grid &g, const TracerArgsT<R> &a, bool fct, cudaStream_t st, const HaloFill *fill,
                                int &nk)
{
    dim3 b(32, 4), gr((g.IMAX + 3) / 4, g.JMAX);
    if (!fct) {
        k_tracer_plain<S, R><<<gr, b, 0, st>>>(g, a);
        ++nk;
        return cudaGetLastError();
    }
    const cudaError_t ef = fct_fused<S, R>(g, a, st, fill, nk);
    if (ef != cudaErrorNotSupported) return ef;
    dim3 gl((g.IMAX + 2 + 3) / 4, g.JMAX + 2);
    k_fct_lo<S, R><<<gl, b, 0, st>>>(g, a);
    k_fct_r<R><<<gr, b, 0, st>>>(g, a);
    nk += 2;
    cudaError_t e = fill_r(g, a, st, fill, nk);
    if (e != cudaSuccess) return e;
    k_fct_apply<S, R><<<gr, b, 0, st>>>(g, a);
    ++nk;
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_tracer_stage(const Grid &g, const TracerArgsT<R> &a, int scheme, bool fct, cudaStream_t st,
                                const HaloFill *fill, int *nk)
{
    int n = 0;
    cudaError_t e;
    switch (scheme) {
    case UD3: e = tracer_stage<UD3, R>(g, a, fct, st, fill, n); break;
    case CD4: e = tracer_stage<CD4, R>(g, a, fct, st, fill, n); break;
    case KOREN: e = tracer_stage<KOREN, R>(g, a, fct, st, fill, n); break;
    case CD2: e = tracer_stage<CD2, R>(g, a, fct, st, fill, n); break;
    case UD5: e = tracer_stage<UD5, R>(g, a, fct, st, fill, n); break;
    case CD6: e = tracer_stage<CD6, R>(g, a, fct, st, fill, n); break;
    default: e = cudaErrorInvalidValue;
    }
    if (nk) *nk = n;
    return e;
}
#ifdef HEVI_FLOAT_TU
template cudaError_t launch_tracer_stage<float>(const Grid &, const TracerArgsT<float> &, int, bool, cudaStream_t,
                                                const HaloFill *, int *);
#else
template cudaError_t launch_tracer_stage<double>(const Grid &, const TracerArgsT<double> &, int, bool, cudaStream_t,
                                                 const HaloFill *, int *);
#endif

}  // namespace hevi
