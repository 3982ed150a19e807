// Tracer advection with flux-corrected transport on the device:
//   ATMOS_DYN_Tstep_tracer_fvm_heve  scale_atmos_dyn_tstep_tracer_fvm_heve.F90:72-240
//   ATMOS_DYN_fct / get_fact_fct     scale_atmos_dyn_common.F90:1922-2734
//   UD1 low-order fluxes             scale_atmos_dyn_fvm_flux_ud1.F90:135-294
//
// A stage without FCT is one kernel (every cell forms its six face fluxes and
// updates). With FCT the limiter needs the low-order solution and the
// limiting factors of the neighbours, so it runs as three kernels around the
// halo fill of R+/R- (the reference's mid-limiter COMM_vars8, :2558-2561):
//   k_fct_lo    low-order update phi_lo on the halo-extended region and the
//               raw anti-diffusive fluxes of every face an interior cell owns
//   k_fct_r     P+/P-, the along-stream (or 7-point) bounds Q+/Q-, R+/R-
//   k_fct_apply limit the anti-diffusive fluxes and update the tracer
// Terrain-following metrics (TracerArgsT::GS, MAPF) enter the num_diff terms and
// the metric factor of every flux divergence; null pointers mean flat terrain.
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
// donor-cell flux at the face between c and c+s (ud1.F90:155-165)
template <typename R>
__device__ __forceinline__ R lflux(const TracerArgsT<R> &a, size_t N3, int dir, size_t c, long s)
{
    const R vel = ld(a.mflx + (size_t)dir * N3 + c);
    const R lo = R(ld(a.QTRC0 + c)), hi = R(ld(a.QTRC0 + c + s));
    return vel * (R(0.5) * (hi + lo) - fsign(R(0.5), vel) * (hi - lo));
}

// ---- stage without FCT, tstep_tracer_fvm_heve.F90:214-236 -------------------
template <int S, typename R>
__global__ void __launch_bounds__(128) k_tracer_plain(const Grid g, const TracerArgsT<R> a)
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

template <int S, typename R>
static cudaError_t tracer_stage(const Grid &g, const TracerArgsT<R> &a, bool fct, cudaStream_t st, const HaloFill *fill)
{
    dim3 b(32, 4), gr((g.IMAX + 3) / 4, g.JMAX);
    if (!fct) {
        k_tracer_plain<S, R><<<gr, b, 0, st>>>(g, a);
        return cudaGetLastError();
    }
    dim3 gl((g.IMAX + 2 + 3) / 4, g.JMAX + 2);
    k_fct_lo<S, R><<<gl, b, 0, st>>>(g, a);
    k_fct_r<R><<<gr, b, 0, st>>>(g, a);
    R *rr[2] = {a.rjp, a.rjm};
    if (fill) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (fill->fn(fill->ctx, reinterpret_cast<void *const *>(rr), 2, (int)sizeof(R))) return cudaErrorUnknown;
    } else {
        periodic_halo(g, Members{}, rr, 2, st);
    }
    k_fct_apply<S, R><<<gr, b, 0, st>>>(g, a);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_tracer_stage(const Grid &g, const TracerArgsT<R> &a, int scheme, bool fct, cudaStream_t st,
                                const HaloFill *fill)
{
    switch (scheme) {
    case UD3: return tracer_stage<UD3, R>(g, a, fct, st, fill);
    case CD4: return tracer_stage<CD4, R>(g, a, fct, st, fill);
    case KOREN: return tracer_stage<KOREN, R>(g, a, fct, st, fill);
    case CD2: return tracer_stage<CD2, R>(g, a, fct, st, fill);
    case UD5: return tracer_stage<UD5, R>(g, a, fct, st, fill);
    case CD6: return tracer_stage<CD6, R>(g, a, fct, st, fill);
    default: return cudaErrorInvalidValue;
    }
}
#ifdef HEVI_FLOAT_TU
template cudaError_t launch_tracer_stage<float>(const Grid &, const TracerArgsT<float> &, int, bool, cudaStream_t,
                                                const HaloFill *);
#else
template cudaError_t launch_tracer_stage<double>(const Grid &, const TracerArgsT<double> &, int, bool, cudaStream_t,
                                                 const HaloFill *);
#endif

}  // namespace hevi
