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
// Terrain-following metrics (TracerArgs::GS, MAPF) enter the num_diff terms and
// the metric factor of every flux divergence; null pointers mean flat terrain.
#include "hevi_kernels.cuh"

namespace hevi {

// stage density, tinteg_tracer_rk3.F90:140-147 / :168-175
__device__ __forceinline__ double dens_of(const TracerArgs &a, size_t c)
{
    const double d = ld(a.DENS + c);
    if (a.dens_mode == 0) return d;
    const double d0 = ld(a.DENS0 + c);
    return a.dens_mode == 1 ? d0 + (d - d0) / 3.0 : d0 + (d - d0) * 0.5;
}

// the num_diff term of a high-order flux; with terrain GSQRT times it, at the
// staggering of the face (fluxZ/X/Y_XYZ: I_XYW, I_UYZ, I_XVZ)
__device__ __forceinline__ double ndq_at(const TracerArgs &a, size_t N3, int dir, size_t c)
{
    const double nd = a.ndq ? ld(a.ndq + (size_t)dir * N3 + c) : 0.0;
    if (!a.GS) return nd;
    const int slice = dir == 0 ? 1 : dir == 1 ? 4 : 5; // I_XYW, I_UYZ, I_XVZ (0-based)
    return ld(a.GS + (size_t)slice * N3 + c) * nd;
}
// x * MAPF(i,j,1) * MAPF(i,j,2) / GSQRT(k,i,j,I_XYZ) with terrain, x on flat terrain
// (the metric factor of every flux divergence, tstep_tracer_fvm_heve.F90:188-236,
// common.F90:2051-2120)
__device__ __forceinline__ double mfac(const Grid &g, const TracerArgs &a, double x, int i, int j, size_t c)
{
    if (!a.GS) return x;
    const size_t p = (size_t)(i - 1) + (size_t)g.IA * (size_t)(j - 1);
    return x * ld(a.MAPF + p) * ld(a.MAPF + p + (size_t)g.IA * g.JA) / ld(a.GS + c);
}

// high-order z flux at the face above level m (fluxZ_XYZ, ud3.F90:157-247, ud5.F90:194-321)
template <int S>
__device__ double hflux_z(const Grid &g, const TracerArgs &a, size_t N3, size_t col, int m)
{
    if (m < g.KS || m > g.KE - 1) return 0.0;
    const double *q = a.QTRC + col - 1;
    const double vel = ld(a.mflx + col + m - 1);
    const double v = zface<S>(vel, m, g.KS, g.KE, [&](int l) { return ld(q + l); });
    return vel * v + ndq_at(a, N3, 0, col + m - 1);
}
// high-order flux at the face between c and c+s (fluxX/Y_XYZ, ud3.F90:251-353); dir 1 = x, 2 = y
template <int S>
__device__ __forceinline__ double hflux_h(const TracerArgs &a, size_t N3, int dir, size_t c, long s)
{
    const double vel = ld(a.mflx + (size_t)dir * N3 + c);
    const double *q = a.QTRC + c;
    constexpr bool W6 = wide_scheme(S);
    return vel * ip6<S>(vel, W6 ? ld(q - 2 * s) : 0.0, ld(q - s), ld(q), ld(q + s), ld(q + 2 * s), W6 ? ld(q + 3 * s) : 0.0)
           + ndq_at(a, N3, dir, c);
}
// donor-cell flux at the face between c and c+s (ud1.F90:155-165)
__device__ __forceinline__ double lflux(const TracerArgs &a, size_t N3, int dir, size_t c, long s)
{
    const double vel = ld(a.mflx + (size_t)dir * N3 + c);
    const double lo = ld(a.QTRC0 + c), hi = ld(a.QTRC0 + c + s);
    return vel * (0.5 * (hi + lo) - fsign(0.5, vel) * (hi - lo));
}

// ---- stage without FCT, tstep_tracer_fvm_heve.F90:214-236 -------------------
template <int S>
__global__ void __launch_bounds__(128) k_tracer_plain(const Grid g, const TracerArgs a)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const size_t col = idx3(g, 1, i, j);
    const double rcdx = ld(g.RCDX + i - 1), rcdy = ld(g.RCDY + j - 1);
    // the z flux through the face above a level; the face below is the previous
    // lane's (lane 0: the previous pass's lane 31; zero below KS)
    double carry = 0.0;
    for (int k0 = g.KS; k0 <= g.KE; k0 += 32) {
        const int k = k0 + threadIdx.x;
        const bool ok = k <= g.KE;
        const size_t c = col + k - 1;
        const double hz = ok ? hflux_z<S>(g, a, N3, col, k) : 0.0;
        double hzm = __shfl_up_sync(0xffffffffu, hz, 1);
        if (threadIdx.x == 0) hzm = carry;
        carry = __shfl_sync(0xffffffffu, hz, 31);
        if (!ok) continue;
        const double hx = hflux_h<S>(a, N3, 1, c, sI), hxm = hflux_h<S>(a, N3, 1, c - sI, sI);
        const double hy = hflux_h<S>(a, N3, 2, c, sJ), hym = hflux_h<S>(a, N3, 2, c - sJ, sJ);
        const double div = (hz - hzm) * ld(g.RCDZ + k - 1) + (hx - hxm) * rcdx + (hy - hym) * rcdy;
        a.QTRCo[c] = (ld(a.QTRC0 + c) * ld(a.DENS0 + c) + a.dtl * (mfac(g, a, -div, i, j, c) + ld(a.RHOQ_t + c))) / dens_of(a, c);
    }
}

// ---- FCT part 1: low-order solution and raw anti-diffusive fluxes (common.F90:1990-2073) ----
template <int S>
__global__ void __launch_bounds__(128) k_fct_lo(const Grid g, const TracerArgs a)
{
    // columns i in IS-1..IE+1, j in JS-1..JE+1
    const int i = g.IS - 1 + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS - 1 + blockIdx.y;
    if (i > g.IE + 1) return;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const size_t col = idx3(g, 1, i, j);
    const bool inter = (i >= g.IS && i <= g.IE && j >= g.JS && j <= g.JE);
    const double rcdx = ld(g.RCDX + i - 1), rcdy = ld(g.RCDY + j - 1);
    for (int k = g.KS + threadIdx.x; k <= g.KE; k += 32) {
        const size_t c = col + k - 1;
        const double lz = (k <= g.KE - 1) ? lflux(a, N3, 0, c, 1) : 0.0;
        const double lzm = (k >= g.KS + 1) ? lflux(a, N3, 0, c - 1, 1) : 0.0;
        const double lx = lflux(a, N3, 1, c, sI), lxm = lflux(a, N3, 1, c - sI, sI);
        const double ly = lflux(a, N3, 2, c, sJ), lym = lflux(a, N3, 2, c - sJ, sJ);
        a.phi_lo[c] = (ld(a.QTRC0 + c) * ld(a.DENS0 + c)
                       + a.dtl * mfac(g, a, -((lz - lzm) * ld(g.RCDZ + k - 1) + (lx - lxm) * rcdx + (ly - lym) * rcdy), i, j, c))
                      / ld(a.DENS + c);
        if (inter) {
            double *aZ = a.anti, *aX = a.anti + N3, *aY = a.anti + 2 * N3;
            aZ[c] = (k <= g.KE - 1) ? hflux_z<S>(g, a, N3, col, k) - lz : 0.0;
            if (k == g.KS) aZ[c - 1] = 0.0;
            aX[c] = hflux_h<S>(a, N3, 1, c, sI) - lx;
            aY[c] = hflux_h<S>(a, N3, 2, c, sJ) - ly;
            if (i == g.IS) aX[c - sI] = hflux_h<S>(a, N3, 1, c - sI, sI) - lxm;
            if (j == g.JS) aY[c - sJ] = hflux_h<S>(a, N3, 2, c - sJ, sJ) - lym;
        }
    }
}

// get_fact_fct, common.F90:2676-2734; f[a][b+1][c+1] = fact(a,b,c)
__device__ __forceinline__ void fact_fct(double f[2][3][3], double rw, double ru, double rv)
{
    const double ugev = fsign(0.5, fabs(ru) - fabs(rv)) + 0.5;
    const double ugew = fsign(0.5, fabs(ru) - fabs(rw)) + 0.5;
    const double vgew = fsign(0.5, fabs(rv) - fabs(rw)) + 0.5;
    const double uzero = fsign(0.5, fabs(ru) - EPS) - 0.5;
    const double vzero = fsign(0.5, fabs(rv) - EPS) - 0.5;
    const double wzero = fsign(0.5, fabs(rw) - EPS) - 0.5;
    const double sign_uv = fsign(0.5, ru * rv) + 0.5;
    const double sign_uw = fsign(0.5, ru * rw) + 0.5;
    const double sign_vw = fsign(0.5, rv * rw) + 0.5;
    const double wu = fabs(rw / (ru + uzero) * (1.0 + uzero));
    const double vu = fabs(rv / (ru + uzero) * (1.0 + uzero));
    const double uv = fabs(ru / (rv + vzero) * (1.0 + vzero));
    const double wv = fabs(rw / (rv + vzero) * (1.0 + vzero));
    const double uw = fabs(ru / (rw + wzero) * (1.0 + wzero));
    const double vw = fabs(rv / (rw + wzero) * (1.0 + wzero));
    const double umax = ugev * ugew * (1.0 + uzero);
    const double vmax = (1.0 - ugev) * vgew;
    const double wmax = 1.0 - ugev * ugew - vmax;
    const double tri = umax * vu * wu + vmax * uv * wv + wmax * uw * vw;
    const double xz = ugew * wu * (1.0 - vu) + (1.0 - ugew) * uw * (1.0 - vw);
    const double yz = vgew * wv * (1.0 - uv) + (1.0 - vgew) * vw * (1.0 - uw);
    const double xy = ugev * vu * (1.0 - wu) + (1.0 - ugev) * uv * (1.0 - wv);
#define FF(x, y, z) f[x][(y) + 1][(z) + 1]
    FF(0, 0, 0) = -ugev * ugew * uzero;
    FF(1, 0, 0) = wmax * (1.0 - uw) * (1.0 - vw);
    FF(0, 1, 0) = umax * (1.0 - vu) * (1.0 - wu);
    FF(0, 0, 1) = vmax * (1.0 - uv) * (1.0 - wv);
    FF(1, 1, 1) = sign_uv * sign_uw * tri;
    FF(1, -1, 1) = (1.0 - sign_uv) * (1.0 - sign_uw) * tri;
    FF(1, 1, -1) = (1.0 - sign_uv) * sign_uw * tri;
    FF(1, -1, -1) = sign_uv * (1.0 - sign_uw) * tri;
    FF(1, 1, 0) = sign_uw * (1.0 - vmax) * xz;
    FF(1, -1, 0) = (1.0 - sign_uw) * (1.0 - vmax) * xz;
    FF(1, 0, 1) = sign_vw * (1.0 - umax) * yz;
    FF(1, 0, -1) = (1.0 - sign_vw) * (1.0 - umax) * yz;
    FF(0, 1, 1) = sign_uv * (1.0 - wmax) * xy;
    FF(0, 1, -1) = (1.0 - sign_uv) * (1.0 - wmax) * xy;
#undef FF
}

// ---- FCT part 2: limiting factors R+ and R- (common.F90:2079-2553) ----------
__global__ void __launch_bounds__(128) k_fct_r(const Grid g, const TracerArgs a)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const size_t col = idx3(g, 1, i, j);
    const double *aZ = a.anti, *aX = a.anti + N3, *aY = a.anti + 2 * N3;
    const double *mZ = a.mflx, *mX = a.mflx + N3, *mY = a.mflx + 2 * N3;
    const double rdx = ld(g.RCDX + i - 1), rdy = ld(g.RCDY + j - 1);
    const int KS = g.KS, KE = g.KE;
    for (int k = KS + threadIdx.x; k <= KE; k += 32) {
        const size_t c = col + k - 1;
        const double rdz = ld(g.RCDZ + k - 1);
        // net incoming / outgoing anti-diffusive change :2077-2120
        const double pz = fmax2(0.0, ld(aZ + c - 1)) - fmin2(0.0, ld(aZ + c));
        const double px = fmax2(0.0, ld(aX + c - sI)) - fmin2(0.0, ld(aX + c));
        const double py = fmax2(0.0, ld(aY + c - sJ)) - fmin2(0.0, ld(aY + c));
        const double pjpls = mfac(g, a, a.dtl * (pz * rdz + px * rdx + py * rdy), i, j, c);
        const double mz = fmax2(0.0, ld(aZ + c)) - fmin2(0.0, ld(aZ + c - 1));
        const double mx = fmax2(0.0, ld(aX + c)) - fmin2(0.0, ld(aX + c - sI));
        const double my = fmax2(0.0, ld(aY + c)) - fmin2(0.0, ld(aY + c - sJ));
        const double pjmns = mfac(g, a, a.dtl * (mz * rdz + mx * rdx + my * rdy), i, j, c);

        const double *PI = a.QTRC0 + c, *PL = a.phi_lo + c;
        double qmax, qmin;
        if (a.along_stream) {
            // along-stream bound :2126-2369; ka / kb are the levels of the upstream
            // and downstream (1,*,*) points (clamped at KS and KE as the reference does)
            double rw;
            long ka, kb;
            if (k == KS) { rw = ld(mZ + c) * rdz; ka = 1; kb = 0; }
            else if (k == KE) { rw = ld(mZ + c - 1) * rdz; ka = 0; kb = -1; }
            else { rw = (ld(mZ + c) + ld(mZ + c - 1)) * rdz; ka = 1; kb = -1; }
            const double ru = (ld(mX + c) + ld(mX + c - sI)) * rdx;
            const double rv = (ld(mY + c) + ld(mY + c - sJ)) * rdy;
            double f[2][3][3];
            fact_fct(f, rw, ru, rv);
#define FA(x, y, z) f[x][(y) + 1][(z) + 1]
#define QA(P) (FA(1, 1, 1) * ld(P + ka + sI + sJ) + FA(0, 1, 1) * ld(P + sI + sJ) + FA(1, 0, 1) * ld(P + ka + sJ)    \
               + FA(0, 0, 1) * ld(P + sJ) + FA(1, -1, 1) * ld(P + ka - sI + sJ) + FA(1, 1, 0) * ld(P + ka + sI)      \
               + FA(0, 1, 0) * ld(P + sI) + FA(1, 0, 0) * ld(P + ka) + FA(1, -1, 0) * ld(P + ka - sI)                 \
               + FA(1, 1, -1) * ld(P + ka + sI - sJ) + FA(0, 1, -1) * ld(P + sI - sJ) + FA(1, 0, -1) * ld(P + ka - sJ) \
               + FA(1, -1, -1) * ld(P + ka - sI - sJ) + FA(0, 0, 0) * ld(P))
#define QB(P) (FA(1, 1, 1) * ld(P + kb - sI - sJ) + FA(0, 1, 1) * ld(P - sI - sJ) + FA(1, 0, 1) * ld(P + kb - sJ)    \
               + FA(0, 0, 1) * ld(P - sJ) + FA(1, -1, 1) * ld(P + kb + sI - sJ) + FA(1, 1, 0) * ld(P + kb - sI)      \
               + FA(0, 1, 0) * ld(P - sI) + FA(1, 0, 0) * ld(P + kb) + FA(1, -1, 0) * ld(P + kb + sI)                 \
               + FA(1, 1, -1) * ld(P + kb - sI + sJ) + FA(0, 1, -1) * ld(P - sI - sJ) + FA(1, 0, -1) * ld(P + kb - sJ) \
               + FA(1, -1, -1) * ld(P + kb + sI + sJ) + FA(0, 0, 0) * ld(P))
            const double qa_in = QA(PI), qb_in = QB(PI), qa_lo = QA(PL), qb_lo = QB(PL);
#undef QA
#undef QB
#undef FA
            const double pin = ld(PI), plo = ld(PL);
            qmax = fmax2(fmax2(fmax2(fmax2(fmax2(pin, qa_in), qb_in), plo), qa_lo), qb_lo);
            qmin = fmin2(fmin2(fmin2(fmin2(fmin2(pin, qa_in), qb_in), plo), qa_lo), qb_lo);
        } else {
            // 7-point bound :2370-2515
            const double pin = ld(PI), plo = ld(PL);
            qmax = fmax2(pin, plo);
            qmin = fmin2(pin, plo);
            const long nb[6] = {1, -1, sI, -sI, sJ, -sJ};
            for (int n = 0; n < 6; ++n) {
                if ((k == KS && nb[n] == -1) || (k == KE && nb[n] == 1)) continue;
                const double x = ld(PI + nb[n]), y = ld(PL + nb[n]);
                qmax = fmax2(fmax2(qmax, x), y);
                qmin = fmin2(fmin2(qmin, x), y);
            }
        }
        const double dn = ld(a.DENS + c), plo = ld(PL);
        const double qjpls = (qmax - plo) * dn;
        const double qjmns = (plo - qmin) * dn;
        double zerosw = 0.5 - fsign(0.5, pjpls - EPS);
        a.rjp[c] = fmin2(1.0, qjpls * (1.0 - zerosw) / (pjpls - zerosw));
        zerosw = 0.5 - fsign(0.5, pjmns - EPS);
        a.rjm[c] = fmin2(1.0, qjmns * (1.0 - zerosw) / (pjmns - zerosw));
    }
}

// limited anti-diffusive flux at the face between c and c+s (common.F90:2563-2660)
__device__ __forceinline__ double limit(const TracerArgs &a, double anti, size_t c, long s)
{
    const double dirsw = 0.5 + fsign(0.5, anti);
    return anti * (1.0 - fmin2(ld(a.rjp + c + s), ld(a.rjm + c)) * (dirsw) - fmin2(ld(a.rjp + c), ld(a.rjm + c + s)) * (1.0 - dirsw));
}

// ---- FCT part 3: limit and update (tstep_tracer_fvm_heve.F90:188-210) ------
template <int S>
__global__ void __launch_bounds__(128) k_fct_apply(const Grid g, const TracerArgs a)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const size_t col = idx3(g, 1, i, j);
    const double *aZ = a.anti, *aX = a.anti + N3, *aY = a.anti + 2 * N3;
    const double rcdx = ld(g.RCDX + i - 1), rcdy = ld(g.RCDY + j - 1);
    for (int k = g.KS + threadIdx.x; k <= g.KE; k += 32) {
        const size_t c = col + k - 1;
        const double az = (k <= g.KE - 1) ? limit(a, ld(aZ + c), c, 1) : 0.0;
        const double azm = (k >= g.KS + 1) ? limit(a, ld(aZ + c - 1), c - 1, 1) : 0.0;
        const double ax = limit(a, ld(aX + c), c, sI), axm = limit(a, ld(aX + c - sI), c - sI, sI);
        const double ay = limit(a, ld(aY + c), c, sJ), aym = limit(a, ld(aY + c - sJ), c - sJ, sJ);
        const double hz = hflux_z<S>(g, a, N3, col, k), hzm = hflux_z<S>(g, a, N3, col, k - 1);
        const double hx = hflux_h<S>(a, N3, 1, c, sI), hxm = hflux_h<S>(a, N3, 1, c - sI, sI);
        const double hy = hflux_h<S>(a, N3, 2, c, sJ), hym = hflux_h<S>(a, N3, 2, c - sJ, sJ);
        const double div = (hz - az - hzm + azm) * ld(g.RCDZ + k - 1) + (hx - ax - hxm + axm) * rcdx
                           + (hy - ay - hym + aym) * rcdy;
        a.QTRCo[c] = (ld(a.QTRC0 + c) * ld(a.DENS0 + c) + a.dtl * (mfac(g, a, -div, i, j, c) + ld(a.RHOQ_t + c))) / ld(a.DENS + c);
    }
}

template <int S>
static cudaError_t tracer_stage(const Grid &g, const TracerArgs &a, bool fct, cudaStream_t st)
{
    dim3 b(32, 4), gr((g.IMAX + 3) / 4, g.JMAX);
    if (!fct) {
        k_tracer_plain<S><<<gr, b, 0, st>>>(g, a);
        return cudaGetLastError();
    }
    dim3 gl((g.IMAX + 2 + 3) / 4, g.JMAX + 2);
    k_fct_lo<S><<<gl, b, 0, st>>>(g, a);
    k_fct_r<<<gr, b, 0, st>>>(g, a);
    double *rr[2] = {a.rjp, a.rjm};
    periodic_halo(g, Members{}, rr, 2, st);
    k_fct_apply<S><<<gr, b, 0, st>>>(g, a);
    return cudaGetLastError();
}

cudaError_t launch_tracer_stage(const Grid &g, const TracerArgs &a, int scheme, bool fct, cudaStream_t st)
{
    switch (scheme) {
    case UD3: return tracer_stage<UD3>(g, a, fct, st);
    case CD4: return tracer_stage<CD4>(g, a, fct, st);
    case KOREN: return tracer_stage<KOREN>(g, a, fct, st);
    case CD2: return tracer_stage<CD2>(g, a, fct, st);
    case UD5: return tracer_stage<UD5>(g, a, fct, st);
    case CD6: return tracer_stage<CD6>(g, a, fct, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace hevi
