// One HEVI short-step stage (ATMOS_DYN_Tstep_short_fvm_hevi,
// scalelib/src/atmos-rm/dynamics/scale_atmos_dyn_tstep_short_fvm_hevi.F90:128-1089)
// as two kernels:
//
//  k_hevi_horiz : one thread per cell (k fastest, coalesced), every flux that
//                 crosses an x or y face -- mass flux mflx_hi(X,Y), theta flux
//                 tflx_hi(X,Y), the horizontal part of the w-momentum flux
//                 divergence -- plus the complete u- and v-momentum updates
//                 (hevi_momx :814-928, hevi_momy :934-1048), which do not depend
//                 on the implicit solve.
//  k_hevi_column: one thread per column, the vertical fluxes, the sources Sr, Sw,
//                 St, the tridiagonal coefficients held in a register window, the
//                 Thomas solve (solve_direct :1092-1127) and the back-update of
//                 rho*w, rho, rho*theta and the vertical fluxes (:665-809).
//
// Flat terrain only (see hevi_common.cuh). Line numbers below refer to the
// reference HEVI file unless a flux file is named.
#include "hevi_kernels.cuh"

// Launch shapes. The defaults are the measured best on B200 for KMAX = 128;
// they can be overridden at build time for tuning sweeps.
#ifndef HEVI_HORIZ_COLS
#define HEVI_HORIZ_COLS 4 // i-columns per block of k_hevi_horiz (blockDim = 32 x HEVI_HORIZ_COLS)
#endif
#ifndef HEVI_HORIZ_MINB
#define HEVI_HORIZ_MINB 8 // minimum resident blocks per SM asked of the register allocator
#endif
#ifndef HEVI_COL_TC
#define HEVI_COL_TC 16 // columns per CTA of k_hevi_column
#endif
#ifndef HEVI_COL_MINB
#define HEVI_COL_MINB 2
#endif

namespace hevi {

// num_diff(:,:,:,v,dir) slice offset; v: DENS=1..RHOT=5, dir: Z=1,X=2,Y=3
__device__ __forceinline__ const double *nd_slice(const StageArgs &a, size_t N3, int v, int dir)
{
    return a.num_diff + N3 * (size_t)((v - 1) + 5 * (dir - 1));
}

__device__ __forceinline__ void flag_nonfinite(const StageArgs &a, double v)
{
    if (!isfinite(v)) atomicOr(a.status, ST_NONFINITE);
}

// store one prognostic value of the stage, folding in the RK4 combine
__device__ __forceinline__ void put_state(const StageArgs &a, size_t N3, int v, double *out, const double *x0,
                                          size_t c, double val, bool combine)
{
    double *acc = a.acc + (size_t)v * N3 + c;
    switch (a.rk_mode) {
    case RK_PLAIN: out[c] = val; flag_nonfinite(a, val); break;
    case RK_STAGE1: out[c] = val; if (combine) *acc = val * 2.0; break;
    case RK_STAGE2: out[c] = val; if (combine) *acc = *acc + val * 4.0; break;
    case RK_STAGE3: out[c] = val; if (combine) *acc = *acc + val * 2.0; break;
    default: {
        double r = combine ? ((*acc + val) - x0[c] * 3.0) / 6.0 : val;
        out[c] = r;
        flag_nonfinite(a, r);
    }
    }
}

// store one flux value (f: 0..2 mflx Z,X,Y; 3..5 tflx Z,X,Y); 'interior' marks the
// cells the RK4 combine averages (k in KS:KE, i in IS:IE, j in JS:JE)
__device__ __forceinline__ void put_flux(const StageArgs &a, size_t N3, int f, size_t c, double val, bool interior)
{
    double *out = (f < 3 ? a.mflx : a.tflx) + (size_t)(f % 3) * N3 + c;
    double *acc = a.facc + (size_t)f * N3 + c;
    switch (a.rk_mode) {
    case RK_PLAIN: *out = val; break;
    case RK_STAGE1: if (interior) *acc = val; break;
    case RK_STAGE2:
    case RK_STAGE3: if (interior) *acc = *acc + val * 2.0; break;
    default: *out = interior ? (*acc + val) / 6.0 : val;
    }
}

// =============================================================================
// 3-D kernel: horizontal fluxes and the u/v momentum updates
// =============================================================================
template <int S>
__global__ void __launch_bounds__(32 * HEVI_HORIZ_COLS, HEVI_HORIZ_MINB) k_hevi_horiz(const Grid g, const StageArgs a)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;

    const double *MX = a.MOMX, *MY = a.MOMY, *MZ = a.MOMZ, *DN = a.DENS, *RT = a.RHOT;
    const double *ndDX = nd_slice(a, N3, 1, 2), *ndDY = nd_slice(a, N3, 1, 3);
    const double *ndWX = nd_slice(a, N3, 2, 2), *ndWY = nd_slice(a, N3, 2, 3);
    const double *ndUZ = nd_slice(a, N3, 3, 1), *ndUX = nd_slice(a, N3, 3, 2), *ndUY = nd_slice(a, N3, 3, 3);
    const double *ndVZ = nd_slice(a, N3, 4, 1), *ndVX = nd_slice(a, N3, 4, 2), *ndVY = nd_slice(a, N3, 4, 3);
    const double *ndTX = nd_slice(a, N3, 5, 2), *ndTY = nd_slice(a, N3, 5, 3);

    const double rcdx = ld(g.RCDX + i - 1), rcdy = ld(g.RCDY + j - 1);
    const double rfdx = ld(g.RFDX + i - 1), rfdy = ld(g.RFDY + j - 1);
    const double fdx = ld(g.FDX + i - 1), fdy = ld(g.FDY + j - 1);
    const double dt = a.dtrk, J33G = a.J33G;
    const bool use_div = a.divdmp_coef != 0.0;
    const double ddc = use_div ? a.divdmp_coef / dt : 0.0;
    const int KS = g.KS, KE = g.KE;
    const bool do_u = i <= g.IEH, do_v = j <= g.JEH;
    const double cor_u = 0.125 * (ld(a.CORIOLI + (i) + (size_t)g.IA * (j - 1)) + ld(a.CORIOLI + (i - 1) + (size_t)g.IA * (j - 1)));
    const double cor_v = -0.125 * (ld(a.CORIOLI + (i - 1) + (size_t)g.IA * (j)) + ld(a.CORIOLI + (i - 1) + (size_t)g.IA * (j - 1)));

    for (int k = KS + threadIdx.x; k <= KE; k += 32) {
        const size_t c = idx3(g, k, i, j);
#define AT(p, dk, di, dj) ld((p) + c + (long)(dk) + (long)(di) * sI + (long)(dj) * sJ)

        // ---- mass fluxes at the u/v faces, hevi_mflx_x/y :399-438 ----
        const double mXe = AT(MX, 0, 0, 0) + AT(ndDX, 0, 0, 0);
        const double mXw = AT(MX, 0, -1, 0) + AT(ndDX, 0, -1, 0);
        const double mYn = AT(MY, 0, 0, 0) + AT(ndDY, 0, 0, 0);
        const double mYs = AT(MY, 0, 0, -1) + AT(ndDY, 0, 0, -1);
        // horizontal part of hevi_sr :464-467
        a.adv_r[c] = -((mXe - mXw) * rcdx + (mYn - mYs) * rcdy);

        // ---- theta fluxes, fluxX/Y_XYZ (ud3.F90:251-353) with POTT = RHOT/DENS :595 ----
        {
            const double Pm2 = AT(RT, 0, -2, 0) / AT(DN, 0, -2, 0);
            const double Pm1 = AT(RT, 0, -1, 0) / AT(DN, 0, -1, 0);
            const double P00 = AT(RT, 0, 0, 0) / AT(DN, 0, 0, 0);
            const double Pp1 = AT(RT, 0, 1, 0) / AT(DN, 0, 1, 0);
            const double Pp2 = AT(RT, 0, 2, 0) / AT(DN, 0, 2, 0);
            const double Qm2 = AT(RT, 0, 0, -2) / AT(DN, 0, 0, -2);
            const double Qm1 = AT(RT, 0, 0, -1) / AT(DN, 0, 0, -1);
            const double Qp1 = AT(RT, 0, 0, 1) / AT(DN, 0, 0, 1);
            const double Qp2 = AT(RT, 0, 0, 2) / AT(DN, 0, 0, 2);
            const double tXe = mXe * ip4<S>(mXe, Pm1, P00, Pp1, Pp2) + AT(ndTX, 0, 0, 0);
            const double tXw = mXw * ip4<S>(mXw, Pm2, Pm1, P00, Pp1) + AT(ndTX, 0, -1, 0);
            const double tYn = mYn * ip4<S>(mYn, Qm1, P00, Qp1, Qp2) + AT(ndTY, 0, 0, 0);
            const double tYs = mYs * ip4<S>(mYs, Qm2, Qm1, P00, Qp1) + AT(ndTY, 0, 0, -1);
            a.adv_t[c] = -((tXe - tXw) * rcdx + (tYn - tYs) * rcdy); // hevi_st :646-648
            put_flux(a, N3, 1, c, mXe, true);
            put_flux(a, N3, 2, c, mYn, true);
            put_flux(a, N3, 4, c, tXe, true);
            put_flux(a, N3, 5, c, tYn, true);
            if (i == g.IS) { put_flux(a, N3, 1, c - sI, mXw, false); put_flux(a, N3, 4, c - sI, tXw, false); }
            if (j == g.JS) { put_flux(a, N3, 2, c - sJ, mYs, false); put_flux(a, N3, 5, c - sJ, tYs, false); }
        }

        // ---- w-momentum horizontal fluxes, fluxX/Y_XYW (ud3.F90:598-748), hevi_sw :560-562 ----
        if (k <= KE - 1) {
            const double f1 = ld(g.F2H1 + k - 1), f2 = ld(g.F2H2 + k - 1);
            const double vXe = (f1 * AT(MX, 1, 0, 0) + f2 * AT(MX, 0, 0, 0))
                               / (f1 * 0.5 * (AT(DN, 1, 0, 0) + AT(DN, 1, 1, 0)) + f2 * 0.5 * (AT(DN, 0, 0, 0) + AT(DN, 0, 1, 0)));
            const double vXw = (f1 * AT(MX, 1, -1, 0) + f2 * AT(MX, 0, -1, 0))
                               / (f1 * 0.5 * (AT(DN, 1, -1, 0) + AT(DN, 1, 0, 0)) + f2 * 0.5 * (AT(DN, 0, -1, 0) + AT(DN, 0, 0, 0)));
            const double vYn = (f1 * AT(MY, 1, 0, 0) + f2 * AT(MY, 0, 0, 0))
                               / (f1 * 0.5 * (AT(DN, 1, 0, 0) + AT(DN, 1, 0, 1)) + f2 * 0.5 * (AT(DN, 0, 0, 0) + AT(DN, 0, 0, 1)));
            const double vYs = (f1 * AT(MY, 1, 0, -1) + f2 * AT(MY, 0, 0, -1))
                               / (f1 * 0.5 * (AT(DN, 1, 0, -1) + AT(DN, 1, 0, 0)) + f2 * 0.5 * (AT(DN, 0, 0, -1) + AT(DN, 0, 0, 0)));
            const double W_m2 = AT(MZ, 0, -2, 0), W_m1 = AT(MZ, 0, -1, 0), W_00 = AT(MZ, 0, 0, 0);
            const double W_p1 = AT(MZ, 0, 1, 0), W_p2 = AT(MZ, 0, 2, 0);
            const double V_m2 = AT(MZ, 0, 0, -2), V_m1 = AT(MZ, 0, 0, -1), V_p1 = AT(MZ, 0, 0, 1), V_p2 = AT(MZ, 0, 0, 2);
            const double qXe = vXe * ip4<S>(vXe, W_m1, W_00, W_p1, W_p2) + AT(ndWX, 0, 0, 0);
            const double qXw = vXw * ip4<S>(vXw, W_m2, W_m1, W_00, W_p1) + AT(ndWX, 0, -1, 0);
            const double qYn = vYn * ip4<S>(vYn, V_m1, W_00, V_p1, V_p2) + AT(ndWY, 0, 0, 0);
            const double qYs = vYs * ip4<S>(vYs, V_m2, V_m1, W_00, V_p1) + AT(ndWY, 0, 0, -1);
            a.adv_w[c] = -((qXe - qXw) * rcdx + (qYn - qYs) * rcdy);
        }

        // pressure deviation at the cell and its +x/+y neighbours, hevi_pres :355
        const double DP00 = AT(a.DPRES0, 0, 0, 0) + AT(a.RT2P, 0, 0, 0) * (AT(RT, 0, 0, 0) - AT(a.REF_rhot, 0, 0, 0));

        // ---- u momentum, hevi_momx :814-928 ----
        if (do_u) {
            // z flux at (u,y,w), fluxZ_UYZ (ud3.F90:753-859); m is the lower level of the face
            auto qZu = [&](int m) -> double {
                if (m < KS || m > KE - 1) return 0.0;
                const long dm = m - k;
                const double den = ld(g.F2H1 + m - 1) * 0.5 * (AT(DN, dm + 1, 0, 0) + AT(DN, dm + 1, 1, 0))
                                   + ld(g.F2H2 + m - 1) * 0.5 * (AT(DN, dm, 0, 0) + AT(DN, dm, 1, 0));
                const double vel = (0.5 * (AT(MZ, dm, 0, 0) + AT(MZ, dm, 1, 0))) / den;
                double q;
                if (m == KS) q = ipL<S>(vel, AT(MX, dm, 0, 0), AT(MX, dm + 1, 0, 0), AT(MX, dm + 2, 0, 0));
                else if (m == KE - 1) q = ipH<S>(vel, AT(MX, dm + 1, 0, 0), AT(MX, dm, 0, 0), AT(MX, dm - 1, 0, 0));
                else q = ip4<S>(vel, AT(MX, dm - 1, 0, 0), AT(MX, dm, 0, 0), AT(MX, dm + 1, 0, 0), AT(MX, dm + 2, 0, 0));
                return J33G * vel * q + AT(ndUZ, dm, 0, 0);
            };
            const double U_m2 = AT(MX, 0, -2, 0), U_m1 = AT(MX, 0, -1, 0), U_00 = AT(MX, 0, 0, 0);
            const double U_p1 = AT(MX, 0, 1, 0), U_p2 = AT(MX, 0, 2, 0);
            // x flux at (x,y,z) with the index shift of fluxX_UYZ (ud3.F90:1053-1109)
            const double vE = (0.5 * (U_p1 + U_00)) / (AT(DN, 0, 1, 0));
            const double qXe = vE * ip4<S>(vE, U_m1, U_00, U_p1, U_p2) + AT(ndUX, 0, 1, 0);
            const double vW = (0.5 * (U_00 + U_m1)) / (AT(DN, 0, 0, 0));
            const double qXw = vW * ip4<S>(vW, U_m2, U_m1, U_00, U_p1) + AT(ndUX, 0, 0, 0);
            // y flux at (u,v,z), fluxY_UYZ (ud3.F90:1113-1167)
            const double vN = (0.5 * (AT(MY, 0, 0, 0) + AT(MY, 0, 1, 0)))
                              / (0.25 * (AT(DN, 0, 0, 0) + AT(DN, 0, 1, 0) + AT(DN, 0, 0, 1) + AT(DN, 0, 1, 1)));
            const double qYn = vN * ip4<S>(vN, AT(MX, 0, 0, -1), U_00, AT(MX, 0, 0, 1), AT(MX, 0, 0, 2)) + AT(ndUY, 0, 0, 0);
            const double vS = (0.5 * (AT(MY, 0, 0, -1) + AT(MY, 0, 1, -1)))
                              / (0.25 * (AT(DN, 0, 0, -1) + AT(DN, 0, 1, -1) + AT(DN, 0, 0, 0) + AT(DN, 0, 1, 0)));
            const double qYs = vS * ip4<S>(vS, AT(MX, 0, 0, -2), AT(MX, 0, 0, -1), U_00, AT(MX, 0, 0, 1)) + AT(ndUY, 0, 0, -1);
            const double advcv = -(qZu(k) - qZu(k - 1)) * ld(g.RCDZ + k - 1);
            const double advch = -((qXe - qXw) * rfdx + (qYn - qYs) * rcdy);
            const double DPe = AT(a.DPRES0, 0, 1, 0) + AT(a.RT2P, 0, 1, 0) * (AT(RT, 0, 1, 0) - AT(a.REF_rhot, 0, 1, 0));
            const double pg = (DPe - DP00) * rfdx;
            const double cf = cor_u * (AT(MY, 0, 1, 0) + AT(MY, 0, 0, 0) + AT(MY, 0, 1, -1) + AT(MY, 0, 0, -1));
            const double div = use_div ? ddc * (AT(a.DDIV, 0, 1, 0) - AT(a.DDIV, 0, 0, 0)) * fdx : 0.0;
            const double val = AT(a.MOMX0, 0, 0, 0) + dt * ((((advcv + advch) - pg) + cf) + div + AT(a.MOMX_t, 0, 0, 0));
            put_state(a, N3, 2, a.MOMX_RK, a.MOMX0, c, val, true);
        }

        // ---- v momentum, hevi_momy :934-1048 ----
        if (do_v) {
            auto qZv = [&](int m) -> double {
                if (m < KS || m > KE - 1) return 0.0;
                const long dm = m - k;
                const double den = ld(g.F2H1 + m - 1) * 0.5 * (AT(DN, dm + 1, 0, 0) + AT(DN, dm + 1, 0, 1))
                                   + ld(g.F2H2 + m - 1) * 0.5 * (AT(DN, dm, 0, 0) + AT(DN, dm, 0, 1));
                const double vel = (0.5 * (AT(MZ, dm, 0, 0) + AT(MZ, dm, 0, 1))) / den;
                double q;
                if (m == KS) q = ipL<S>(vel, AT(MY, dm, 0, 0), AT(MY, dm + 1, 0, 0), AT(MY, dm + 2, 0, 0));
                else if (m == KE - 1) q = ipH<S>(vel, AT(MY, dm + 1, 0, 0), AT(MY, dm, 0, 0), AT(MY, dm - 1, 0, 0));
                else q = ip4<S>(vel, AT(MY, dm - 1, 0, 0), AT(MY, dm, 0, 0), AT(MY, dm + 1, 0, 0), AT(MY, dm + 2, 0, 0));
                return J33G * vel * q + AT(ndVZ, dm, 0, 0);
            };
            const double Y_m2 = AT(MY, 0, 0, -2), Y_m1 = AT(MY, 0, 0, -1), Y_00 = AT(MY, 0, 0, 0);
            const double Y_p1 = AT(MY, 0, 0, 1), Y_p2 = AT(MY, 0, 0, 2);
            // x flux at (u,v,z), fluxX_XVZ (ud3.F90:1473-1527)
            const double vE = (0.5 * (AT(MX, 0, 0, 0) + AT(MX, 0, 0, 1)))
                              / (0.25 * (AT(DN, 0, 0, 0) + AT(DN, 0, 1, 0) + AT(DN, 0, 0, 1) + AT(DN, 0, 1, 1)));
            const double qXe = vE * ip4<S>(vE, AT(MY, 0, -1, 0), Y_00, AT(MY, 0, 1, 0), AT(MY, 0, 2, 0)) + AT(ndVX, 0, 0, 0);
            const double vW = (0.5 * (AT(MX, 0, -1, 0) + AT(MX, 0, -1, 1)))
                              / (0.25 * (AT(DN, 0, -1, 0) + AT(DN, 0, 0, 0) + AT(DN, 0, -1, 1) + AT(DN, 0, 0, 1)));
            const double qXw = vW * ip4<S>(vW, AT(MY, 0, -2, 0), AT(MY, 0, -1, 0), Y_00, AT(MY, 0, 1, 0)) + AT(ndVX, 0, -1, 0);
            // y flux with the index shift of fluxY_XVZ (ud3.F90:1531-1587)
            const double vN = (0.5 * (Y_p1 + Y_00)) / (AT(DN, 0, 0, 1));
            const double qYn = vN * ip4<S>(vN, Y_m1, Y_00, Y_p1, Y_p2) + AT(ndVY, 0, 0, 1);
            const double vS = (0.5 * (Y_00 + Y_m1)) / (AT(DN, 0, 0, 0));
            const double qYs = vS * ip4<S>(vS, Y_m2, Y_m1, Y_00, Y_p1) + AT(ndVY, 0, 0, 0);
            const double advcv = -(qZv(k) - qZv(k - 1)) * ld(g.RCDZ + k - 1);
            const double advch = -((qXe - qXw) * rcdx + (qYn - qYs) * rfdy);
            const double DPn = AT(a.DPRES0, 0, 0, 1) + AT(a.RT2P, 0, 0, 1) * (AT(RT, 0, 0, 1) - AT(a.REF_rhot, 0, 0, 1));
            const double pg = (DPn - DP00) * rfdy;
            const double cf = cor_v * (AT(MX, 0, 0, 1) + AT(MX, 0, 0, 0) + AT(MX, 0, -1, 1) + AT(MX, 0, -1, 0));
            const double div = use_div ? ddc * (AT(a.DDIV, 0, 0, 1) - AT(a.DDIV, 0, 0, 0)) * fdy : 0.0;
            const double val = AT(a.MOMY0, 0, 0, 0) + dt * ((((advcv + advch) - pg) + cf) + div + AT(a.MOMY_t, 0, 0, 0));
            put_state(a, N3, 3, a.MOMY_RK, a.MOMY0, c, val, true);
        }
#undef AT
    }
}

// =============================================================================
// column kernel: vertical fluxes, sources, implicit solve, back-update
// =============================================================================
//
// One CTA owns a tile of TC consecutive columns (i .. i+TC-1 at one j), all
// levels. A column is KA contiguous doubles, so the tile of each field is one
// contiguous block and warp w reads column w with its lanes along k (256-byte
// coalesced accesses). The work runs in four phases over per-level arrays in
// shared memory (one array per quantity, [column][level], odd row pitch):
//   1. POTT = RHOT/DENS                                                 (k-parallel)
//   2. PT (theta at w-faces, valueW_Z), tZ (fluxZ_XYZ), Sr, St, A       (k-parallel)
//   3. right-hand side C of the tridiagonal system (:698-722)            (k-parallel)
//   4. Thomas solve, solve_direct :1092-1127                             (one thread per column)
//   5. back-update of DENS, RHOT, MOMZ and the vertical fluxes (:728-790) (k-parallel)
// The arithmetic of every value keeps the reference's operation order, so
// the results are bit-identical to the sequential formulation.
constexpr int MAXKA = 260;    // largest KA (KMAX + 4) the column kernel accepts
constexpr int COL_ARRAYS = 6; // per-level shared arrays

enum ColArr : int { CA_C = 0, CA_PT = 1, CA_A = 2, CA_SR = 3, CA_ST = 4, CA_TZ = 5 };
// CA_C holds POTT in phases 1-2, then the RHS C, then f, then the solution.
// CA_A holds A(k), then e(k) once level k is eliminated.

__host__ __device__ inline int col_pitch(int KA) { return KA | 1; }

template <int S>
__global__ void __launch_bounds__(32 * HEVI_COL_TC, HEVI_COL_MINB) k_hevi_column(const Grid g, const StageArgs a)
{
    extern __shared__ double sm[];
    const int TC = blockDim.y;
    const int lane = threadIdx.x, w = threadIdx.y;
    const int i0 = g.IS + blockIdx.x * TC;
    const int j = g.JS + blockIdx.y;
    const int i = i0 + w;           // this warp's column in the k-parallel phases
    const bool col_ok = i <= g.IE;
    const size_t N3 = n3(g);
    const int KS = g.KS, KE = g.KE;
    const int KP = col_pitch(g.KA);
    const size_t col = idx3(g, 1, i, j); // offset of level 1 of this warp's column
    const double *ndDZ = nd_slice(a, N3, 1, 1), *ndWZ = nd_slice(a, N3, 2, 1), *ndTZ = nd_slice(a, N3, 5, 1);
    const double dt = a.dtrk, J33G = a.J33G, dt2 = dt * dt;
    const bool use_div = a.divdmp_coef != 0.0;
    const double ddc = use_div ? a.divdmp_coef / dt : 0.0;
    // shared arrays: SA(arr, c, L) for column c of the tile, level L (1-based)
#define SA(arr, c, L) sm[((size_t)(arr) * TC + (c)) * KP + (L) - 1]
#define CL(p, L) ld((p) + col + (L) - 1)

    // ---- phase 1: POTT(L) = RHOT/DENS, :586-600 ----
    if (col_ok)
        for (int L = KS + lane; L <= KE; L += 32) SA(CA_C, w, L) = CL(a.RHOT, L) / CL(a.DENS, L);
    __syncthreads();

    // ---- phase 2: PT, tZ, Sr, St, A ----
    if (col_ok) {
        // valueW_Z (ud3.F90:98-153) with the w-momentum sign, and fluxZ_XYZ (ud3.F90:157-247)
        auto pt_tz = [&](int L, double &pt, double &tz) {
            if (L < KS || L > KE - 1) { pt = 0.0; tz = 0.0; return; }
            const double mZ = CL(ndDZ, L); // hevi_mflx_z :383-391 (flat terrain)
            const double M0 = CL(a.MOMZ, L);
            double pi, ti;
            if (L == KS) {
                const double P0 = SA(CA_C, w, L), P1 = SA(CA_C, w, L + 1), P2 = SA(CA_C, w, L + 2);
                pi = ipL<S>(M0, P0, P1, P2);
                ti = ipL<S>(mZ, P0, P1, P2);
            } else if (L == KE - 1) {
                const double Pm1 = SA(CA_C, w, L - 1), P0 = SA(CA_C, w, L), P1 = SA(CA_C, w, L + 1);
                pi = ipH<S>(M0, P1, P0, Pm1);
                ti = ipH<S>(mZ, P1, P0, Pm1);
            } else {
                const double Pm1 = SA(CA_C, w, L - 1), P0 = SA(CA_C, w, L), P1 = SA(CA_C, w, L + 1), P2 = SA(CA_C, w, L + 2);
                pi = ip4<S>(M0, Pm1, P0, P1, P2);
                ti = ip4<S>(mZ, Pm1, P0, P1, P2);
            }
            pt = pi;
            tz = mZ * ti + CL(ndTZ, L);
        };
        for (int L = KS + lane; L <= KE; L += 32) {
            double PT, tZ, PTm, tZm;
            pt_tz(L, PT, tZ);
            pt_tz(L - 1, PTm, tZm);
            (void)PTm;
            const double mZ = (L <= KE - 1) ? CL(ndDZ, L) : 0.0;
            const double mZm1 = (L - 1 >= KS) ? CL(ndDZ, L - 1) : 0.0;
            const double rcdz = ld(g.RCDZ + L - 1);
            // hevi_sr :464-467 and hevi_st :646-649 (metric factors are 1)
            const double Sr = (-(mZ - mZm1) * rcdz + CL(a.adv_r, L)) + CL(a.DENS_t, L);
            const double St = (-(tZ - tZm) * rcdz + CL(a.adv_t, L)) + CL(a.RHOT_t, L);
            const double RTL = CL(a.RT2P, L);
            SA(CA_PT, w, L) = PT;
            SA(CA_TZ, w, L) = tZ;
            SA(CA_SR, w, L) = Sr;
            SA(CA_ST, w, L) = St;
            SA(CA_A, w, L) = dt2 * J33G * rcdz * RTL * J33G; // :696
        }
    }
    __syncthreads();

    // ---- phase 3: right-hand side C(k) of the unknown levels k = KS..KE-1, :698-722 ----
    if (col_ok) {
        // vertical w-momentum flux at the level k+1/2 ... , fluxZ_XYW (ud3.F90:358-452), zero outside KS..KE-2
        auto qZ_at = [&](int k) -> double {
            if (k < KS || k > KE - 2) return 0.0;
            const double Mk = CL(a.MOMZ, k), Mk1 = CL(a.MOMZ, k + 1);
            const double vel = (0.5 * (Mk + Mk1)) / CL(a.DENS, k + 1);
            const double q = (k == KS) ? ipL<S>(vel, Mk, Mk1, CL(a.MOMZ, k + 2))
                                       : ip4<S>(vel, CL(a.MOMZ, k - 1), Mk, Mk1, CL(a.MOMZ, k + 2));
            return J33G * vel * q + CL(ndWZ, k + 1);
        };
        auto dpres = [&](int L) { return CL(a.DPRES0, L) + CL(a.RT2P, L) * (CL(a.RHOT, L) - CL(a.REF_rhot, L)); }; // :355
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            // hevi_sw :557-566
            const double advcv = -(qZ_at(k) - qZ_at(k - 1)) * ld(g.RFDZ + k - 1);
            const double wdmp = -ld(a.wdamp + k - 1) * CL(a.MOMZ0, k);
            const double div = use_div ? ddc * (CL(a.DDIV, k + 1) - CL(a.DDIV, k)) * ld(g.FDZ + k - 1) : 0.0;
            const double Sw = (advcv + CL(a.adv_w, k)) + wdmp + div + CL(a.MOMZ_t, k);
            const double rfdz = ld(g.RFDZ + k - 1);
            const double RTL1 = CL(a.RT2P, k + 1), RTL0 = CL(a.RT2P, k);
            const double pg = -(dpres(k + 1) + RTL1 * dt * SA(CA_ST, w, k + 1) - dpres(k) - RTL0 * dt * SA(CA_ST, w, k)) * rfdz * J33G
                              - GRAV * (ld(g.F2H1 + k - 1) * (CL(a.DENS, k + 1) - CL(a.REF_dens, k + 1) + SA(CA_SR, w, k + 1) * dt)
                                        + ld(g.F2H2 + k - 1) * (CL(a.DENS, k) - CL(a.REF_dens, k) + SA(CA_SR, w, k) * dt));
            SA(CA_C, w, k) = CL(a.MOMZ, k) + dt * (pg + Sw);
        }
    }
    __syncthreads();

    // ---- phase 4: Thomas solve, one thread per column (solve_direct :1110-1124) ----
    if (w == 0 && lane < TC && i0 + lane <= g.IE) {
        const int c = lane;
        double e_prev = 0.0, f_prev = 0.0;
        for (int k = KS; k <= KE - 1; ++k) {
            const double rfdz = ld(g.RFDZ + k - 1);
            const double B = GRAV * dt2 * J33G / (ld(g.CDZ + k) + ld(g.CDZ + k - 1));
            const double Ak = SA(CA_A, c, k), Ak1 = SA(CA_A, c, k + 1);
            const double F2 = 1.0 + (SA(CA_PT, c, k) * rfdz * (Ak1 + Ak));
            const double Ck = SA(CA_C, c, k);
            if (k == KS) {
                const double F1 = -(SA(CA_PT, c, k + 1) * rfdz * Ak1 + B);
                const double rdenom = 1.0 / F2;
                e_prev = -F1 * rdenom;
                f_prev = Ck * rdenom;
            } else if (k <= KE - 2) {
                const double F1 = -(SA(CA_PT, c, k + 1) * rfdz * Ak1 + B);
                const double F3 = -(SA(CA_PT, c, k - 1) * rfdz * Ak - B);
                const double rdenom = 1.0 / (F2 + F3 * e_prev);
                e_prev = -F1 * rdenom;
                f_prev = (Ck - F3 * f_prev) * rdenom;
            } else {
                const double F3 = -(SA(CA_PT, c, k - 1) * rfdz * Ak - B);
                f_prev = (Ck - F3 * f_prev) / (F2 + F3 * e_prev); // the solution at KE-1
            }
            SA(CA_A, c, k) = e_prev;
            SA(CA_C, c, k) = f_prev;
        }
        // back substitution, C(k) = e(k) C(k+1) + f(k)
        double Cnext = f_prev;
        for (int k = KE - 2; k >= KS; --k) {
            Cnext = SA(CA_A, c, k) * Cnext + SA(CA_C, c, k);
            SA(CA_C, c, k) = Cnext;
        }
        SA(CA_C, c, KE) = 0.0;
        SA(CA_C, c, KS - 1) = 0.0;
        SA(CA_PT, c, KE) = 0.0;
        SA(CA_PT, c, KS - 1) = 0.0;
    }
    __syncthreads();

    // ---- phase 5: back-update, :728-790 ----
    if (col_ok) {
        for (int m = KS + lane; m <= KE; m += 32) {
            const size_t c = col + m - 1;
            const double rcdz = ld(g.RCDZ + m - 1);
            const double Cm = SA(CA_C, w, m), Cm1 = SA(CA_C, w, m - 1);
            double adr, adt;
            if (m == KE) {
                adr = Cm1 * J33G * rcdz;
                adt = Cm1 * SA(CA_PT, w, KE - 1) * J33G * rcdz;
            } else if (m == KS) {
                adr = -Cm * J33G * rcdz;
                adt = -Cm * SA(CA_PT, w, KS) * J33G * rcdz;
            } else {
                adr = -(Cm - Cm1) * J33G * rcdz;
                adt = -(Cm * SA(CA_PT, w, m) - Cm1 * SA(CA_PT, w, m - 1)) * J33G * rcdz;
            }
            put_state(a, N3, 0, a.DENS_RK, a.DENS0, c, ld(a.DENS0 + c) + dt * (adr + SA(CA_SR, w, m)), true);
            put_state(a, N3, 4, a.RHOT_RK, a.RHOT0, c, ld(a.RHOT0 + c) + dt * (adt + SA(CA_ST, w, m)), true);
            if (m <= KE - 1) {
                put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, ld(a.MOMZ0 + c) + (Cm - ld(a.MOMZ + c)), true);
                put_flux(a, N3, 0, c, ld(ndDZ + c) + J33G * Cm, true);
                put_flux(a, N3, 3, c, SA(CA_TZ, w, m) + J33G * Cm * SA(CA_PT, w, m), true);
            } else {
                put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, 0.0, false);
                put_flux(a, N3, 0, c, 0.0, true);
                put_flux(a, N3, 3, c, 0.0, true);
            }
        }
        if (lane == 0) {
            // rigid-lid and surface values (:753-754) and the zero fluxes at KS-1 (:371, ud3.F90:222)
            put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, col + KS - 2, 0.0, false);
            put_flux(a, N3, 0, col + KS - 2, 0.0, false);
            put_flux(a, N3, 3, col + KS - 2, 0.0, false);
        }
    }
    // hevi_mflx_z :369-393 also fills the halo column i = IS-1 with the explicit
    // part of the vertical mass flux; the solver never updates it
    if (blockIdx.x == 0 && w == TC - 1 && (a.rk_mode == RK_PLAIN || a.rk_mode == RK_FINAL)) {
        const size_t ch = idx3(g, 1, g.IS - 1, j);
        for (int k = KS - 1 + lane; k <= KE; k += 32)
            a.mflx[ch + k - 1] = (k >= KS && k <= KE - 1) ? ld(ndDZ + ch + k - 1) : 0.0;
    }
#undef SA
#undef CL
}

// ---- host launchers ---------------------------------------------------------
cudaError_t launch_hevi_horiz(const Grid &g, const StageArgs &a, int scheme, cudaStream_t st)
{
    dim3 bh(32, HEVI_HORIZ_COLS);
    dim3 gh((g.IMAX + HEVI_HORIZ_COLS - 1) / HEVI_HORIZ_COLS, g.JMAX);
    if (scheme == UD3) k_hevi_horiz<UD3><<<gh, bh, 0, st>>>(g, a);
    else k_hevi_horiz<CD4><<<gh, bh, 0, st>>>(g, a);
    return cudaGetLastError();
}

// columns per CTA: HEVI_COL_TC, halved until HEVI_COL_MINB CTAs fit one SM's shared memory
static int column_tile(int KA)
{
    int tc = HEVI_COL_TC;
    while (tc > 1 && (size_t)COL_ARRAYS * tc * col_pitch(KA) * sizeof(double) > (size_t)224 * 1024 / HEVI_COL_MINB) tc /= 2;
    return tc;
}

cudaError_t launch_hevi_column(const Grid &g, const StageArgs &a, int scheme, cudaStream_t st)
{
    if (g.KA > MAXKA) return cudaErrorInvalidValue;
    const int TC = column_tile(g.KA);
    const size_t smem = (size_t)COL_ARRAYS * TC * col_pitch(g.KA) * sizeof(double);
    cudaError_t e = scheme == UD3
        ? cudaFuncSetAttribute(k_hevi_column<UD3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
        : cudaFuncSetAttribute(k_hevi_column<CD4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 bc(32, TC);
    dim3 gc((g.IMAX + TC - 1) / TC, g.JMAX);
    if (scheme == UD3) k_hevi_column<UD3><<<gc, bc, smem, st>>>(g, a);
    else k_hevi_column<CD4><<<gc, bc, smem, st>>>(g, a);
    return cudaGetLastError();
}

}  // namespace hevi
