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
__global__ void __launch_bounds__(128) k_hevi_horiz(const Grid g, const StageArgs a)
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
constexpr int MAXKA = 260; // largest KA (KMAX + 4) the column kernel accepts

template <int S>
__global__ void __launch_bounds__(128) k_hevi_column(const Grid g, const StageArgs a)
{
    const int i = g.IS - 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const int KS = g.KS, KE = g.KE;
    const size_t col = idx3(g, 1, i, j); // offset of level 1
    const double *ndDZ = nd_slice(a, N3, 1, 1), *ndWZ = nd_slice(a, N3, 2, 1), *ndTZ = nd_slice(a, N3, 5, 1);
#define CL(p, k) ld((p) + col + (k) - 1)

    if (i == g.IS - 1) {
        // hevi_mflx_z :369-393 also fills the halo column i = IS-1 with the
        // explicit part of the vertical mass flux; the solver never updates it
        if (a.rk_mode == RK_PLAIN || a.rk_mode == RK_FINAL) {
            a.mflx[col + KS - 2] = 0.0;
            for (int k = KS; k <= KE - 1; ++k) a.mflx[col + k - 1] = CL(ndDZ, k);
            a.mflx[col + KE - 1] = 0.0;
        }
        return;
    }

    const double dt = a.dtrk, J33G = a.J33G, dt2 = dt * dt;
    const bool use_div = a.divdmp_coef != 0.0;
    const double ddc = use_div ? a.divdmp_coef / dt : 0.0;

    // per-level values kept for the back substitution and the final update
    double e_[MAXKA], f_[MAXKA], pt_[MAXKA], sr_[MAXKA], st_[MAXKA], tz_[MAXKA];

    // sliding windows (suffix = level offset from the current level L)
    double Pm1 = 0.0, P0, P1, P2 = 0.0;           // POTT(L-1..L+2)
    double Mm2 = 0.0, Mm1 = 0.0, M0, M1 = 0.0;    // MOMZ(L-2..L+1)
    double Dm1 = 0.0, D0;                         // DENS(L-1), DENS(L)
    double Pd1, Pd2 = 0.0;                        // DENS(L+1), DENS(L+2) for POTT
    double mZm1 = 0.0, tZm1 = 0.0, qZm1 = 0.0;    // mZ(L-1), tZ(L-1), qZ(L-2)
    double PTm1 = 0.0, PTm2 = 0.0;                // PT(L-1), PT(L-2)
    double Am1 = 0.0, DPm1 = 0.0, RPm1 = 0.0, RDm1 = 0.0, Srm1 = 0.0, Stm1 = 0.0;
    double e_prev = 0.0, f_prev = 0.0, Cfin = 0.0;

    D0 = CL(a.DENS, KS);
    P0 = CL(a.RHOT, KS) / D0;
    Pd1 = CL(a.DENS, KS + 1);
    P1 = CL(a.RHOT, KS + 1) / Pd1;
    M0 = CL(a.MOMZ, KS);

    for (int L = KS; L <= KE; ++L) {
        // advance the look-ahead windows
        if (L + 2 <= KE) { Pd2 = CL(a.DENS, L + 2); P2 = CL(a.RHOT, L + 2) / Pd2; }
        if (L + 1 <= KE) M1 = CL(a.MOMZ, L + 1);

        // ---- level-L quantities ----
        const double mZ = (L <= KE - 1) ? CL(ndDZ, L) : 0.0; // hevi_mflx_z :383-391 (flat terrain)
        double PT = 0.0, tZ = 0.0;
        if (L <= KE - 1) {
            // valueW_Z (ud3.F90:98-153) and fluxZ_XYZ (ud3.F90:157-247)
            double pi, ti;
            if (L == KS) {
                pi = ipL<S>(M0, P0, P1, P2);
                ti = ipL<S>(mZ, P0, P1, P2);
            } else if (L == KE - 1) {
                pi = ipH<S>(M0, P1, P0, Pm1);
                ti = ipH<S>(mZ, P1, P0, Pm1);
            } else {
                pi = ip4<S>(M0, Pm1, P0, P1, P2);
                ti = ip4<S>(mZ, Pm1, P0, P1, P2);
            }
            PT = pi;
            tZ = mZ * ti + CL(ndTZ, L);
        }
        const double rcdz = ld(g.RCDZ + L - 1);
        // hevi_sr :464-467 and hevi_st :646-649 (metric factors are 1)
        const double Sr = (-(mZ - mZm1) * rcdz + CL(a.adv_r, L)) + CL(a.DENS_t, L);
        const double St = (-(tZ - tZm1) * rcdz + CL(a.adv_t, L)) + CL(a.RHOT_t, L);
        const double RTL = CL(a.RT2P, L);
        const double RH = CL(a.RHOT, L);
        const double DP = CL(a.DPRES0, L) + RTL * (RH - CL(a.REF_rhot, L)); // :355
        const double A = dt2 * J33G * rcdz * RTL * J33G;                   // :696
        const double RD = CL(a.REF_dens, L);
        pt_[L - 1] = PT; sr_[L - 1] = Sr; st_[L - 1] = St; tz_[L - 1] = tZ;

        if (L >= KS + 1) {
            const int k = L - 1; // unknown level solved in this iteration
            // vertical w-momentum flux at level k, fluxZ_XYW (ud3.F90:358-452, index shifted by -1)
            double qZ = 0.0;
            if (k <= KE - 2) {
                const double vel = (0.5 * (Mm1 + M0)) / D0;
                const double q = (k == KS) ? ipL<S>(vel, Mm1, M0, M1) : ip4<S>(vel, Mm2, Mm1, M0, M1);
                qZ = J33G * vel * q + CL(ndWZ, k + 1);
            }
            // hevi_sw :557-566
            const double advcv = -(qZ - qZm1) * ld(g.RFDZ + k - 1);
            const double wdmp = -ld(a.wdamp + k - 1) * CL(a.MOMZ0, k);
            const double div = use_div ? ddc * (CL(a.DDIV, k + 1) - CL(a.DDIV, k)) * ld(g.FDZ + k - 1) : 0.0;
            const double Sw = (advcv + CL(a.adv_w, k)) + wdmp + div + CL(a.MOMZ_t, k);
            // coefficients :698-709
            const double rfdz = ld(g.RFDZ + k - 1);
            const double B = GRAV * dt2 * J33G / (ld(g.CDZ + k) + ld(g.CDZ + k - 1));
            const double F2 = 1.0 + (PTm1 * rfdz * (A + Am1));
            // right-hand side :710-718
            const double pg = -(DP + RTL * dt * St - DPm1 - RPm1 * dt * Stm1) * rfdz * J33G
                              - GRAV * (ld(g.F2H1 + k - 1) * (D0 - RD + Sr * dt)
                                        + ld(g.F2H2 + k - 1) * (Dm1 - RDm1 + Srm1 * dt));
            const double C = Mm1 + dt * (pg + Sw);
            // Thomas forward sweep, solve_direct :1110-1121
            if (k == KS) {
                const double F1 = -(PT * rfdz * A + B);
                const double rdenom = 1.0 / F2;
                e_prev = -F1 * rdenom;
                f_prev = C * rdenom;
                e_[k - 1] = e_prev; f_[k - 1] = f_prev;
            } else if (k <= KE - 2) {
                const double F1 = -(PT * rfdz * A + B);
                const double F3 = -(PTm2 * rfdz * Am1 - B);
                const double rdenom = 1.0 / (F2 + F3 * e_prev);
                e_prev = -F1 * rdenom;
                f_prev = (C - F3 * f_prev) * rdenom;
                e_[k - 1] = e_prev; f_[k - 1] = f_prev;
            } else {
                const double F3 = -(PTm2 * rfdz * Am1 - B);
                Cfin = (C - F3 * f_prev) / (F2 + F3 * e_prev);
            }
            qZm1 = qZ;
        }

        // shift windows to L+1
        Pm1 = P0; P0 = P1; P1 = P2;
        Dm1 = D0; D0 = Pd1; Pd1 = Pd2;
        Mm2 = Mm1; Mm1 = M0; M0 = M1;
        mZm1 = mZ; tZm1 = tZ;
        PTm2 = PTm1; PTm1 = PT;
        Am1 = A; DPm1 = DP; RPm1 = RTL; RDm1 = RD; Srm1 = Sr; Stm1 = St;
    }

    // ---- back substitution and update, :728-790 ----
    const size_t c0 = col;
    auto fin = [&](int m, double Cm, double Cm1) {
        const size_t c = c0 + m - 1;
        const double rcdz = ld(g.RCDZ + m - 1);
        double adr, adt;
        if (m == KE) {
            adr = Cm1 * J33G * rcdz;
            adt = Cm1 * pt_[KE - 2] * J33G * rcdz;
        } else if (m == KS) {
            adr = -Cm * J33G * rcdz;
            adt = -Cm * pt_[KS - 1] * J33G * rcdz;
        } else {
            adr = -(Cm - Cm1) * J33G * rcdz;
            adt = -(Cm * pt_[m - 1] - Cm1 * pt_[m - 2]) * J33G * rcdz;
        }
        put_state(a, N3, 0, a.DENS_RK, a.DENS0, c, ld(a.DENS0 + c) + dt * (adr + sr_[m - 1]), true);
        put_state(a, N3, 4, a.RHOT_RK, a.RHOT0, c, ld(a.RHOT0 + c) + dt * (adt + st_[m - 1]), true);
        if (m <= KE - 1) {
            put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, ld(a.MOMZ0 + c) + (Cm - ld(a.MOMZ + c)), true);
            put_flux(a, N3, 0, c, ld(ndDZ + c) + J33G * Cm, true);
            put_flux(a, N3, 3, c, tz_[m - 1] + J33G * Cm * pt_[m - 1], true);
        } else {
            put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, 0.0, false);
            put_flux(a, N3, 0, c, 0.0, true);
            put_flux(a, N3, 3, c, 0.0, true);
        }
    };
    double Cnext = Cfin;             // C at level KE-1
    fin(KE, 0.0, Cnext);
    for (int k = KE - 2; k >= KS; --k) {
        const double Ck = e_[k - 1] * Cnext + f_[k - 1];
        fin(k + 1, Cnext, Ck);
        Cnext = Ck;
    }
    fin(KS, Cnext, 0.0);
    // rigid-lid and surface values (:753-754) and the zero fluxes at KS-1 (:371, ud3.F90:222)
    put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c0 + KS - 2, 0.0, false);
    put_flux(a, N3, 0, c0 + KS - 2, 0.0, false);
    put_flux(a, N3, 3, c0 + KS - 2, 0.0, false);
#undef CL
}

// ---- host launchers ---------------------------------------------------------
cudaError_t launch_hevi_horiz(const Grid &g, const StageArgs &a, int scheme, cudaStream_t st)
{
    dim3 bh(32, 4);
    dim3 gh((g.IMAX + 3) / 4, g.JMAX);
    if (scheme == UD3) k_hevi_horiz<UD3><<<gh, bh, 0, st>>>(g, a);
    else k_hevi_horiz<CD4><<<gh, bh, 0, st>>>(g, a);
    return cudaGetLastError();
}

cudaError_t launch_hevi_column(const Grid &g, const StageArgs &a, int scheme, cudaStream_t st)
{
    if (g.KA > MAXKA) return cudaErrorInvalidValue;
    dim3 bc(128);
    dim3 gc((g.IMAX + 1 + 127) / 128, g.JMAX);
    if (scheme == UD3) k_hevi_column<UD3><<<gc, bc, 0, st>>>(g, a);
    else k_hevi_column<CD4><<<gc, bc, 0, st>>>(g, a);
    return cudaGetLastError();
}

}  // namespace hevi
