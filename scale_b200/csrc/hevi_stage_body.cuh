// Device body of the fused HEVI stage (one CTA's tile, hevi_stage_block) and
// the per-cell pieces it shares with the HEVE stage: included by
// hevi_stage.cu, whose kernels run it with the read-only cache path, and by
// persist.cu, whose persistent short step reads with coherent loads
// (HEVI_COHERENT_LOADS) the fields that earlier phases of the same launch write.
#pragma once
#include "hevi_kernels.cuh"

// Launch shape. A CTA is HEVI_COL_TC warps, one column each; the tile is
// TX x (HEVI_COL_TC/TX) columns with TX one of the compiled widths
// STAGE_TILE_XS, chosen per workload (the default is the measured best on B200
// for KMAX = 128, or the autotuner's pick), as is the raster height.
#ifndef HEVI_COL_TC
#define HEVI_COL_TC 16 // columns (warps) per CTA
#endif
#ifndef HEVI_COL_MINB
#define HEVI_COL_MINB 2 // resident CTAs per SM the register allocator must allow
#endif
#include "hevi_epilogue.cuh"

namespace hevi {

// cell offsets are 32-bit (a field has fewer than 2^31 points, checked at setup)
#define AT(p, dk, di, dj) ld((p) + (int)(c + (dk) + (di) * sI + (dj) * sJ))
// an FP64 field used in the flux arithmetic
#define AR(p, dk, di, dj) R(AT(p, dk, di, dj))

// mass fluxes at the u/v faces of cell c, hevi_mflx_x/y :399-438
template <typename R> struct MassFlux { R Xe, Xw, Yn, Ys; };
template <typename R>
__device__ __forceinline__ MassFlux<R> mass_flux(const StageArgsT<R> &a, const Nd<R> &nd, int c, int sI, int sJ)
{
    MassFlux<R> m;
    m.Xe = AR(a.MOMX, 0, 0, 0) + AT(nd.DX(), 0, 0, 0);
    m.Xw = AR(a.MOMX, 0, -1, 0) + AT(nd.DX(), 0, -1, 0);
    m.Yn = AR(a.MOMY, 0, 0, 0) + AT(nd.DY(), 0, 0, 0);
    m.Ys = AR(a.MOMY, 0, 0, -1) + AT(nd.DY(), 0, 0, -1);
    return m;
}

// horizontal w-momentum flux divergence at cell c (k <= KE-1),
// fluxX/Y_XYW (ud3.F90:598-748), hevi_sw :560-562
template <int S, typename R>
__device__ __forceinline__ R adv_w_h(const Grid &g, const StageArgsT<R> &a, const Nd<R> &nd, int c, int k,
                                     int sI, int sJ, R rcdx, R rcdy)
{
    const double *MX = a.MOMX, *MY = a.MOMY, *MZ = a.MOMZ, *DN = a.DENS;
    const R f1 = R(ld(g.F2H1 + k - 1)), f2 = R(ld(g.F2H2 + k - 1)), h = R(0.5);
    const R vXe = (f1 * AR(MX, 1, 0, 0) + f2 * AR(MX, 0, 0, 0))
                  / (f1 * h * (AR(DN, 1, 0, 0) + AR(DN, 1, 1, 0)) + f2 * h * (AR(DN, 0, 0, 0) + AR(DN, 0, 1, 0)));
    const R vXw = (f1 * AR(MX, 1, -1, 0) + f2 * AR(MX, 0, -1, 0))
                  / (f1 * h * (AR(DN, 1, -1, 0) + AR(DN, 1, 0, 0)) + f2 * h * (AR(DN, 0, -1, 0) + AR(DN, 0, 0, 0)));
    const R vYn = (f1 * AR(MY, 1, 0, 0) + f2 * AR(MY, 0, 0, 0))
                  / (f1 * h * (AR(DN, 1, 0, 0) + AR(DN, 1, 0, 1)) + f2 * h * (AR(DN, 0, 0, 0) + AR(DN, 0, 0, 1)));
    const R vYs = (f1 * AR(MY, 1, 0, -1) + f2 * AR(MY, 0, 0, -1))
                  / (f1 * h * (AR(DN, 1, 0, -1) + AR(DN, 1, 0, 0)) + f2 * h * (AR(DN, 0, 0, -1) + AR(DN, 0, 0, 0)));
    constexpr bool W6 = wide_scheme(S); // the third points are read by the 6-point schemes only
    const R W_m2 = AR(MZ, 0, -2, 0), W_m1 = AR(MZ, 0, -1, 0), W_00 = AR(MZ, 0, 0, 0);
    const R W_p1 = AR(MZ, 0, 1, 0), W_p2 = AR(MZ, 0, 2, 0);
    const R V_m2 = AR(MZ, 0, 0, -2), V_m1 = AR(MZ, 0, 0, -1), V_p1 = AR(MZ, 0, 0, 1), V_p2 = AR(MZ, 0, 0, 2);
    const R W_m3 = W6 ? AR(MZ, 0, -3, 0) : R(0.0), W_p3 = W6 ? AR(MZ, 0, 3, 0) : R(0.0);
    const R V_m3 = W6 ? AR(MZ, 0, 0, -3) : R(0.0), V_p3 = W6 ? AR(MZ, 0, 0, 3) : R(0.0);
    const R qXe = vXe * ip6<S>(vXe, W_m2, W_m1, W_00, W_p1, W_p2, W_p3) + AT(nd.WX(), 0, 0, 0);
    const R qXw = vXw * ip6<S>(vXw, W_m3, W_m2, W_m1, W_00, W_p1, W_p2) + AT(nd.WX(), 0, -1, 0);
    const R qYn = vYn * ip6<S>(vYn, V_m2, V_m1, W_00, V_p1, V_p2, V_p3) + AT(nd.WY(), 0, 0, 0);
    const R qYs = vYs * ip6<S>(vYs, V_m3, V_m2, V_m1, W_00, V_p1, V_p2) + AT(nd.WY(), 0, 0, -1);
    return -((qXe - qXw) * rcdx + (qYn - qYs) * rcdy);
}

// rho*u (V = 0, hevi_momx :814-928) or rho*v (V = 1, hevi_momy :934-1048) of cell (k,i,j).
// Called by all 32 lanes of a warp for 32 consecutive levels of one column;
// 'valid' is false for lanes above KE. The z-face flux below a level is the
// one above the level of the previous lane, passed by a warp shuffle. The
// advective and Coriolis terms are flux arithmetic (R); the pressure gradient
// of the deviation from the base state and the update of the state are FP64.
// HEVE = true takes the divergence-damping term as the HEVE module writes it,
// divdmp_coef / dtrk * FDX(i) * (DDIV(i+1) - DDIV(i)) (tstep_short_fvm_heve.F90:907,
// :1154), instead of the HEVI form (DDIV(i+1) - DDIV(i)) * ... * FDX(i).
template <int S, int V, typename R, bool HEVE = false>
__device__ __forceinline__ void update_mom(const Grid &g, const StageArgsT<R> &a, const Nd<R> &nd, size_t N3, int k, int i,
                                           int j, bool valid)
{
    const int c = (int)idx3(g, k, i, j);
    const int sI = g.KA, sJ = g.KA * g.IA;
    const double *MX = a.MOMX, *MY = a.MOMY, *MZ = a.MOMZ, *DN = a.DENS, *RT = a.RHOT;
    const double dt = a.dtrk;
    const R J33G = R(a.J33G), h = R(0.5), qr = R(0.25);
    const bool use_div = a.divdmp_coef != 0.0;
    const R ddc = use_div ? R(a.divdmp_coef / dt) : R(0.0);
    const int KS = g.KS, KE = g.KE;
    const unsigned FULL = 0xffffffffu;
    constexpr bool W6 = wide_scheme(S); // the third points are read by the 6-point schemes only

    // z flux at (u,y,w), fluxZ_UYZ (ud3.F90:753-859); m is the lower level of the face
    auto qZu = [&](int m) -> R {
        if (m < KS || m > KE - 1) return R(0.0);
        const long dm = m - k;
        const R den = R(ld(g.F2H1 + m - 1)) * h * (AR(DN, dm + 1, 0, 0) + AR(DN, dm + 1, 1, 0))
                      + R(ld(g.F2H2 + m - 1)) * h * (AR(DN, dm, 0, 0) + AR(DN, dm, 1, 0));
        const R vel = (h * (AR(MZ, dm, 0, 0) + AR(MZ, dm, 1, 0))) / den;
        const R q = zface<S>(vel, m, KS, KE, [&](int l) { return AR(MX, l - k, 0, 0); });
        return J33G * vel * q + lds(nd.UZ() + c + dm);
    };
    // z flux at (x,v,w), fluxZ_XVZ (ud3.F90:1173-1279)
    auto qZv = [&](int m) -> R {
        if (m < KS || m > KE - 1) return R(0.0);
        const long dm = m - k;
        const R den = R(ld(g.F2H1 + m - 1)) * h * (AR(DN, dm + 1, 0, 0) + AR(DN, dm + 1, 0, 1))
                      + R(ld(g.F2H2 + m - 1)) * h * (AR(DN, dm, 0, 0) + AR(DN, dm, 0, 1));
        const R vel = (h * (AR(MZ, dm, 0, 0) + AR(MZ, dm, 0, 1))) / den;
        const R q = zface<S>(vel, m, KS, KE, [&](int l) { return AR(MY, l - k, 0, 0); });
        return J33G * vel * q + lds(nd.VZ() + c + dm);
    };

    // the flux through the face above this level; the one below comes from the
    // lane of the level below (lane 0 computes it)
    const bool do_u = V == 0 && i <= g.IEH, do_v = V == 1 && j <= g.JEH;
    if (!do_u && !do_v) return; // warp-uniform
    const R q_k = valid ? (V == 0 ? qZu(k) : qZv(k)) : R(0.0);
    R q_km = __shfl_up_sync(FULL, q_k, 1);
    if (!valid) return;
    if (threadIdx.x == 0) q_km = V == 0 ? qZu(k - 1) : qZv(k - 1);

    // pressure deviation at the cell and its +x/+y neighbours, hevi_pres :355
    const double DP00 = AT(a.DPRES0, 0, 0, 0) + AT(a.RT2P, 0, 0, 0) * (AT(RT, 0, 0, 0) - AT(a.REF_rhot, 0, 0, 0));

    if (do_u) {
        const R rcdy = R(ld(g.RCDY + j - 1)), fdx = R(ld(g.FDX + i - 1));
        const double rfdx = ld(g.RFDX + i - 1);
        const R cor_u = R(0.125) * (R(ld(a.CORIOLI + g.c2 + (i) + (size_t)g.IA * (j - 1))) + R(ld(a.CORIOLI + g.c2 + (i - 1) + (size_t)g.IA * (j - 1))));
        const R U_m2 = AR(MX, 0, -2, 0), U_m1 = AR(MX, 0, -1, 0), U_00 = AR(MX, 0, 0, 0);
        const R U_p1 = AR(MX, 0, 1, 0), U_p2 = AR(MX, 0, 2, 0);
        // x flux at (x,y,z) with the index shift of fluxX_UYZ (ud3.F90:1053-1109)
        const R vE = (h * (U_p1 + U_00)) / (AR(DN, 0, 1, 0));
        const R U_m3 = W6 ? AR(MX, 0, -3, 0) : R(0.0), U_p3 = W6 ? AR(MX, 0, 3, 0) : R(0.0);
        const R qXe = vE * ip6<S>(vE, U_m2, U_m1, U_00, U_p1, U_p2, U_p3) + AT(nd.UX(), 0, 1, 0);
        const R vW = (h * (U_00 + U_m1)) / (AR(DN, 0, 0, 0));
        const R qXw = vW * ip6<S>(vW, U_m3, U_m2, U_m1, U_00, U_p1, U_p2) + AT(nd.UX(), 0, 0, 0);
        // y flux at (u,v,z), fluxY_UYZ (ud3.F90:1113-1167)
        const R vN = (h * (AR(MY, 0, 0, 0) + AR(MY, 0, 1, 0)))
                     / (qr * (AR(DN, 0, 0, 0) + AR(DN, 0, 1, 0) + AR(DN, 0, 0, 1) + AR(DN, 0, 1, 1)));
        const R qYn = vN * ip6<S>(vN, W6 ? AR(MX, 0, 0, -2) : R(0.0), AR(MX, 0, 0, -1), U_00, AR(MX, 0, 0, 1),
                                  AR(MX, 0, 0, 2), W6 ? AR(MX, 0, 0, 3) : R(0.0)) + AT(nd.UY(), 0, 0, 0);
        const R vS = (h * (AR(MY, 0, 0, -1) + AR(MY, 0, 1, -1)))
                     / (qr * (AR(DN, 0, 0, -1) + AR(DN, 0, 1, -1) + AR(DN, 0, 0, 0) + AR(DN, 0, 1, 0)));
        const R qYs = vS * ip6<S>(vS, W6 ? AR(MX, 0, 0, -3) : R(0.0), AR(MX, 0, 0, -2), AR(MX, 0, 0, -1), U_00,
                                  AR(MX, 0, 0, 1), W6 ? AR(MX, 0, 0, 2) : R(0.0)) + AT(nd.UY(), 0, 0, -1);
        const R advcv = -(q_k - q_km) * R(ld(g.RCDZ + k - 1));
        const R advch = -((qXe - qXw) * R(rfdx) + (qYn - qYs) * rcdy);
        const double DPe = AT(a.DPRES0, 0, 1, 0) + AT(a.RT2P, 0, 1, 0) * (AT(RT, 0, 1, 0) - AT(a.REF_rhot, 0, 1, 0));
        const double pg = (DPe - DP00) * rfdx;
        const R cf = cor_u * (AR(MY, 0, 1, 0) + AR(MY, 0, 0, 0) + AR(MY, 0, 1, -1) + AR(MY, 0, 0, -1));
        const R div = !use_div ? R(0.0)
                      : HEVE ? ddc * fdx * (AT(a.DDIV, 0, 1, 0) - AT(a.DDIV, 0, 0, 0))
                             : ddc * (AT(a.DDIV, 0, 1, 0) - AT(a.DDIV, 0, 0, 0)) * fdx;
        const double val = lds(a.MOMX0 + c) + dt * (((((double)(advcv + advch)) - pg) + (double)cf) + (double)div + (double)lds(a.MOMX_t + c));
        put_state(a, N3, 2, a.MOMX_RK, a.MOMX0, c, val, true);
    }

    if (do_v) {
        const R rcdx = R(ld(g.RCDX + i - 1)), fdy = R(ld(g.FDY + j - 1));
        const double rfdy = ld(g.RFDY + j - 1);
        const R cor_v = R(-0.125) * (R(ld(a.CORIOLI + g.c2 + (i - 1) + (size_t)g.IA * (j))) + R(ld(a.CORIOLI + g.c2 + (i - 1) + (size_t)g.IA * (j - 1))));
        const R Y_m2 = AR(MY, 0, 0, -2), Y_m1 = AR(MY, 0, 0, -1), Y_00 = AR(MY, 0, 0, 0);
        const R Y_p1 = AR(MY, 0, 0, 1), Y_p2 = AR(MY, 0, 0, 2);
        // x flux at (u,v,z), fluxX_XVZ (ud3.F90:1473-1527)
        const R vE = (h * (AR(MX, 0, 0, 0) + AR(MX, 0, 0, 1)))
                     / (qr * (AR(DN, 0, 0, 0) + AR(DN, 0, 1, 0) + AR(DN, 0, 0, 1) + AR(DN, 0, 1, 1)));
        const R qXe = vE * ip6<S>(vE, W6 ? AR(MY, 0, -2, 0) : R(0.0), AR(MY, 0, -1, 0), Y_00, AR(MY, 0, 1, 0),
                                  AR(MY, 0, 2, 0), W6 ? AR(MY, 0, 3, 0) : R(0.0)) + AT(nd.VX(), 0, 0, 0);
        const R vW = (h * (AR(MX, 0, -1, 0) + AR(MX, 0, -1, 1)))
                     / (qr * (AR(DN, 0, -1, 0) + AR(DN, 0, 0, 0) + AR(DN, 0, -1, 1) + AR(DN, 0, 0, 1)));
        const R qXw = vW * ip6<S>(vW, W6 ? AR(MY, 0, -3, 0) : R(0.0), AR(MY, 0, -2, 0), AR(MY, 0, -1, 0), Y_00,
                                  AR(MY, 0, 1, 0), W6 ? AR(MY, 0, 2, 0) : R(0.0)) + AT(nd.VX(), 0, -1, 0);
        // y flux with the index shift of fluxY_XVZ (ud3.F90:1531-1587)
        const R vN = (h * (Y_p1 + Y_00)) / (AR(DN, 0, 0, 1));
        const R Y_m3 = W6 ? AR(MY, 0, 0, -3) : R(0.0), Y_p3 = W6 ? AR(MY, 0, 0, 3) : R(0.0);
        const R qYn = vN * ip6<S>(vN, Y_m2, Y_m1, Y_00, Y_p1, Y_p2, Y_p3) + AT(nd.VY(), 0, 0, 1);
        const R vS = (h * (Y_00 + Y_m1)) / (AR(DN, 0, 0, 0));
        const R qYs = vS * ip6<S>(vS, Y_m3, Y_m2, Y_m1, Y_00, Y_p1, Y_p2) + AT(nd.VY(), 0, 0, 0);
        const R advcv = -(q_k - q_km) * R(ld(g.RCDZ + k - 1));
        const R advch = -((qXe - qXw) * rcdx + (qYn - qYs) * R(rfdy));
        const double DPn = AT(a.DPRES0, 0, 0, 1) + AT(a.RT2P, 0, 0, 1) * (AT(RT, 0, 0, 1) - AT(a.REF_rhot, 0, 0, 1));
        const double pg = (DPn - DP00) * rfdy;
        const R cf = cor_v * (AR(MX, 0, 0, 1) + AR(MX, 0, 0, 0) + AR(MX, 0, -1, 1) + AR(MX, 0, -1, 0));
        const R div = !use_div ? R(0.0)
                      : HEVE ? ddc * fdy * (AT(a.DDIV, 0, 0, 1) - AT(a.DDIV, 0, 0, 0))
                             : ddc * (AT(a.DDIV, 0, 0, 1) - AT(a.DDIV, 0, 0, 0)) * fdy;
        const double val = lds(a.MOMY0 + c) + dt * (((((double)(advcv + advch)) - pg) + (double)cf) + (double)div + (double)lds(a.MOMY_t + c));
        put_state(a, N3, 3, a.MOMY_RK, a.MOMY0, c, val, true);
    }
}

// =============================================================================
// the stage kernel
// =============================================================================
constexpr int MAXKA = 260;    // largest KA (KMAX + 4) the kernel accepts
#if HEVI_COL_SCRATCH
constexpr int COL_ARRAYS = 3; // per-level shared arrays
#else
constexpr int COL_ARRAYS = 6;
#endif

enum ColArr : int { CA_C = 0, CA_PT = 1, CA_A = 2, CA_SR = 3, CA_ST = 4, CA_TZ = 5 };
// CA_C holds POTT in phases 1-2, then the RHS C, then f, then the solution.
// CA_A holds A(k), then e(k) once level k is eliminated.

__host__ __device__ inline int col_pitch(int KA) { return KA | 1; }

// One CTA's tile: block x of the launch over all members. The body of
// k_hevi_stage and of the stage phases of the persistent short step.
template <int S, typename R, int TX, int NM>
__device__ __forceinline__ void hevi_stage_block(const Grid &gt, const StageArgsT<R> &a, const BatchT<NM> &B, int x)
{
    extern __shared__ double sm[];
    constexpr int TC = HEVI_COL_TC, TY = TC / TX;
    static_assert(TX * TY == TC, "the tile width must divide the CTA's column count");
    int b;
    const Grid g = block_domain(gt, B, b, x); // this CTA's ensemble member (the domain itself when NM = 1)
    const int lane = threadIdx.x, w = threadIdx.y;
    const int tx = w % TX, ty = w / TX; // this warp's column in the tile
    // 2-D raster: consecutive CTAs walk down a.raster rows of tiles, then step
    // in i, so the CTAs resident together cover a compact patch
    int ti, tj;
    {
        const int nti = (g.IMAX + TX - 1) / TX, ntj = (g.JMAX + TY - 1) / TY, RJ = a.raster;
        const int grp = b / (nti * RJ), rem = b - grp * (nti * RJ);
        const int rows = min(RJ, ntj - grp * RJ);
        tj = grp * RJ + rem % rows;
        ti = rem / rows;
    }
    const int i0 = g.IS + ti * TX, j0 = g.JS + tj * TY;
    const int i = i0 + tx, j = j0 + ty; // this warp's column in the k-parallel phases
    const bool col_ok = i <= g.IE && j <= g.JE;
    const size_t N3 = n3(g);
    const int sI = g.KA, sJ = g.KA * g.IA;
    const int KS = g.KS, KE = g.KE;
    const int KP = col_pitch(g.KA);
    const int col = (int)idx3(g, 1, i, j); // offset of level 1 of this warp's column
    const Nd<R> nd(a, N3);
    const double dt = a.dtrk, J33G = a.J33G, dt2 = dt * dt;
    const bool use_div = a.divdmp_coef != 0.0;
    const R ddc = use_div ? R(a.divdmp_coef / dt) : R(0.0);
    const R rcdx = col_ok ? R(ld(g.RCDX + i - 1)) : R(0.0), rcdy = col_ok ? R(ld(g.RCDY + j - 1)) : R(0.0);
    // shared arrays: SA(arr, cc, L) for column cc of the tile, level L (1-based)
#define SA(arr, cc, L) sm[((size_t)(arr) * TC + (cc)) * KP + (L) - 1]
#define CL(p, L) ld((p) + col + (L) - 1)
#if HEVI_COL_SCRATCH
    // Sr, St, tZ of this warp's column in the global scratch (written and read
    // back by this CTA only; L2-cached loads see the block's own stores)
#define XS_PUT(q, L, v) (a.colscr[(size_t)((q) - CA_SR) * N3 + col + (L) - 1] = (v))
#define XS(q, L) __ldcg(a.colscr + (size_t)((q) - CA_SR) * N3 + col + (L) - 1)
#else
#define XS_PUT(q, L, v) (SA(q, w, L) = (v))
#define XS(q, L) R(SA(q, w, L))
#endif

    // ---- phase 1: POTT (:586-600), x/y mass fluxes (:399-438), Sr (:443-479), A (:696) ----
    if (col_ok) {
        for (int L = KS + lane; L <= KE; L += 32) {
            const int c = col + L - 1;
            SA(CA_C, w, L) = R(ld(a.RHOT + c)) / R(ld(a.DENS + c));
            const MassFlux<R> m = mass_flux(a, nd, c, sI, sJ);
            const R adv_r = -((m.Xe - m.Xw) * rcdx + (m.Yn - m.Ys) * rcdy);
            put_flux(a, N3, 1, c, m.Xe, true);
            put_flux(a, N3, 2, c, m.Yn, true);
            if (i == g.IS) put_flux(a, N3, 1, c - sI, m.Xw, false);
            if (j == g.JS) put_flux(a, N3, 2, c - sJ, m.Ys, false);
            const R mZ = (L <= KE - 1) ? ld(nd.DZ() + c) : R(0.0); // hevi_mflx_z :383-391 (flat terrain)
            const R mZm1 = (L - 1 >= KS) ? ld(nd.DZ() + c - 1) : R(0.0);
            const R rcdz = R(ld(g.RCDZ + L - 1));
            XS_PUT(CA_SR, L, (-(mZ - mZm1) * rcdz + adv_r) + lds(a.DENS_t + c));
            SA(CA_A, w, L) = dt2 * J33G * ld(g.RCDZ + L - 1) * ld(a.RT2P + c) * J33G;
        }
    }
    __syncthreads();

    // ---- phase 2: PT, tZ (valueW_Z ud3.F90:98-153, fluxZ_XYZ :157-247), x/y theta fluxes, St ----
    if (col_ok) {
        auto pt_tz = [&](int L, R &pt, R &tz) {
            if (L < KS || L > KE - 1) { pt = R(0.0); tz = R(0.0); return; }
            const R mZ = CL(nd.DZ(), L);
            const R M0 = R(CL(a.MOMZ, L));
            auto P = [&](int l) { return R(SA(CA_C, w, l)); };
            const R pi = zface<S>(M0, L, KS, KE, P), ti = zface<S>(mZ, L, KS, KE, P);
            pt = pi;
            tz = mZ * ti + lds(nd.TZ() + col + L - 1);
        };
        for (int L = KS + lane; L <= KE; L += 32) {
            const int c = col + L - 1;
            R PT, tZ, PTm, tZm;
            pt_tz(L, PT, tZ);
            pt_tz(L - 1, PTm, tZm);
            (void)PTm;
            // POTT at x-neighbours (from the tile when it holds them) and y-neighbours
            auto pott_x = [&](int d) -> R {
                const int td = tx + d;
                if (td >= 0 && td < TX && i + d <= g.IE) return R(SA(CA_C, w + d, L));
                return AR(a.RHOT, 0, d, 0) / AR(a.DENS, 0, d, 0);
            };
            auto pott_y = [&](int d) -> R {
                const int td = ty + d;
                if (td >= 0 && td < TY && j + d <= g.JE) return R(SA(CA_C, w + d * TX, L));
                return AR(a.RHOT, 0, 0, d) / AR(a.DENS, 0, 0, d);
            };
            constexpr bool W6 = wide_scheme(S);
            const R Pm2 = pott_x(-2), Pm1 = pott_x(-1), P00 = R(SA(CA_C, w, L)), Pp1 = pott_x(1), Pp2 = pott_x(2);
            const R Qm2 = pott_y(-2), Qm1 = pott_y(-1), Qp1 = pott_y(1), Qp2 = pott_y(2);
            const R Pm3 = W6 ? pott_x(-3) : R(0.0), Pp3 = W6 ? pott_x(3) : R(0.0);
            const R Qm3 = W6 ? pott_y(-3) : R(0.0), Qp3 = W6 ? pott_y(3) : R(0.0);
            const MassFlux<R> m = mass_flux(a, nd, c, sI, sJ);
            // fluxX/Y_XYZ (ud3.F90:251-353)
            const R tXe = m.Xe * ip6<S>(m.Xe, Pm2, Pm1, P00, Pp1, Pp2, Pp3) + AT(nd.TX(), 0, 0, 0);
            const R tXw = m.Xw * ip6<S>(m.Xw, Pm3, Pm2, Pm1, P00, Pp1, Pp2) + AT(nd.TX(), 0, -1, 0);
            const R tYn = m.Yn * ip6<S>(m.Yn, Qm2, Qm1, P00, Qp1, Qp2, Qp3) + AT(nd.TY(), 0, 0, 0);
            const R tYs = m.Ys * ip6<S>(m.Ys, Qm3, Qm2, Qm1, P00, Qp1, Qp2) + AT(nd.TY(), 0, 0, -1);
            const R adv_t = -((tXe - tXw) * rcdx + (tYn - tYs) * rcdy); // hevi_st :646-648
            put_flux(a, N3, 4, c, tXe, true);
            put_flux(a, N3, 5, c, tYn, true);
            if (i == g.IS) put_flux(a, N3, 4, c - sI, tXw, false);
            if (j == g.JS) put_flux(a, N3, 5, c - sJ, tYs, false);
            const R rcdz = R(ld(g.RCDZ + L - 1));
            SA(CA_PT, w, L) = PT;
            XS_PUT(CA_TZ, L, tZ);
            XS_PUT(CA_ST, L, (-(tZ - tZm) * rcdz + adv_t) + lds(a.RHOT_t + c)); // hevi_st :646-649
        }
    }
    __syncthreads();

    // ---- phase 3: Sw (hevi_sw :528-578) and the right-hand side C(k), k = KS..KE-1 (:698-722) ----
    if (col_ok) {
        const R J33R = R(J33G);
        // vertical w-momentum flux above level k, fluxZ_XYW (ud3.F90:358-452), zero outside KS..KE-2
        auto qZ_at = [&](int k) -> R {
            if (k < KS || k > KE - 2) return R(0.0);
            const R Mk = R(CL(a.MOMZ, k)), Mk1 = R(CL(a.MOMZ, k + 1));
            const R vel = (R(0.5) * (Mk + Mk1)) / R(CL(a.DENS, k + 1));
            // fluxZ_XYW writes flux(k) for k = KS..KE-2 (ud3.F90:376-432, ud5.F90:479-571)
            const R q = zface<S>(vel, k, KS, KE, [&](int l) { return R(CL(a.MOMZ, l)); });
            return J33R * vel * q + lds(nd.WZ() + col + k);
        };
        auto dpres = [&](int L) { return CL(a.DPRES0, L) + CL(a.RT2P, L) * (CL(a.RHOT, L) - CL(a.REF_rhot, L)); }; // :355
        for (int k0 = KS; k0 <= KE - 1; k0 += 32) {
            const int k = k0 + lane;
            const bool ok = k <= KE - 1;
            // the flux above level k; the one below is the previous lane's (lane 0 computes it)
            const R q_k = ok ? qZ_at(k) : R(0.0);
            R q_km = __shfl_up_sync(0xffffffffu, q_k, 1);
            if (!ok) continue;
            if (lane == 0) q_km = qZ_at(k - 1);
            const int c = col + k - 1;
            const R adv_w = adv_w_h<S>(g, a, nd, c, k, sI, sJ, rcdx, rcdy);
            const R advcv = -(q_k - q_km) * R(ld(g.RFDZ + k - 1));
            const R wdmp = -R(ld(a.wdamp + g.z0 + k - 1)) * R(CL(a.MOMZ0, k));
            const R div = use_div ? ddc * (CL(a.DDIV, k + 1) - CL(a.DDIV, k)) * R(ld(g.FDZ + k - 1)) : R(0.0);
            const R Sw = (advcv + adv_w) + wdmp + div + lds(a.MOMZ_t + c);
            const double rfdz = ld(g.RFDZ + k - 1);
            const double RTL1 = CL(a.RT2P, k + 1), RTL0 = CL(a.RT2P, k);
            const double pg = -(dpres(k + 1) + RTL1 * dt * (double)XS(CA_ST, k + 1) - dpres(k) - RTL0 * dt * (double)XS(CA_ST, k)) * rfdz * J33G
                              - GRAV * (ld(g.F2H1 + k - 1) * (CL(a.DENS, k + 1) - lds(a.REF_dens + c + 1) + (double)XS(CA_SR, k + 1) * dt)
                                        + ld(g.F2H2 + k - 1) * (CL(a.DENS, k) - lds(a.REF_dens + c) + (double)XS(CA_SR, k) * dt));
            SA(CA_C, w, k) = CL(a.MOMZ, k) + dt * (pg + (double)Sw);
        }
    }
    __syncthreads();

    // ---- phase 4: Thomas solve (warp 0) while the other warps update rho*u, rho*v ----
    if (w == 0) {
        if (lane < TC && i0 + lane % TX <= g.IE && j0 + lane / TX <= g.JE) {
            const int cc = lane;
            double e_prev = 0.0, f_prev = 0.0;
            for (int k = KS; k <= KE - 1; ++k) {
                const double rfdz = ld(g.RFDZ + k - 1);
                const double B = GRAV * dt2 * J33G / (ld(g.CDZ + k) + ld(g.CDZ + k - 1));
                const double Ak = SA(CA_A, cc, k), Ak1 = SA(CA_A, cc, k + 1);
                const double F2 = 1.0 + (SA(CA_PT, cc, k) * rfdz * (Ak1 + Ak));
                const double Ck = SA(CA_C, cc, k);
                if (k == KS) {
                    const double F1 = -(SA(CA_PT, cc, k + 1) * rfdz * Ak1 + B);
                    const double rdenom = 1.0 / F2;
                    e_prev = -F1 * rdenom;
                    f_prev = Ck * rdenom;
                } else if (k <= KE - 2) {
                    const double F1 = -(SA(CA_PT, cc, k + 1) * rfdz * Ak1 + B);
                    const double F3 = -(SA(CA_PT, cc, k - 1) * rfdz * Ak - B);
                    const double rdenom = 1.0 / (F2 + F3 * e_prev);
                    e_prev = -F1 * rdenom;
                    f_prev = (Ck - F3 * f_prev) * rdenom;
                } else {
                    const double F3 = -(SA(CA_PT, cc, k - 1) * rfdz * Ak - B);
                    f_prev = (Ck - F3 * f_prev) / (F2 + F3 * e_prev); // the solution at KE-1
                }
                SA(CA_A, cc, k) = e_prev;
                SA(CA_C, cc, k) = f_prev;
            }
            // back substitution, C(k) = e(k) C(k+1) + f(k)
            double Cnext = f_prev;
            for (int k = KE - 2; k >= KS; --k) {
                Cnext = SA(CA_A, cc, k) * Cnext + SA(CA_C, cc, k);
                SA(CA_C, cc, k) = Cnext;
            }
            SA(CA_C, cc, KE) = 0.0;
            SA(CA_C, cc, KS - 1) = 0.0;
            SA(CA_PT, cc, KS - 1) = 0.0;
        }
    }
    if (w > 0 || TC == 1) {
        // rho*u / rho*v of the tile: (32-level chunk, column, component) items over
        // the worker warps, chunk-major so that the warps work on one chunk of the
        // tile at a time and share its neighbour data in L1
        const int nworkers = TC > 1 ? TC - 1 : 1, wid = TC > 1 ? w - 1 : 0;
        const int NL = (g.KMAX + 31) / 32;
        for (int it = wid; it < 2 * TC * NL; it += nworkers) {
            const int item = it >> 1, cc = item % TC, L = KS + (item / TC) * 32 + lane;
            const int ii = i0 + cc % TX, jj = j0 + cc / TX;
            if (ii <= g.IE && jj <= g.JE) { // warp-uniform branch
                if (it & 1) update_mom<S, 1>(g, a, nd, N3, L, ii, jj, L <= KE);
                else update_mom<S, 0>(g, a, nd, N3, L, ii, jj, L <= KE);
            }
        }
    }
    __syncthreads();

    // ---- phase 5: back-update, :728-790 ----
    if (col_ok) {
        for (int m = KS + lane; m <= KE; m += 32) {
            const int c = col + m - 1;
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
            put_state(a, N3, 0, a.DENS_RK, a.DENS0, c, lds(a.DENS0 + c) + dt * (adr + (double)XS(CA_SR, m)), true);
            put_state(a, N3, 4, a.RHOT_RK, a.RHOT0, c, lds(a.RHOT0 + c) + dt * (adt + (double)XS(CA_ST, m)), true);
            if (m <= KE - 1) {
                put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, ld(a.MOMZ0 + c) + (Cm - ld(a.MOMZ + c)), true);
                put_flux(a, N3, 0, c, R((double)ld(nd.DZ() + c) + J33G * Cm), true);
                put_flux(a, N3, 3, c, R((double)XS(CA_TZ, m) + J33G * Cm * SA(CA_PT, w, m)), true);
            } else {
                put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, 0.0, false);
                put_flux(a, N3, 0, c, R(0.0), true);
                put_flux(a, N3, 3, c, R(0.0), true);
            }
        }
        if (lane == 0) {
            // rigid-lid and surface values (:753-754) and the zero fluxes at KS-1 (:371, ud3.F90:222)
            put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, col + KS - 2, 0.0, false);
            put_flux(a, N3, 0, col + KS - 2, R(0.0), false);
            put_flux(a, N3, 3, col + KS - 2, R(0.0), false);
        }
    }
    // hevi_mflx_z :369-393 also fills the halo column i = IS-1 with the explicit
    // part of the vertical mass flux; the solver never updates it
    if (ti == 0 && tx == 0 && col_ok && (a.rk_mode == RK_PLAIN || a.rk_mode == RK_FINAL || a.rk_mode == RK_HEUN3)) {
        const size_t ch = idx3(g, 1, g.IS - 1, j);
        for (int k = KS - 1 + lane; k <= KE; k += 32)
            a.mflx[ch + k - 1] = (k >= KS && k <= KE - 1) ? ld(nd.DZ() + ch + k - 1) : R(0.0);
    }
#undef SA
#undef CL
#undef XS
#undef XS_PUT
}

}  // namespace hevi
