/*
 * Oracle restatement of one HEVI short-step stage and the RK4 short integrator.
 *   ATMOS_DYN_Tstep_short_fvm_hevi : scale_atmos_dyn_tstep_short_fvm_hevi.F90:128-1089
 *   solve_direct                   : scale_atmos_dyn_tstep_short_fvm_hevi.F90:1092-1127
 *   check_equation                 : scale_atmos_dyn_tstep_short_fvm_hevi.F90:1131-1271
 *   ATMOS_DYN_tinteg_short_rk4     : scale_atmos_dyn_tinteg_short_rk4.F90:199-650
 * IBLOCK/JBLOCK take their default (the whole domain is one block,
 * scale_atmos_grid_cartesC_index.F90:267-268).
 */
#include "og_internal.h"

/* F2H of the HEVI module (tstep_short_fvm_hevi.F90:62): idx selects the GSQRT slice */
#define F2Hh(k, p, idx) (CDZ[(k) + (p) - 2] * GSQRT[I3((k) + (p) - 1, i, j) + ((size_t)(idx) - 1) * N3] /     \
                         (CDZ[(k) - 1] * GSQRT[I3(k, i, j) + ((size_t)(idx) - 1) * N3]                        \
                          + CDZ[(k)] * GSQRT[I3((k) + 1, i, j) + ((size_t)(idx) - 1) * N3]))
#define GS(k, i, j, idx) GSQRT[I3(k, i, j) + ((size_t)(idx) - 1) * N3]
#define J13(k, i, j, idx) J13G[I3(k, i, j) + ((size_t)(idx) - 1) * N3]
#define J23(k, i, j, idx) J23G[I3(k, i, j) + ((size_t)(idx) - 1) * N3]
#define MAPFv(i, j, a, b) MAPF[I2(i, j) + (size_t)IA * (size_t)JA * ((size_t)((a) - 1) + 2 * (size_t)((b) - 1))]
#define NDv(k, i, j, v, dir) num_diff[I3(k, i, j) + N3 * (size_t)(((v) - 1) + 5 * ((dir) - 1))]
#define COR(i, j) CORIOLI[I2(i, j)]

/* solve_direct, tstep_short_fvm_hevi.F90:1092-1127; C(1..KMAX-1) stored 0-based */
static void solve_direct(int KS, int KE, int KMAX, double *C, const double *F1, const double *F2, const double *F3,
                         double *e, double *f)
{
    (void)KE;
    double rdenom = 1.0 / F2[KS - 1];
    e[0] = -F1[KS - 1] * rdenom;
    f[0] = C[0] * rdenom;
    for (int k = 2; k <= KMAX - 2; ++k) {
        rdenom = 1.0 / (F2[k + KS - 2] + F3[k + KS - 2] * e[k - 2]);
        e[k - 1] = -F1[k + KS - 2] * rdenom;
        f[k - 1] = (C[k - 1] - F3[k + KS - 2] * f[k - 2]) * rdenom;
    }
    C[KMAX - 2] = (C[KMAX - 2] - F3[KE - 2] * f[KMAX - 3]) / (F2[KE - 2] + F3[KE - 2] * e[KMAX - 3]);
    for (int k = KMAX - 2; k >= 1; --k)
        C[k - 1] = e[k - 1] * C[k] + f[k - 1];
}

int og_stage_work_alloc(og_stage_work *w, size_t N3)
{
    w->POTT = og_alloc_undef(N3);
    w->DPRES = og_alloc_undef(N3);
    w->qflx_hi = og_alloc_undef(3 * N3);
    w->qflx_J13 = og_alloc_undef(N3);
    w->qflx_J23 = og_alloc_undef(N3);
    w->Sr = og_alloc_undef(N3);
    w->Sw = og_alloc_undef(N3);
    w->St = og_alloc_undef(N3);
    return (w->POTT && w->DPRES && w->qflx_hi && w->qflx_J13 && w->qflx_J23 && w->Sr && w->Sw && w->St) ? 0 : -1;
}
void og_stage_work_free(og_stage_work *w)
{
    free(w->POTT); free(w->DPRES); free(w->qflx_hi); free(w->qflx_J13); free(w->qflx_J23);
    free(w->Sr); free(w->Sw); free(w->St);
}

/* The stage body; the solver's vertical momentum C(:,i,j) can be exported for the residual check. */
static int hevi_stage(
    const og_dims *d, int scheme, og_stage_work *w, double *Cout,
    double *DENS_RK, double *MOMZ_RK, double *MOMX_RK, double *MOMY_RK, double *RHOT_RK,
    double *mflx_hi, double *tflx_hi,
    const double *DENS0, const double *MOMZ0, const double *MOMX0, const double *MOMY0, const double *RHOT0,
    const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY, const double *RHOT,
    const double *DENS_t, const double *MOMZ_t, const double *MOMX_t, const double *MOMY_t, const double *RHOT_t,
    const double *DPRES0, const double *RT2P, const double *CORIOLI,
    const double *num_diff, const double *wdamp_coef, double divdmp_coef, const double *DDIV,
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY,
    const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, double J33G,
    const double *MAPF, const double *REF_dens, const double *REF_rhot,
    double dtrk)
{
    OG_DIMS(d);
    const double GRAV = OG_GRAV;
    const int IFS_OFF = 1, JFS_OFF = 1; /* BND_W = BND_S = .false. (periodic) */
    const int IIS = IS, IIE = IE, JJS = JS, JJE = JE;
    const og_blk blk = {IIS, IIE, JJS, JJE};
    double *POTT = w->POTT, *DPRES = w->DPRES, *qflx_J13 = w->qflx_J13, *qflx_J23 = w->qflx_J23;
    double *Sr = w->Sr, *Sw = w->Sw, *St = w->St;
    double *qZ = w->qflx_hi, *qX = w->qflx_hi + N3, *qY = w->qflx_hi + 2 * N3;
    double *mZ = mflx_hi, *mX = mflx_hi + N3, *mY = mflx_hi + 2 * N3;
    double *tZ = tflx_hi, *tX = tflx_hi + N3, *tY = tflx_hi + 2 * N3;

    /* hevi_pres :343-361 */
#pragma omp parallel for collapse(2)
    for (int j = JJS; j <= JJE + 1; ++j)
        for (int i = IIS; i <= IIE + 1; ++i) {
            for (int k = KS; k <= KE; ++k)
                DPRES[I3(k, i, j)] = DPRES0[I3(k, i, j)] + RT2P[I3(k, i, j)] * (RHOT[I3(k, i, j)] - REF_rhot[I3(k, i, j)]);
            DPRES[I3(KS - 1, i, j)] = DPRES0[I3(KS - 1, i, j)] - DENS[I3(KS, i, j)] * (PHI[I3(KS - 1, i, j)] - PHI[I3(KS + 1, i, j)]);
            DPRES[I3(KE + 1, i, j)] = DPRES0[I3(KE + 1, i, j)] - DENS[I3(KE, i, j)] * (PHI[I3(KE + 1, i, j)] - PHI[I3(KE - 1, i, j)]);
        }

    /* hevi_mflx_z :365-397 */
#pragma omp parallel for collapse(2)
    for (int j = JJS; j <= JJE; ++j)
        for (int i = IIS - 1; i <= IIE; ++i) {
            mZ[I3(KS - 1, i, j)] = 0.0;
            for (int k = KS; k <= KE - 1; ++k)
                mZ[I3(k, i, j)] = J13(k, i, j, I_XYW) * 0.25 / MAPFv(i, j, 2, I_XY)
                                      * (MOMX[I3(k + 1, i, j)] + MOMX[I3(k + 1, i - 1, j)] + MOMX[I3(k, i, j)] + MOMX[I3(k, i - 1, j)])
                                  + J23(k, i, j, I_XYW) * 0.25 / MAPFv(i, j, 1, I_XY)
                                      * (MOMY[I3(k + 1, i, j)] + MOMY[I3(k + 1, i, j - 1)] + MOMY[I3(k, i, j)] + MOMY[I3(k, i, j - 1)])
                                  + GS(k, i, j, I_XYW) / (MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY)) * NDv(k, i, j, I_DENS, ZDIR);
            mZ[I3(KE, i, j)] = 0.0;
        }

    /* hevi_mflx_x :399-421 */
    {
        const int iss = (IIS - 1 > IS - IFS_OFF) ? IIS - 1 : IS - IFS_OFF;
        const int iee = IIE < IEH ? IIE : IEH;
#pragma omp parallel for collapse(2)
        for (int j = JJS; j <= JJE; ++j)
            for (int i = iss; i <= iee; ++i)
                for (int k = KS; k <= KE; ++k)
                    mX[I3(k, i, j)] = GS(k, i, j, I_UYZ) / MAPFv(i, j, 2, I_UY) * (MOMX[I3(k, i, j)] + NDv(k, i, j, I_DENS, XDIR));
    }
    /* :423-438 */
    {
        const int jss = (JJS - 1 > JS - JFS_OFF) ? JJS - 1 : JS - JFS_OFF;
        const int jee = JJE < JEH ? JJE : JEH;
#pragma omp parallel for collapse(2)
        for (int j = jss; j <= jee; ++j)
            for (int i = IIS; i <= IIE; ++i)
                for (int k = KS; k <= KE; ++k)
                    mY[I3(k, i, j)] = GS(k, i, j, I_XVZ) / MAPFv(i, j, 1, I_XV) * (MOMY[I3(k, i, j)] + NDv(k, i, j, I_DENS, YDIR));
    }

    /* hevi_sr :443-479 */
#pragma omp parallel for collapse(2)
    for (int j = JJS; j <= JJE; ++j)
        for (int i = IIS; i <= IIE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double advcv = -(mZ[I3(k, i, j)] - mZ[I3(k - 1, i, j)]) * RCDZ[k - 1];
                double advch = -((mX[I3(k, i, j)] - mX[I3(k, i - 1, j)]) * RCDX[i - 1]
                                 + (mY[I3(k, i, j)] - mY[I3(k, i, j - 1)]) * RCDY[j - 1]);
                Sr[I3(k, i, j)] = (advcv + advch) * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY) / GS(k, i, j, I_XYZ) + DENS_t[I3(k, i, j)];
            }

    /* momentum (z) fluxes :485-525 */
    og_fluxZ_XYW(d, scheme, qZ, MOMZ, MOMZ, DENS, G4(GSQRT, I_XYZ), J33G, ND(num_diff, I_MOMZ, ZDIR), blk);
    og_fluxJ13_XYW(d, scheme, qflx_J13, MOMX, MOMZ, DENS, G4(J13G, I_XYZ), MAPF4(MAPF, I_XY), blk);
    og_fluxJ23_XYW(d, scheme, qflx_J23, MOMY, MOMZ, DENS, G4(J23G, I_XYZ), MAPF4(MAPF, I_XY), blk);
    og_fluxX_XYW(d, scheme, qX, MOMX, MOMZ, DENS, G4(GSQRT, I_UYW), MAPF4(MAPF, I_UY), ND(num_diff, I_MOMZ, XDIR), CDZ, blk);
    og_fluxY_XYW(d, scheme, qY, MOMY, MOMZ, DENS, G4(GSQRT, I_XVW), MAPF4(MAPF, I_XV), ND(num_diff, I_MOMZ, YDIR), CDZ, blk);

    /* hevi_sw :528-578 */
#pragma omp parallel for collapse(2)
    for (int j = JJS; j <= JJE; ++j)
        for (int i = IIS; i <= IIE; ++i)
            for (int k = KS; k <= KE - 1; ++k) {
                double advcv = -(qZ[I3(k, i, j)] - qZ[I3(k - 1, i, j)]
                                 + qflx_J13[I3(k, i, j)] - qflx_J13[I3(k - 1, i, j)]
                                 + qflx_J23[I3(k, i, j)] - qflx_J23[I3(k - 1, i, j)]) * RFDZ[k - 1];
                double advch = -((qX[I3(k, i, j)] - qX[I3(k, i - 1, j)]) * RCDX[i - 1]
                                 + (qY[I3(k, i, j)] - qY[I3(k, i, j - 1)]) * RCDY[j - 1])
                               * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY);
                double wdmp = -wdamp_coef[k - 1] * MOMZ0[I3(k, i, j)];
                double div = divdmp_coef / dtrk * (DDIV[I3(k + 1, i, j)] - DDIV[I3(k, i, j)]) * FDZ[k - 1];
                Sw[I3(k, i, j)] = (advcv + advch) / GS(k, i, j, I_XYW) + wdmp + div + MOMZ_t[I3(k, i, j)];
            }

    /* POTT :586-598 (halo-extended) */
#pragma omp parallel for collapse(2)
    for (int j = JJS - d->JHALO; j <= JJE + d->JHALO; ++j)
        for (int i = IIS - d->IHALO; i <= IIE + d->IHALO; ++i)
            for (int k = KS; k <= KE; ++k)
                POTT[I3(k, i, j)] = RHOT[I3(k, i, j)] / DENS[I3(k, i, j)];

    /* theta fluxes :603-622 */
    og_fluxZ_XYZ(d, scheme, tZ, mZ, POTT, G4(GSQRT, I_XYW), ND(num_diff, I_RHOT, ZDIR), blk);
    og_fluxX_XYZ(d, scheme, tX, mX, POTT, G4(GSQRT, I_UYZ), ND(num_diff, I_RHOT, XDIR), blk);
    og_fluxY_XYZ(d, scheme, tY, mY, POTT, G4(GSQRT, I_XVZ), ND(num_diff, I_RHOT, YDIR), blk);

    /* hevi_st :625-661 */
#pragma omp parallel for collapse(2)
    for (int j = JJS; j <= JJE; ++j)
        for (int i = IIS; i <= IIE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double advcv = -(tZ[I3(k, i, j)] - tZ[I3(k - 1, i, j)]) * RCDZ[k - 1];
                double advch = -((tX[I3(k, i, j)] - tX[I3(k, i - 1, j)]) * RCDX[i - 1]
                                 + (tY[I3(k, i, j)] - tY[I3(k, i, j - 1)]) * RCDY[j - 1]);
                St[I3(k, i, j)] = (advcv + advch) * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY) / GS(k, i, j, I_XYZ) + RHOT_t[I3(k, i, j)];
            }

    /* hevi_solver :665-809 */
#pragma omp parallel for collapse(2)
    for (int j = JJS; j <= JJE; ++j)
        for (int i = IIS; i <= IIE; ++i) {
            double colbuf[6 * KA];
            double *A = colbuf, *PT = A + KA, *F1 = A + 2 * KA, *F2 = A + 3 * KA, *F3 = A + 4 * KA, *C = A + 5 * KA;
            double e[KMAX > 2 ? KMAX : 2], f[KMAX > 2 ? KMAX : 2];
            double mz_col[KA], pott_col[KA];
            for (int k = 1; k <= KA; ++k) { mz_col[k - 1] = MOMZ[I3(k, i, j)]; pott_col[k - 1] = POTT[I3(k, i, j)]; }
            og_valueW_Z(d, scheme, PT, mz_col, pott_col);

            for (int k = KS; k <= KE; ++k)
                A[k - 1] = dtrk * dtrk * J33G * RCDZ[k - 1] * RT2P[I3(k, i, j)] * J33G / GS(k, i, j, I_XYZ);
            double B = GRAV * (dtrk * dtrk) * J33G / (CDZ[KS] + CDZ[KS - 1]);
            F1[KS - 1] = -(PT[KS] * RFDZ[KS - 1] * A[KS] + B) / GS(KS, i, j, I_XYW);
            F2[KS - 1] = 1.0 + (PT[KS - 1] * RFDZ[KS - 1] * (A[KS] + A[KS - 1])) / GS(KS, i, j, I_XYW);
            for (int k = KS + 1; k <= KE - 2; ++k) {
                B = GRAV * (dtrk * dtrk) * J33G / (CDZ[k] + CDZ[k - 1]);
                F1[k - 1] = -(PT[k] * RFDZ[k - 1] * A[k] + B) / GS(k, i, j, I_XYW);
                F2[k - 1] = 1.0 + (PT[k - 1] * RFDZ[k - 1] * (A[k] + A[k - 1])) / GS(k, i, j, I_XYW);
                F3[k - 1] = -(PT[k - 2] * RFDZ[k - 1] * A[k - 1] - B) / GS(k, i, j, I_XYW);
            }
            B = GRAV * (dtrk * dtrk) * J33G / (CDZ[KE - 1] + CDZ[KE - 2]);
            F2[KE - 2] = 1.0 + (PT[KE - 2] * RFDZ[KE - 2] * (A[KE - 1] + A[KE - 2])) / GS(KE - 1, i, j, I_XYW);
            F3[KE - 2] = -(PT[KE - 3] * RFDZ[KE - 2] * A[KE - 2] - B) / GS(KE - 1, i, j, I_XYW);
            for (int k = KS; k <= KE - 1; ++k) {
                double pg = -(DPRES[I3(k + 1, i, j)] + RT2P[I3(k + 1, i, j)] * dtrk * St[I3(k + 1, i, j)]
                              - DPRES[I3(k, i, j)] - RT2P[I3(k, i, j)] * dtrk * St[I3(k, i, j)])
                                * RFDZ[k - 1] * J33G / GS(k, i, j, I_XYW)
                            - GRAV * (F2Hh(k, 1, I_XYZ) * (DENS[I3(k + 1, i, j)] - REF_dens[I3(k + 1, i, j)] + Sr[I3(k + 1, i, j)] * dtrk)
                                      + F2Hh(k, 2, I_XYZ) * (DENS[I3(k, i, j)] - REF_dens[I3(k, i, j)] + Sr[I3(k, i, j)] * dtrk));
                C[k - KS] = MOMZ[I3(k, i, j)] + dtrk * (pg + Sw[I3(k, i, j)]);
            }

            solve_direct(KS, KE, KMAX, C, F1, F2, F3, e, f);
            if (Cout)
                for (int k = KS; k <= KE - 1; ++k) Cout[I3(k, i, j)] = C[k - KS];

            for (int k = KS; k <= KE - 1; ++k) {
                mZ[I3(k, i, j)] = mZ[I3(k, i, j)] + J33G * C[k - KS] / (MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY));
                tZ[I3(k, i, j)] = tZ[I3(k, i, j)] + J33G * C[k - KS] * PT[k - 1] / (MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY));
                MOMZ_RK[I3(k, i, j)] = MOMZ0[I3(k, i, j)] + (C[k - KS] - MOMZ[I3(k, i, j)]);
            }
            MOMZ_RK[I3(KS - 1, i, j)] = 0.0;
            MOMZ_RK[I3(KE, i, j)] = 0.0;

            double advcv = -C[0] * J33G * RCDZ[KS - 1] / GS(KS, i, j, I_XYZ);
            DENS_RK[I3(KS, i, j)] = DENS0[I3(KS, i, j)] + dtrk * (advcv + Sr[I3(KS, i, j)]);
            advcv = -C[0] * PT[KS - 1] * J33G * RCDZ[KS - 1] / GS(KS, i, j, I_XYZ);
            RHOT_RK[I3(KS, i, j)] = RHOT0[I3(KS, i, j)] + dtrk * (advcv + St[I3(KS, i, j)]);
            for (int k = KS + 1; k <= KE - 1; ++k) {
                advcv = -(C[k - KS] - C[k - KS - 1]) * J33G * RCDZ[k - 1] / GS(k, i, j, I_XYZ);
                DENS_RK[I3(k, i, j)] = DENS0[I3(k, i, j)] + dtrk * (advcv + Sr[I3(k, i, j)]);
                advcv = -(C[k - KS] * PT[k - 1] - C[k - KS - 1] * PT[k - 2]) * J33G * RCDZ[k - 1] / GS(k, i, j, I_XYZ);
                RHOT_RK[I3(k, i, j)] = RHOT0[I3(k, i, j)] + dtrk * (advcv + St[I3(k, i, j)]);
            }
            advcv = C[KE - KS - 1] * J33G * RCDZ[KE - 1] / GS(KE, i, j, I_XYZ);
            DENS_RK[I3(KE, i, j)] = DENS0[I3(KE, i, j)] + dtrk * (advcv + Sr[I3(KE, i, j)]);
            advcv = C[KE - KS - 1] * PT[KE - 2] * J33G * RCDZ[KE - 1] / GS(KE, i, j, I_XYZ);
            RHOT_RK[I3(KE, i, j)] = RHOT0[I3(KE, i, j)] + dtrk * (advcv + St[I3(KE, i, j)]);
        }

    /* hevi_momx :814-928 */
    og_fluxZ_UYZ(d, scheme, qZ, MOMZ, MOMX, DENS, G4(GSQRT, I_UYW), J33G, ND(num_diff, I_MOMX, ZDIR), CDZ, blk);
    og_fluxJ13_UYZ(d, scheme, qflx_J13, MOMX, MOMX, DENS, G4(GSQRT, I_UYZ), G4(J13G, I_UYW), MAPF4(MAPF, I_UY), CDZ, blk);
    og_fluxJ23_UYZ(d, scheme, qflx_J23, MOMY, MOMX, DENS, G4(GSQRT, I_UYZ), G4(J23G, I_UYW), MAPF4(MAPF, I_UY), CDZ, blk);
    og_fluxX_UYZ(d, scheme, qX, MOMX, MOMX, DENS, G4(GSQRT, I_XYZ), MAPF4(MAPF, I_XY), ND(num_diff, I_MOMX, XDIR), blk);
    og_fluxY_UYZ(d, scheme, qY, MOMY, MOMX, DENS, G4(GSQRT, I_UVZ), MAPF4(MAPF, I_UV), ND(num_diff, I_MOMX, YDIR), blk);
    {
        const int iee = IIE < IEH ? IIE : IEH;
#pragma omp parallel for collapse(2)
        for (int j = JJS; j <= JJE; ++j)
            for (int i = IIS; i <= iee; ++i)
                for (int k = KS; k <= KE; ++k) {
                    double advcv = -(qZ[I3(k, i, j)] - qZ[I3(k - 1, i, j)]
                                     + qflx_J13[I3(k, i, j)] - qflx_J13[I3(k - 1, i, j)]
                                     + qflx_J23[I3(k, i, j)] - qflx_J23[I3(k - 1, i, j)]) * RCDZ[k - 1];
                    double advch = -((qX[I3(k, i, j)] - qX[I3(k, i - 1, j)]) * RFDX[i - 1]
                                     + (qY[I3(k, i, j)] - qY[I3(k, i, j - 1)]) * RCDY[j - 1])
                                   * MAPFv(i, j, 1, I_UY) * MAPFv(i, j, 2, I_UY);
                    double pg = ((GS(k, i + 1, j, I_XYZ) * DPRES[I3(k, i + 1, j)]
                                  - GS(k, i, j, I_XYZ) * DPRES[I3(k, i, j)]) * RFDX[i - 1]
                                 + (J13(k, i, j, I_UYW)
                                        * 0.5 * (F2Hh(k, 1, I_UYZ) * (DPRES[I3(k + 1, i + 1, j)] + DPRES[I3(k + 1, i, j)])
                                                 + F2Hh(k, 2, I_UYZ) * (DPRES[I3(k, i + 1, j)] + DPRES[I3(k, i, j)]))
                                    - J13(k - 1, i, j, I_UYW)
                                        * 0.5 * (F2Hh(k, 1, I_UYZ) * (DPRES[I3(k, i + 1, j)] + DPRES[I3(k, i, j)])
                                                 + F2Hh(k, 2, I_UYZ) * (DPRES[I3(k - 1, i + 1, j)] + DPRES[I3(k - 1, i, j)])))
                                       * RCDZ[k - 1])
                                * MAPFv(i, j, 1, I_UY);
                    double sumy = MOMY[I3(k, i, j)] + MOMY[I3(k, i, j - 1)] + MOMY[I3(k, i + 1, j)] + MOMY[I3(k, i + 1, j - 1)];
                    double cf = 0.125 * (COR(i + 1, j) + COR(i, j))
                                    * (MOMY[I3(k, i + 1, j)] + MOMY[I3(k, i, j)] + MOMY[I3(k, i + 1, j - 1)] + MOMY[I3(k, i, j - 1)])
                                + 0.25 * MAPFv(i, j, 1, I_UY) * MAPFv(i, j, 2, I_UY)
                                    * sumy
                                    * (sumy * 0.25 * (1.0 / MAPFv(i + 1, j, 2, I_XY) - 1.0 / MAPFv(i, j, 2, I_XY)) * RFDX[i - 1]
                                       - MOMX[I3(k, i, j)] * (1.0 / MAPFv(i, j, 1, I_UV) - 1.0 / MAPFv(i, j - 1, 1, I_UV)) * RCDY[j - 1])
                                    * 2.0 / (DENS[I3(k, i + 1, j)] + DENS[I3(k, i, j)]);
                    double div = divdmp_coef / dtrk * (DDIV[I3(k, i + 1, j)] / MAPFv(i + 1, j, 2, I_XY) - DDIV[I3(k, i, j)] / MAPFv(i, j, 1, I_XY))
                                 * MAPFv(i, j, 1, I_UY) * MAPFv(i, j, 2, I_UY) * FDX[i - 1];
                    MOMX_RK[I3(k, i, j)] = MOMX0[I3(k, i, j)]
                                           + dtrk * ((advcv + advch - pg) / GS(k, i, j, I_UYZ) + cf + div + MOMX_t[I3(k, i, j)]);
                }
    }

    /* hevi_momy :934-1048 */
    og_fluxZ_XVZ(d, scheme, qZ, MOMZ, MOMY, DENS, G4(GSQRT, I_XVW), J33G, ND(num_diff, I_MOMY, ZDIR), CDZ, blk);
    og_fluxJ13_XVZ(d, scheme, qflx_J13, MOMX, MOMY, DENS, G4(GSQRT, I_XVZ), G4(J13G, I_XVW), MAPF4(MAPF, I_XV), CDZ, blk);
    og_fluxJ23_XVZ(d, scheme, qflx_J23, MOMY, MOMY, DENS, G4(GSQRT, I_XVZ), G4(J23G, I_XVW), MAPF4(MAPF, I_XV), CDZ, blk);
    og_fluxX_XVZ(d, scheme, qX, MOMX, MOMY, DENS, G4(GSQRT, I_UVZ), MAPF4(MAPF, I_UV), ND(num_diff, I_MOMY, XDIR), blk);
    og_fluxY_XVZ(d, scheme, qY, MOMY, MOMY, DENS, G4(GSQRT, I_XYZ), MAPF4(MAPF, I_XY), ND(num_diff, I_MOMY, YDIR), blk);
    {
        const int jee = JJE < JEH ? JJE : JEH;
#pragma omp parallel for collapse(2)
        for (int j = JJS; j <= jee; ++j)
            for (int i = IIS; i <= IIE; ++i)
                for (int k = KS; k <= KE; ++k) {
                    double advcv = -(qZ[I3(k, i, j)] - qZ[I3(k - 1, i, j)]
                                     + qflx_J13[I3(k, i, j)] - qflx_J13[I3(k - 1, i, j)]
                                     + qflx_J23[I3(k, i, j)] - qflx_J23[I3(k - 1, i, j)]) * RCDZ[k - 1];
                    double advch = -((qX[I3(k, i, j)] - qX[I3(k, i - 1, j)]) * RCDX[i - 1]
                                     + (qY[I3(k, i, j)] - qY[I3(k, i, j - 1)]) * RFDY[j - 1])
                                   * MAPFv(i, j, 1, I_XV) * MAPFv(i, j, 2, I_XV);
                    double pg = ((GS(k, i, j + 1, I_XYZ) * DPRES[I3(k, i, j + 1)]
                                  - GS(k, i, j, I_XYZ) * DPRES[I3(k, i, j)]) * RFDY[j - 1]
                                 + (J23(k, i, j, I_XVW)
                                        * 0.5 * (F2Hh(k, 1, I_XVZ) * (DPRES[I3(k + 1, i, j + 1)] + DPRES[I3(k + 1, i, j)])
                                                 + F2Hh(k, 2, I_XVZ) * (DPRES[I3(k, i, j + 1)] + DPRES[I3(k, i, j)]))
                                    - J23(k - 1, i, j, I_XVW)
                                        * 0.5 * (F2Hh(k - 1, 1, I_XVZ) * (DPRES[I3(k, i, j + 1)] + DPRES[I3(k, i, j)])
                                                 + F2Hh(k - 1, 2, I_XVZ) * (DPRES[I3(k - 1, i, j + 1)] + DPRES[I3(k - 1, i, j)])))
                                       * RCDZ[k - 1])
                                * MAPFv(i, j, 2, I_XV);
                    double sumx = MOMX[I3(k, i, j)] + MOMX[I3(k, i - 1, j)] + MOMX[I3(k, i, j + 1)] + MOMX[I3(k, i - 1, j + 1)];
                    double cf = -0.125 * (COR(i, j + 1) + COR(i, j))
                                    * (MOMX[I3(k, i, j + 1)] + MOMX[I3(k, i, j)] + MOMX[I3(k, i - 1, j + 1)] + MOMX[I3(k, i - 1, j)])
                                - 0.25 * MAPFv(i, j, 1, I_XV) * MAPFv(i, j, 2, I_XV)
                                    * sumx
                                    * (MOMY[I3(k, i, j)] * (1.0 / MAPFv(i, j, 2, I_UV) - 1.0 / MAPFv(i - 1, j, 2, I_UV)) * RCDX[i - 1]
                                       - 0.25 * (MOMX[I3(k, i, j)] + MOMX[I3(k, i - 1, j)] + MOMX[I3(k, i, j + 1)] + MOMX[I3(k, i - 1, j + 1)])
                                           * (1.0 / MAPFv(i, j + 1, 1, I_XY) - 1.0 / MAPFv(i, j, 1, I_XY)) * RFDY[j - 1])
                                    * 2.0 / (DENS[I3(k, i, j + 1)] + DENS[I3(k, i, j)]);
                    double div = divdmp_coef / dtrk * (DDIV[I3(k, i, j + 1)] / MAPFv(i, j + 1, 1, I_XY) - DDIV[I3(k, i, j)] / MAPFv(i, j, 1, I_XY))
                                 * MAPFv(i, j, 1, I_XV) * MAPFv(i, j, 2, I_XV) * FDY[j - 1];
                    MOMY_RK[I3(k, i, j)] = MOMY0[I3(k, i, j)]
                                           + dtrk * ((advcv + advch - pg) / GS(k, i, j, I_XVZ) + cf + div + MOMY_t[I3(k, i, j)]);
                }
    }
    return 0;
}

int og_tstep_short_fvm_hevi(
    const og_dims *d, int scheme,
    double *DENS_RK, double *MOMZ_RK, double *MOMX_RK, double *MOMY_RK, double *RHOT_RK,
    double *mflx_hi, double *tflx_hi,
    const double *DENS0, const double *MOMZ0, const double *MOMX0, const double *MOMY0, const double *RHOT0,
    const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY, const double *RHOT,
    const double *DENS_t, const double *MOMZ_t, const double *MOMX_t, const double *MOMY_t, const double *RHOT_t,
    const double *DPRES0, const double *RT2P, const double *CORIOLI,
    const double *num_diff, const double *wdamp_coef, double divdmp_coef, const double *DDIV,
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY,
    const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, double J33G,
    const double *MAPF, const double *REF_dens, const double *REF_rhot,
    double dtrk)
{
    OG_DIMS(d);
    og_stage_work w;
    if (og_stage_work_alloc(&w, N3)) { og_stage_work_free(&w); return -1; }
    int rc = hevi_stage(d, scheme, &w, NULL, DENS_RK, MOMZ_RK, MOMX_RK, MOMY_RK, RHOT_RK, mflx_hi, tflx_hi,
                        DENS0, MOMZ0, MOMX0, MOMY0, RHOT0, DENS, MOMZ, MOMX, MOMY, RHOT,
                        DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, DPRES0, RT2P, CORIOLI,
                        num_diff, wdamp_coef, divdmp_coef, DDIV, CDZ, FDZ, FDX, FDY, RCDZ, RCDX, RCDY,
                        RFDZ, RFDX, RFDY, PHI, GSQRT, J13G, J23G, J33G, MAPF, REF_dens, REF_rhot, dtrk);
    og_stage_work_free(&w);
    return rc;
}

/* periodic COMM_vars8 on a single rank: every halo cell takes the value of its
 * periodic image (scale_comm_cartesC.F90:1600-2043, 2787-3023), all KA levels */
/* the halo exchange of a decomposed domain, when one is registered */
static og_halo_fn halo_hook = 0;
static void *halo_user = 0;

void og_set_halo_exchange(og_halo_fn fn, void *user)
{
    halo_hook = fn;
    halo_user = user;
}

void og_halo_periodic(const og_dims *d, double *var, int nfields)
{
    if (halo_hook) {
        halo_hook(var, nfields, halo_user);
        return;
    }
    OG_DIMS(d);
    const int IMAX = d->IMAX, JMAX = d->JMAX;
    for (int n = 0; n < nfields; ++n) {
        double *v = var + (size_t)n * N3;
#pragma omp parallel for collapse(2)
        for (int j = 1; j <= JA; ++j)
            for (int i = 1; i <= IA; ++i) {
                if (i >= IS && i <= IE && j >= JS && j <= JE) continue;
                int si = i < IS ? i + IMAX : (i > IE ? i - IMAX : i);
                int sj = j < JS ? j + JMAX : (j > JE ? j - JMAX : j);
                for (int k = 1; k <= KA; ++k) v[I3(k, i, j)] = v[I3(k, si, sj)];
            }
    }
}

/* the HEVI stage body with the signature of og_heve_stage */
static int hevi_stage_fn(
    const og_dims *d, int scheme, og_stage_work *w,
    double *DENS_RK, double *MOMZ_RK, double *MOMX_RK, double *MOMY_RK, double *RHOT_RK,
    double *mflx_hi, double *tflx_hi,
    const double *DENS0, const double *MOMZ0, const double *MOMX0, const double *MOMY0, const double *RHOT0,
    const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY, const double *RHOT,
    const double *DENS_t, const double *MOMZ_t, const double *MOMX_t, const double *MOMY_t, const double *RHOT_t,
    const double *DPRES0, const double *RT2P, const double *CORIOLI,
    const double *num_diff, const double *wdamp_coef, double divdmp_coef, const double *DDIV,
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY,
    const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, double J33G,
    const double *MAPF, const double *REF_dens, const double *REF_rhot,
    double dtrk)
{
    return hevi_stage(d, scheme, w, NULL, DENS_RK, MOMZ_RK, MOMX_RK, MOMY_RK, RHOT_RK, mflx_hi, tflx_hi,
                      DENS0, MOMZ0, MOMX0, MOMY0, RHOT0, DENS, MOMZ, MOMX, MOMY, RHOT,
                      DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, DPRES0, RT2P, CORIOLI,
                      num_diff, wdamp_coef, divdmp_coef, DDIV, CDZ, FDZ, FDX, FDY, RCDZ, RCDX, RCDY,
                      RFDZ, RFDX, RFDY, PHI, GSQRT, J13G, J23G, J33G, MAPF, REF_dens, REF_rhot, dtrk);
}

/* RK4 short integrator, tinteg_short_rk4.F90:199-650, periodic (Copy_boundary is a no-op);
 * stage is the registered short step (ATMOS_DYN_Tstep_short: HEVI or HEVE) */
static int tinteg_short_rk4(
    og_stage_fn stage, const og_dims *d, int scheme,
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT,
    double *mflx_hi, double *tflx_hi,
    const double *DENS_t, const double *MOMZ_t, const double *MOMX_t, const double *MOMY_t, const double *RHOT_t,
    const double *DPRES0, const double *RT2P, const double *CORIOLI,
    const double *num_diff, const double *wdamp_coef, double divdmp_coef, const double *DDIV,
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY,
    const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, double J33G,
    const double *MAPF, const double *REF_dens, const double *REF_rhot,
    double dt)
{
    OG_DIMS(d);
    /* module RK buffers start as UNDEF (rk4.F90:175-197) */
    double *RK[3];
    for (int s = 0; s < 3; ++s) RK[s] = og_alloc_undef(5 * N3);
    double *S0 = og_alloc(5 * N3);
    double *mRK = og_alloc_undef(3 * 3 * N3), *tRK = og_alloc_undef(3 * 3 * N3);
    og_stage_work w;
    int bad = og_stage_work_alloc(&w, N3) || !RK[0] || !RK[1] || !RK[2] || !S0 || !mRK || !tRK;
    if (bad) {
        for (int s = 0; s < 3; ++s) free(RK[s]);
        free(S0); free(mRK); free(tRK); og_stage_work_free(&w);
        return -1;
    }
    double *X[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    for (int v = 0; v < 5; ++v) memcpy(S0 + v * N3, X[v], N3 * sizeof(double));
    const double *X0[5] = {S0, S0 + N3, S0 + 2 * N3, S0 + 3 * N3, S0 + 4 * N3};

    const double dts[4] = {dt / 2.0, dt / 2.0, dt, dt};
    for (int s = 0; s < 4; ++s) {
        double *out[5];
        double *mo, *to;
        const double *in[5];
        if (s < 3) {
            for (int v = 0; v < 5; ++v) out[v] = RK[s] + v * N3;
            mo = mRK + (size_t)s * 3 * N3;
            to = tRK + (size_t)s * 3 * N3;
        } else {
            for (int v = 0; v < 5; ++v) out[v] = X[v];
            mo = mflx_hi;
            to = tflx_hi;
        }
        if (s == 0) for (int v = 0; v < 5; ++v) in[v] = X[v];
        else for (int v = 0; v < 5; ++v) in[v] = RK[s - 1] + v * N3;
        stage(d, scheme, &w, out[0], out[1], out[2], out[3], out[4], mo, to,
                   X0[0], X0[1], X0[2], X0[3], X0[4], in[0], in[1], in[2], in[3], in[4],
                   DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, DPRES0, RT2P, CORIOLI,
                   num_diff, wdamp_coef, divdmp_coef, DDIV, CDZ, FDZ, FDX, FDY, RCDZ, RCDX, RCDY,
                   RFDZ, RFDX, RFDY, PHI, GSQRT, J13G, J23G, J33G, MAPF, REF_dens, REF_rhot, dts[s]);
        if (s < 3) og_halo_periodic(d, RK[s], 5);
    }

    /* combine :562-650 */
    for (int v = 0; v < 5; ++v) {
        double *x = X[v];
        const double *r1 = RK[0] + v * N3, *r2 = RK[1] + v * N3, *r3 = RK[2] + v * N3, *x0 = X0[v];
        const int kend = (v == 1) ? KE - 1 : KE; /* MOMZ: KS..KE-1 */
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i)
                for (int k = KS; k <= kend; ++k) {
                    size_t q = I3(k, i, j);
                    x[q] = (r1[q] * 2.0 + r2[q] * 4.0 + r3[q] * 2.0 + x[q] - x0[q] * 3.0) / 6.0;
                }
    }
    for (int n = 0; n < 3; ++n) {
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i)
                for (int k = KS; k <= KE; ++k) {
                    size_t q = I3(k, i, j) + (size_t)n * N3;
                    mflx_hi[q] = (mRK[q] + mRK[q + 3 * N3] * 2.0 + mRK[q + 6 * N3] * 2.0 + mflx_hi[q]) / 6.0;
                    tflx_hi[q] = (tRK[q] + tRK[q + 3 * N3] * 2.0 + tRK[q + 6 * N3] * 2.0 + tflx_hi[q]) / 6.0;
                }
    }
    for (int s = 0; s < 3; ++s) free(RK[s]);
    free(S0); free(mRK); free(tRK); og_stage_work_free(&w);
    return 0;
}

int og_tinteg_short_rk4(
    const og_dims *d, int scheme,
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT,
    double *mflx_hi, double *tflx_hi,
    const double *DENS_t, const double *MOMZ_t, const double *MOMX_t, const double *MOMY_t, const double *RHOT_t,
    const double *DPRES0, const double *RT2P, const double *CORIOLI,
    const double *num_diff, const double *wdamp_coef, double divdmp_coef, const double *DDIV,
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY,
    const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, double J33G,
    const double *MAPF, const double *REF_dens, const double *REF_rhot,
    double dt)
{
    return tinteg_short_rk4(hevi_stage_fn, d, scheme, DENS, MOMZ, MOMX, MOMY, RHOT, mflx_hi, tflx_hi, DENS_t, MOMZ_t, MOMX_t, MOMY_t,
                            RHOT_t, DPRES0, RT2P, CORIOLI, num_diff, wdamp_coef, divdmp_coef, DDIV, CDZ, FDZ, FDX, FDY,
                            RCDZ, RCDX, RCDY, RFDZ, RFDX, RFDY, PHI, GSQRT, J13G, J23G, J33G, MAPF, REF_dens,
                            REF_rhot, dt);
}

/* RK3 short integrator, tinteg_short_rk3.F90:188-576 (setup :89-184): the
 * registered short step at dt*(1/3), dt*fact_dt2 and dt, each of the first two
 * followed by the periodic halo of its output; fact_dt2 = 1/2 for RK3WS2002
 * (the result is the third stage), 2/3 for RK3 (Heun: the state becomes
 * (r1*3 + r3*3 - phi0*2)/4 and the fluxes (F1 + F3*3)/4 on the interior, :486-566) */
static int tinteg_short_rk3(
    og_stage_fn stage, int ws2002, const og_dims *d, int scheme,
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT,
    double *mflx_hi, double *tflx_hi,
    const double *DENS_t, const double *MOMZ_t, const double *MOMX_t, const double *MOMY_t, const double *RHOT_t,
    const double *DPRES0, const double *RT2P, const double *CORIOLI,
    const double *num_diff, const double *wdamp_coef, double divdmp_coef, const double *DDIV,
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY,
    const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, double J33G,
    const double *MAPF, const double *REF_dens, const double *REF_rhot,
    double dt)
{
    OG_DIMS(d);
    const double fact_dt1 = 1.0 / 3.0, fact_dt2 = ws2002 ? 1.0 / 2.0 : 2.0 / 3.0;
    double *RK[2] = {og_alloc_undef(5 * N3), og_alloc_undef(5 * N3)};
    double *S0 = og_alloc(5 * N3);
    double *mRK = og_alloc_undef(2 * 3 * N3), *tRK = og_alloc_undef(2 * 3 * N3);
    og_stage_work w;
    int bad = og_stage_work_alloc(&w, N3) || !RK[0] || !RK[1] || !S0 || !mRK || !tRK;
    if (bad) {
        free(RK[0]); free(RK[1]); free(S0); free(mRK); free(tRK); og_stage_work_free(&w);
        return -1;
    }
    double *X[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    for (int v = 0; v < 5; ++v) memcpy(S0 + v * N3, X[v], N3 * sizeof(double));
    const double *X0[5] = {S0, S0 + N3, S0 + 2 * N3, S0 + 3 * N3, S0 + 4 * N3};
    const double dts[3] = {dt * fact_dt1, dt * fact_dt2, dt};
    for (int s = 0; s < 3; ++s) {
        double *out[5], *mo, *to;
        const double *in[5];
        if (s < 2) {
            for (int v = 0; v < 5; ++v) out[v] = RK[s] + v * N3;
            mo = mRK + (size_t)s * 3 * N3;
            to = tRK + (size_t)s * 3 * N3;
        } else {
            for (int v = 0; v < 5; ++v) out[v] = X[v];
            mo = mflx_hi;
            to = tflx_hi;
        }
        if (s == 0) for (int v = 0; v < 5; ++v) in[v] = X[v];
        else for (int v = 0; v < 5; ++v) in[v] = RK[s - 1] + v * N3;
        stage(d, scheme, &w, out[0], out[1], out[2], out[3], out[4], mo, to,
              X0[0], X0[1], X0[2], X0[3], X0[4], in[0], in[1], in[2], in[3], in[4],
              DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, DPRES0, RT2P, CORIOLI,
              num_diff, wdamp_coef, divdmp_coef, DDIV, CDZ, FDZ, FDX, FDY, RCDZ, RCDX, RCDY,
              RFDZ, RFDX, RFDY, PHI, GSQRT, J13G, J23G, J33G, MAPF, REF_dens, REF_rhot, dts[s]);
        if (s < 2) og_halo_periodic(d, RK[s], 5);
    }
    if (!ws2002) {
        for (int v = 0; v < 5; ++v) {
            double *x = X[v];
            const double *r1 = RK[0] + v * N3, *x0 = X0[v];
            const int kend = (v == 1) ? KE - 1 : KE; /* MOMZ: KS..KE-1 */
#pragma omp parallel for collapse(2)
            for (int j = JS; j <= JE; ++j)
                for (int i = IS; i <= IE; ++i)
                    for (int k = KS; k <= kend; ++k) {
                        size_t q = I3(k, i, j);
                        x[q] = (r1[q] * 3.0 + x[q] * 3.0 - x0[q] * 2.0) / 4.0;
                    }
        }
        for (int n = 0; n < 3; ++n) {
#pragma omp parallel for collapse(2)
            for (int j = JS; j <= JE; ++j)
                for (int i = IS; i <= IE; ++i)
                    for (int k = KS; k <= KE; ++k) {
                        size_t q = I3(k, i, j) + (size_t)n * N3;
                        mflx_hi[q] = (mRK[q] + mflx_hi[q] * 3.0) / 4.0;
                        tflx_hi[q] = (tRK[q] + tflx_hi[q] * 3.0) / 4.0;
                    }
        }
    }
    free(RK[0]); free(RK[1]); free(S0); free(mRK); free(tRK);
    og_stage_work_free(&w);
    return 0;
}

int og_tinteg_short_rk3(
    const og_dims *d, int scheme, int ws2002,
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT,
    double *mflx_hi, double *tflx_hi,
    const double *DENS_t, const double *MOMZ_t, const double *MOMX_t, const double *MOMY_t, const double *RHOT_t,
    const double *DPRES0, const double *RT2P, const double *CORIOLI,
    const double *num_diff, const double *wdamp_coef, double divdmp_coef, const double *DDIV,
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY,
    const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, double J33G,
    const double *MAPF, const double *REF_dens, const double *REF_rhot,
    double dt)
{
    return tinteg_short_rk3(og_short_type_get() ? og_heve_stage : hevi_stage_fn, ws2002, d, scheme, DENS, MOMZ,
                            MOMX, MOMY, RHOT, mflx_hi, tflx_hi, DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, DPRES0, RT2P,
                            CORIOLI, num_diff, wdamp_coef, divdmp_coef, DDIV, CDZ, FDZ, FDX, FDY, RCDZ, RCDX, RCDY,
                            RFDZ, RFDX, RFDY, PHI, GSQRT, J13G, J23G, J33G, MAPF, REF_dens, REF_rhot, dt);
}

/* the same RK4 with the HEVE short step registered (ATMOS_DYN_TSTEP_SHORT_TYPE = "HEVE") */
int og_tinteg_short_rk4_heve(
    const og_dims *d, int scheme,
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT,
    double *mflx_hi, double *tflx_hi,
    const double *DENS_t, const double *MOMZ_t, const double *MOMX_t, const double *MOMY_t, const double *RHOT_t,
    const double *DPRES0, const double *RT2P, const double *CORIOLI,
    const double *num_diff, const double *wdamp_coef, double divdmp_coef, const double *DDIV,
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY,
    const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, double J33G,
    const double *MAPF, const double *REF_dens, const double *REF_rhot,
    double dt)
{
    return tinteg_short_rk4(og_heve_stage, d, scheme, DENS, MOMZ, MOMX, MOMY, RHOT, mflx_hi, tflx_hi, DENS_t, MOMZ_t, MOMX_t, MOMY_t,
                            RHOT_t, DPRES0, RT2P, CORIOLI, num_diff, wdamp_coef, divdmp_coef, DDIV, CDZ, FDZ, FDX, FDY,
                            RCDZ, RCDX, RCDY, RFDZ, RFDX, RFDY, PHI, GSQRT, J13G, J23G, J33G, MAPF, REF_dens,
                            REF_rhot, dt);
}

/* check_equation port: returns the largest |error| the reference's DEBUG check
 * would compute over all interior columns (it aborts above 1e-6). Valid for the
 * combination the check was written for: CD4 face values and uniform dz. */
double og_hevi_max_residual(
    const og_dims *d, int scheme,
    const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY, const double *RHOT,
    const double *DPRES0, const double *RT2P, const double *num_diff,
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY,
    const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *REF_dens, const double *REF_rhot, double dtrk)
{
    OG_DIMS(d);
    const double small = 1e-6, GRAV = OG_GRAV, J33G = 1.0;
    double *zero = (double *)calloc(N3, sizeof(double));
    double *one = og_alloc(7 * N3), *jz = (double *)calloc(7 * N3, sizeof(double));
    double *mapf = og_alloc((size_t)IA * JA * 8), *cor = (double *)calloc((size_t)IA * JA, sizeof(double));
    double *wd = (double *)calloc(KA, sizeof(double));
    double *out = og_alloc(5 * N3), *mflx = (double *)calloc(3 * N3, sizeof(double)), *tflx = (double *)calloc(3 * N3, sizeof(double));
    double *C = (double *)calloc(N3, sizeof(double));
    og_stage_work w;
    memset(&w, 0, sizeof(w));
    double worst = 0.0;
    if (!zero || !one || !jz || !mapf || !cor || !wd || !out || !mflx || !tflx || !C || og_stage_work_alloc(&w, N3)) {
        worst = INFINITY;
        goto done;
    }
    for (size_t q = 0; q < 7 * N3; ++q) one[q] = 1.0;
    for (size_t q = 0; q < (size_t)IA * JA * 8; ++q) mapf[q] = 1.0;
    hevi_stage(d, scheme, &w, C, out, out + N3, out + 2 * N3, out + 3 * N3, out + 4 * N3, mflx, tflx,
               DENS, MOMZ, MOMX, MOMY, RHOT, DENS, MOMZ, MOMX, MOMY, RHOT, zero, zero, zero, zero, zero,
               DPRES0, RT2P, cor, num_diff, wd, 0.0, zero, CDZ, FDZ, FDX, FDY, RCDZ, RCDX, RCDY,
               RFDZ, RFDX, RFDY, PHI, one, jz, jz, J33G, mapf, REF_dens, REF_rhot, dtrk);
    for (int j = JS; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i) {
            double MZ[KA], DN[KA], RN[KA], DP[KA], PO[KA], PT[KA];
            for (int k = 1; k <= KA; ++k) MZ[k - 1] = 0.0;
            for (int k = KS; k <= KE - 1; ++k) MZ[k - 1] = C[I3(k, i, j)];
            for (int k = KS + 1; k <= KE - 1; ++k)
                DN[k - 1] = DENS[I3(k, i, j)] + dtrk * (-J33G * (MZ[k - 1] - MZ[k - 2]) * RCDZ[k - 1] / 1.0 + w.Sr[I3(k, i, j)]);
            DN[KS - 1] = DENS[I3(KS, i, j)] + dtrk * (-J33G * MZ[KS - 1] * RCDZ[KS - 1] / 1.0 + w.Sr[I3(KS, i, j)]);
            DN[KE - 1] = DENS[I3(KE, i, j)] + dtrk * (J33G * MZ[KE - 2] * RCDZ[KE - 1] / 1.0 + w.Sr[I3(KE, i, j)]);
            for (int k = KS; k <= KE; ++k) PO[k - 1] = RHOT[I3(k, i, j)] / DENS[I3(k, i, j)];
            for (int k = KS + 1; k <= KE - 2; ++k)
                PT[k - 1] = (7.0 * (PO[k] + PO[k - 1]) - (PO[k + 1] + PO[k - 2])) / 12.0;
            PT[KS - 2] = 0.0;
            PT[KS - 1] = (PO[KS] + PO[KS - 1]) * 0.5;
            PT[KE - 2] = (PO[KE - 1] + PO[KE - 2]) * 0.5;
            PT[KE - 1] = 0.0;
            for (int k = KS + 1; k <= KE - 1; ++k)
                RN[k - 1] = RHOT[I3(k, i, j)] + dtrk * (-J33G * (MZ[k - 1] * PT[k - 1] - MZ[k - 2] * PT[k - 2]) * RCDZ[k - 1] / 1.0 + w.St[I3(k, i, j)]);
            RN[KS - 1] = RHOT[I3(KS, i, j)] + dtrk * (-J33G * MZ[KS - 1] * PT[KS - 1] * RCDZ[KS - 1] / 1.0 + w.St[I3(KS, i, j)]);
            RN[KE - 1] = RHOT[I3(KE, i, j)] + dtrk * (J33G * MZ[KE - 2] * PT[KE - 2] * RCDZ[KE - 1] / 1.0 + w.St[I3(KE, i, j)]);
            for (int k = KS; k <= KE; ++k) DP[k - 1] = w.DPRES[I3(k, i, j)] + RT2P[I3(k, i, j)] * (RN[k - 1] - RHOT[I3(k, i, j)]);
            for (int k = KS; k <= KE; ++k) {
                double lhs = (DN[k - 1] - DENS[I3(k, i, j)]) / dtrk;
                double rhs = -J33G * (MZ[k - 1] - MZ[k - 2]) * RCDZ[k - 1] / 1.0 + w.Sr[I3(k, i, j)];
                double err = fabs(lhs) < small ? rhs : (lhs - rhs) / lhs;
                if (fabs(err) > worst) worst = fabs(err);
            }
            for (int k = KS; k <= KE - 1; ++k) {
                double lhs = (MZ[k - 1] - MOMZ[I3(k, i, j)]) / dtrk;
                double rhs = -J33G * (DP[k] - DP[k - 1]) * RFDZ[k - 1] / 1.0
                             - GRAV * (DN[k] - REF_dens[I3(k + 1, i, j)] + DN[k - 1] - REF_dens[I3(k, i, j)]) * 0.5
                             + w.Sw[I3(k, i, j)];
                double err = fabs(lhs) < small ? rhs : (lhs - rhs) / lhs;
                if (fabs(err) > worst) worst = fabs(err);
            }
            for (int k = KS; k <= KE; ++k) {
                double lhs = (RN[k - 1] - RHOT[I3(k, i, j)]) / dtrk;
                double rhs = -J33G * (MZ[k - 1] * PT[k - 1] - MZ[k - 2] * PT[k - 2]) * RCDZ[k - 1] / 1.0 + w.St[I3(k, i, j)];
                double err = fabs(lhs) < small ? rhs : (lhs - rhs) / lhs;
                if (fabs(err) > worst) worst = fabs(err);
            }
        }
done:
    free(zero); free(one); free(jz); free(mapf); free(cor); free(wd); free(out); free(mflx); free(tflx); free(C);
    og_stage_work_free(&w);
    return worst;
}
