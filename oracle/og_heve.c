/*
 * Oracle restatement (test infrastructure) of one HEVE short-step stage, the
 * fully explicit alternative to HEVI:
 *   ATMOS_DYN_Tstep_short_fvm_heve : scale_atmos_dyn_tstep_short_fvm_heve.F90:109-1518
 * without the momentum / theta FCT branches (FLAG_FCT_MOMENTUM = FLAG_FCT_T =
 * .false.: :386-447, :716-810, :958-1057, :1207-1309, :1388-1515 are not
 * restated), one block (IBLOCK/JBLOCK default) and periodic boundaries
 * (IFS_OFF = JFS_OFF = 1). The metric factors (GSQRT, J13G, J23G, MAPF) are
 * kept as written. Line numbers below refer to the HEVE file. The flux
 * routines are those of og_flux.c, shared with HEVI.
 */
#include "og_internal.h"

/* F2H of the HEVE module (tstep_short_fvm_heve.F90:51): idx selects the GSQRT slice */
#define F2He(k, p, idx) (CDZ[(k) + (p) - 2] * GSQRT[I3((k) + (p) - 1, i, j) + ((size_t)(idx) - 1) * N3] /     \
                         (CDZ[(k) - 1] * GSQRT[I3(k, i, j) + ((size_t)(idx) - 1) * N3]                        \
                          + CDZ[(k)] * GSQRT[I3((k) + 1, i, j) + ((size_t)(idx) - 1) * N3]))
#define GS(k, i, j, idx) GSQRT[I3(k, i, j) + ((size_t)(idx) - 1) * N3]
#define J13(k, i, j, idx) J13G[I3(k, i, j) + ((size_t)(idx) - 1) * N3]
#define J23(k, i, j, idx) J23G[I3(k, i, j) + ((size_t)(idx) - 1) * N3]
#define MAPFv(i, j, a, b) MAPF[I2(i, j) + (size_t)IA * (size_t)JA * ((size_t)((a) - 1) + 2 * (size_t)((b) - 1))]
#define NDv(k, i, j, v, dir) num_diff[I3(k, i, j) + N3 * (size_t)(((v) - 1) + 5 * ((dir) - 1))]
#define COR(i, j) CORIOLI[I2(i, j)]

int og_heve_stage(
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
    OG_DIMS(d);
    const double GRAV = OG_GRAV;
    const int IFS_OFF = 1, JFS_OFF = 1; /* BND_W = BND_S = .false. (periodic) */
    const int IIS = IS, IIE = IE, JJS = JS, JJE = JE;
    const og_blk blk = {IIS, IIE, JJS, JJE};
    double *POTT = w->POTT, *DPRES = w->DPRES, *qflx_J13 = w->qflx_J13, *qflx_J23 = w->qflx_J23;
    double *qZ = w->qflx_hi, *qX = w->qflx_hi + N3, *qY = w->qflx_hi + 2 * N3;
    double *mZ = mflx_hi, *mX = mflx_hi + N3, *mY = mflx_hi + 2 * N3;
    double *tZ = tflx_hi, *tX = tflx_hi + N3, *tY = tflx_hi + 2 * N3;

    /* pressure, :360-373 */
#pragma omp parallel for collapse(2)
    for (int j = JJS - 2; j <= JJE + 2; ++j)
        for (int i = IIS - 2; i <= IIE + 2; ++i) {
            for (int k = KS; k <= KE; ++k)
                DPRES[I3(k, i, j)] = DPRES0[I3(k, i, j)] + RT2P[I3(k, i, j)] * (RHOT[I3(k, i, j)] - REF_rhot[I3(k, i, j)]);
            DPRES[I3(KS - 1, i, j)] = DPRES0[I3(KS - 1, i, j)] - DENS[I3(KS, i, j)] * (PHI[I3(KS - 1, i, j)] - PHI[I3(KS + 1, i, j)]);
            DPRES[I3(KE + 1, i, j)] = DPRES0[I3(KE + 1, i, j)] - DENS[I3(KE, i, j)] * (PHI[I3(KE + 1, i, j)] - PHI[I3(KE - 1, i, j)]);
        }
    /* potential temperature, :375-382 */
#pragma omp parallel for collapse(2)
    for (int j = JJS - d->JHALO; j <= JJE + d->JHALO; ++j)
        for (int i = IIS - d->IHALO; i <= IIE + d->IHALO; ++i)
            for (int k = KS; k <= KE; ++k) POTT[I3(k, i, j)] = RHOT[I3(k, i, j)] / DENS[I3(k, i, j)];

    /* mass fluxes, :460-510 */
#pragma omp parallel for collapse(2)
    for (int j = JJS; j <= JJE; ++j)
        for (int i = IIS; i <= IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k)
                mZ[I3(k, i, j)] = J33G * MOMZ[I3(k, i, j)] / (MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY))
                                  + J13(k, i, j, I_XYW) * 0.25
                                        * (MOMX[I3(k + 1, i, j)] + MOMX[I3(k + 1, i - 1, j)] + MOMX[I3(k, i, j)] + MOMX[I3(k, i - 1, j)])
                                        / MAPFv(i, j, 2, I_XY)
                                  + J23(k, i, j, I_XYW) * 0.25
                                        * (MOMY[I3(k + 1, i, j)] + MOMY[I3(k + 1, i, j - 1)] + MOMY[I3(k, i, j)] + MOMY[I3(k, i, j - 1)])
                                        / MAPFv(i, j, 1, I_XY)
                                  + GS(k, i, j, I_XYW) * NDv(k, i, j, I_DENS, ZDIR) / (MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY));
            mZ[I3(KS - 1, i, j)] = 0.0;
            mZ[I3(KE, i, j)] = 0.0;
        }
    {
        const int iee = IIE < IEH ? IIE : IEH;
#pragma omp parallel for collapse(2)
        for (int j = JJS; j <= JJE; ++j)
            for (int i = IIS - IFS_OFF; i <= iee; ++i)
                for (int k = KS; k <= KE; ++k)
                    mX[I3(k, i, j)] = GS(k, i, j, I_UYZ) / MAPFv(i, j, 2, I_UY) * (MOMX[I3(k, i, j)] + NDv(k, i, j, I_DENS, XDIR));
        const int jee = JJE < JEH ? JJE : JEH;
#pragma omp parallel for collapse(2)
        for (int j = JJS - JFS_OFF; j <= jee; ++j)
            for (int i = IIS; i <= IIE; ++i)
                for (int k = KS; k <= KE; ++k)
                    mY[I3(k, i, j)] = GS(k, i, j, I_XVZ) / MAPFv(i, j, 1, I_XV) * (MOMY[I3(k, i, j)] + NDv(k, i, j, I_DENS, YDIR));
    }

    /* density, :512-532 */
#pragma omp parallel for collapse(2)
    for (int j = JJS; j <= JJE; ++j)
        for (int i = IIS; i <= IIE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double advcv = -(mZ[I3(k, i, j)] - mZ[I3(k - 1, i, j)]) * RCDZ[k - 1];
                double advch = -(mX[I3(k, i, j)] - mX[I3(k, i - 1, j)]) * RCDX[i - 1]
                               - (mY[I3(k, i, j)] - mY[I3(k, i, j - 1)]) * RCDY[j - 1];
                DENS_RK[I3(k, i, j)] = DENS0[I3(k, i, j)]
                                       + dtrk * ((advcv + advch) * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY) / GS(k, i, j, I_XYZ)
                                                 + DENS_t[I3(k, i, j)]);
            }

    /* momentum (z): fluxes :586-620, pressure gradient :622-631, buoyancy :633-644, update :646-688 */
    og_fluxZ_XYW(d, scheme, qZ, MOMZ, MOMZ, DENS, G4(GSQRT, I_XYZ), J33G, ND(num_diff, I_MOMZ, ZDIR), blk);
    og_fluxJ13_XYW(d, scheme, qflx_J13, MOMX, MOMZ, DENS, G4(J13G, I_XYZ), MAPF4(MAPF, I_XY), blk);
    og_fluxJ23_XYW(d, scheme, qflx_J23, MOMY, MOMZ, DENS, G4(J23G, I_XYZ), MAPF4(MAPF, I_XY), blk);
    og_fluxX_XYW(d, scheme, qX, MOMX, MOMZ, DENS, G4(GSQRT, I_UYW), MAPF4(MAPF, I_UY), ND(num_diff, I_MOMZ, XDIR), CDZ, blk);
    og_fluxY_XYW(d, scheme, qY, MOMY, MOMZ, DENS, G4(GSQRT, I_XVW), MAPF4(MAPF, I_XV), ND(num_diff, I_MOMZ, YDIR), CDZ, blk);
#pragma omp parallel for collapse(2)
    for (int j = JJS; j <= JJE; ++j)
        for (int i = IIS; i <= IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double pgf = J33G * (DPRES[I3(k + 1, i, j)] - DPRES[I3(k, i, j)]) * RFDZ[k - 1];
                double buoy = GRAV * GS(k, i, j, I_XYW)
                              * (F2He(k, 1, I_XYZ) * (DENS[I3(k + 1, i, j)] - REF_dens[I3(k + 1, i, j)])
                                 + F2He(k, 2, I_XYZ) * (DENS[I3(k, i, j)] - REF_dens[I3(k, i, j)]));
                double advcv = -(qZ[I3(k, i, j)] - qZ[I3(k - 1, i, j)]
                                 + qflx_J13[I3(k, i, j)] - qflx_J13[I3(k - 1, i, j)]
                                 + qflx_J23[I3(k, i, j)] - qflx_J23[I3(k - 1, i, j)]) * RFDZ[k - 1];
                double advch = -((qX[I3(k, i, j)] - qX[I3(k, i - 1, j)]) * RCDX[i - 1]
                                 + (qY[I3(k, i, j)] - qY[I3(k, i, j - 1)]) * RCDY[j - 1])
                               * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY);
                double wdamp = -wdamp_coef[k - 1] * MOMZ0[I3(k, i, j)];
                double div = divdmp_coef / dtrk * FDZ[k - 1] * (DDIV[I3(k + 1, i, j)] - DDIV[I3(k, i, j)]);
                MOMZ_RK[I3(k, i, j)] = MOMZ0[I3(k, i, j)]
                                       + dtrk * ((advcv + advch - pgf - buoy) / GS(k, i, j, I_XYW) + wdamp + div
                                                 + MOMZ_t[I3(k, i, j)]);
            }
            MOMZ_RK[I3(KS - 1, i, j)] = 0.0;
            MOMZ_RK[I3(KE, i, j)] = 0.0;
        }

    /* momentum (x): fluxes :829-860, pressure gradient :862-879, Coriolis :881-897, update :899-922 */
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
                    double pgf = ((GS(k, i + 1, j, I_XYZ) * DPRES[I3(k, i + 1, j)]
                                   - GS(k, i, j, I_XYZ) * DPRES[I3(k, i, j)]) * RFDX[i - 1]
                                  + (J13(k, i, j, I_UYW)
                                         * 0.5 * (F2He(k, 1, I_UYZ) * (DPRES[I3(k + 1, i + 1, j)] + DPRES[I3(k + 1, i, j)])
                                                  + F2He(k, 2, I_UYZ) * (DPRES[I3(k, i + 1, j)] + DPRES[I3(k, i, j)]))
                                     - J13(k - 1, i, j, I_UYW)
                                         * 0.5 * (F2He(k, 1, I_UYZ) * (DPRES[I3(k, i + 1, j)] + DPRES[I3(k, i, j)])
                                                  + F2He(k, 2, I_UYZ) * (DPRES[I3(k - 1, i + 1, j)] + DPRES[I3(k - 1, i, j)])))
                                        * RCDZ[k - 1])
                                 * MAPFv(i, j, 1, I_UY);
                    double sumy = MOMY[I3(k, i, j)] + MOMY[I3(k, i, j - 1)] + MOMY[I3(k, i + 1, j)] + MOMY[I3(k, i + 1, j - 1)];
                    double cor = 0.125 * (COR(i + 1, j) + COR(i, j))
                                     * (MOMY[I3(k, i + 1, j)] + MOMY[I3(k, i, j)] + MOMY[I3(k, i + 1, j - 1)] + MOMY[I3(k, i, j - 1)])
                                 + 0.25 * MAPFv(i, j, 1, I_UY) * MAPFv(i, j, 2, I_UY)
                                     * sumy
                                     * (sumy * 0.25 * (1.0 / MAPFv(i + 1, j, 2, I_XY) - 1.0 / MAPFv(i, j, 2, I_XY)) * RFDX[i - 1]
                                        - MOMX[I3(k, i, j)] * (1.0 / MAPFv(i, j, 1, I_UV) - 1.0 / MAPFv(i, j - 1, 1, I_UV)) * RCDY[j - 1])
                                     * 2.0 / (DENS[I3(k, i + 1, j)] + DENS[I3(k, i, j)]);
                    double advcv = -(qZ[I3(k, i, j)] - qZ[I3(k - 1, i, j)]
                                     + qflx_J13[I3(k, i, j)] - qflx_J13[I3(k - 1, i, j)]
                                     + qflx_J23[I3(k, i, j)] - qflx_J23[I3(k - 1, i, j)]) * RCDZ[k - 1];
                    double advch = -((qX[I3(k, i, j)] - qX[I3(k, i - 1, j)]) * RFDX[i - 1]
                                     + (qY[I3(k, i, j)] - qY[I3(k, i, j - 1)]) * RCDY[j - 1])
                                   * MAPFv(i, j, 1, I_UY) * MAPFv(i, j, 2, I_UY);
                    double div = divdmp_coef / dtrk * FDX[i - 1] * (DDIV[I3(k, i + 1, j)] - DDIV[I3(k, i, j)]);
                    MOMX_RK[I3(k, i, j)] = MOMX0[I3(k, i, j)]
                                           + dtrk * ((advcv + advch - pgf) / GS(k, i, j, I_UYZ) + cor + div + MOMX_t[I3(k, i, j)]);
                }
    }

    /* momentum (y): fluxes :1076-1107, pressure gradient :1109-1126, Coriolis :1128-1144, update :1146-1170 */
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
                    double pgf = ((GS(k, i, j + 1, I_XYZ) * DPRES[I3(k, i, j + 1)]
                                   - GS(k, i, j, I_XYZ) * DPRES[I3(k, i, j)]) * RFDY[j - 1]
                                  + (J23(k, i, j, I_XVW)
                                         * 0.5 * (F2He(k, 1, I_XVZ) * (DPRES[I3(k + 1, i, j + 1)] + DPRES[I3(k + 1, i, j)])
                                                  + F2He(k, 2, I_XVZ) * (DPRES[I3(k, i, j + 1)] + DPRES[I3(k, i, j)]))
                                     - J23(k - 1, i, j, I_XVW)
                                         * 0.5 * (F2He(k - 1, 1, I_XVZ) * (DPRES[I3(k, i, j + 1)] + DPRES[I3(k, i, j)])
                                                  + F2He(k - 1, 2, I_XVZ) * (DPRES[I3(k - 1, i, j + 1)] + DPRES[I3(k - 1, i, j)])))
                                        * RCDZ[k - 1])
                                 * MAPFv(i, j, 2, I_XV);
                    double sumx = MOMX[I3(k, i, j)] + MOMX[I3(k, i - 1, j)] + MOMX[I3(k, i, j + 1)] + MOMX[I3(k, i - 1, j + 1)];
                    double cor = -0.125 * (COR(i, j + 1) + COR(i, j))
                                     * (MOMX[I3(k, i, j + 1)] + MOMX[I3(k, i, j)] + MOMX[I3(k, i - 1, j + 1)] + MOMX[I3(k, i - 1, j)])
                                 - 0.25 * MAPFv(i, j, 1, I_XV) * MAPFv(i, j, 2, I_XV)
                                     * sumx
                                     * (MOMY[I3(k, i, j)] * (1.0 / MAPFv(i, j, 2, I_UV) - 1.0 / MAPFv(i - 1, j, 2, I_UV)) * RCDX[i - 1]
                                        - 0.25 * (MOMX[I3(k, i, j)] + MOMX[I3(k, i - 1, j)] + MOMX[I3(k, i, j + 1)] + MOMX[I3(k, i - 1, j + 1)])
                                            * (1.0 / MAPFv(i, j + 1, 1, I_XY) - 1.0 / MAPFv(i, j, 1, I_XY)) * RFDY[j - 1])
                                     * 2.0 / (DENS[I3(k, i, j)] + DENS[I3(k, i, j + 1)]);
                    double advcv = -(qZ[I3(k, i, j)] - qZ[I3(k - 1, i, j)]
                                     + qflx_J13[I3(k, i, j)] - qflx_J13[I3(k - 1, i, j)]
                                     + qflx_J23[I3(k, i, j)] - qflx_J23[I3(k - 1, i, j)]) * RCDZ[k - 1];
                    double advch = -((qX[I3(k, i, j)] - qX[I3(k, i - 1, j)]) * RCDX[i - 1]
                                     + (qY[I3(k, i, j)] - qY[I3(k, i, j - 1)]) * RFDY[j - 1])
                                   * MAPFv(i, j, 1, I_XV) * MAPFv(i, j, 2, I_XV);
                    double div = divdmp_coef / dtrk * FDY[j - 1] * (DDIV[I3(k, i, j + 1)] - DDIV[I3(k, i, j)]);
                    MOMY_RK[I3(k, i, j)] = MOMY0[I3(k, i, j)]
                                           + dtrk * ((advcv + advch - pgf) / GS(k, i, j, I_XVZ) + cor + div + MOMY_t[I3(k, i, j)]);
                }
    }

    /* rho*theta: fluxes :1328-1348, update :1350-1371 */
    og_fluxZ_XYZ(d, scheme, tZ, mZ, POTT, G4(GSQRT, I_XYW), ND(num_diff, I_RHOT, ZDIR), blk);
    og_fluxX_XYZ(d, scheme, tX, mX, POTT, G4(GSQRT, I_UYZ), ND(num_diff, I_RHOT, XDIR), blk);
    og_fluxY_XYZ(d, scheme, tY, mY, POTT, G4(GSQRT, I_XVZ), ND(num_diff, I_RHOT, YDIR), blk);
#pragma omp parallel for collapse(2)
    for (int j = JJS; j <= JJE; ++j)
        for (int i = IIS; i <= IIE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double advcv = -(tZ[I3(k, i, j)] - tZ[I3(k - 1, i, j)]) * RCDZ[k - 1];
                double advch = -(tX[I3(k, i, j)] - tX[I3(k, i - 1, j)]) * RCDX[i - 1]
                               - (tY[I3(k, i, j)] - tY[I3(k, i, j - 1)]) * RCDY[j - 1];
                RHOT_RK[I3(k, i, j)] = RHOT0[I3(k, i, j)]
                                       + dtrk * ((advcv + advch) * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY) / GS(k, i, j, I_XYZ)
                                                 + RHOT_t[I3(k, i, j)]);
            }
    return 0;
}

int og_tstep_short_fvm_heve(
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
    int rc = og_heve_stage(d, scheme, &w, DENS_RK, MOMZ_RK, MOMX_RK, MOMY_RK, RHOT_RK, mflx_hi, tflx_hi,
                           DENS0, MOMZ0, MOMX0, MOMY0, RHOT0, DENS, MOMZ, MOMX, MOMY, RHOT,
                           DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, DPRES0, RT2P, CORIOLI,
                           num_diff, wdamp_coef, divdmp_coef, DDIV, CDZ, FDZ, FDX, FDY, RCDZ, RCDX, RCDY,
                           RFDZ, RFDX, RFDY, PHI, GSQRT, J13G, J23G, J33G, MAPF, REF_dens, REF_rhot, dtrk);
    og_stage_work_free(&w);
    return rc;
}
