/*
 * Oracle restatement of tracer advection and of the large step that drives
 * the short step:
 *   ATMOS_DYN_Tstep_tracer_fvm_heve : scale_atmos_dyn_tstep_tracer_fvm_heve.F90:72-240
 *   ATMOS_DYN_tinteg_tracer_rk3     : scale_atmos_dyn_tinteg_tracer_rk3.F90:92-210
 *   ATMOS_DYN_Tstep_large_fvm_heve  : scale_atmos_dyn_tstep_large_fvm_heve.F90:171-1130
 *   check_mass budget sum           : scale_atmos_dyn.F90:530-688
 */
#include "og_internal.h"
#ifdef _OPENMP
#include <omp.h>
#endif

int og_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int og_tstep_tracer_fvm_heve(
    const og_dims *d, int scheme,
    double *QTRCo, const double *QTRC, const double *QTRC0, const double *RHOQ_t,
    const double *DENS0, const double *DENS, const double *mflx_hi, const double *num_diff_q,
    const double *GSQRT, const double *MAPF_XY,
    const double *CDZ, const double *RCDZ, const double *RCDX, const double *RCDY,
    double dtl, int FLAG_FCT_TRACER, int FLAG_FCT_ALONG_STREAM)
{
    OG_DIMS(d);
    (void)CDZ;
    double *qflx_hi = og_alloc_undef(3 * N3), *qflx_lo = NULL, *qflx_anti = NULL;
    if (!qflx_hi) return -1;
    const og_blk blk = {IS, IE, JS, JE};
    const og_blk ext = {IS - 1, IE + 1, JS - 1, JE + 1};
    const double *mZ = mflx_hi, *mX = mflx_hi + N3, *mY = mflx_hi + 2 * N3;
    /* :127-147 */
    og_fluxZ_XYZ(d, scheme, qflx_hi, mZ, QTRC, G4(GSQRT, I_XYW), num_diff_q, blk);
    og_fluxX_XYZ(d, scheme, qflx_hi + N3, mX, QTRC, G4(GSQRT, I_UYZ), num_diff_q + N3, blk);
    og_fluxY_XYZ(d, scheme, qflx_hi + 2 * N3, mY, QTRC, G4(GSQRT, I_XVZ), num_diff_q + 2 * N3, blk);
#define M1(i, j) MAPF_XY[I2(i, j)]
#define M2(i, j) MAPF_XY[I2(i, j) + (size_t)IA * (size_t)JA]
#define GXYZ(k, i, j) GSQRT[I3(k, i, j)]
    const double *hZ = qflx_hi, *hX = qflx_hi + N3, *hY = qflx_hi + 2 * N3;
    if (FLAG_FCT_TRACER) {
        qflx_lo = og_alloc_undef(3 * N3);
        qflx_anti = og_alloc_undef(3 * N3);
        if (!qflx_lo || !qflx_anti) { free(qflx_hi); free(qflx_lo); free(qflx_anti); return -1; }
        /* :149-167 */
        og_fluxZ_XYZ_ud1(d, qflx_lo, mZ, QTRC0, ext);
        og_fluxX_XYZ_ud1(d, qflx_lo + N3, mX, QTRC0, ext);
        og_fluxY_XYZ_ud1(d, qflx_lo + 2 * N3, mY, QTRC0, ext);
        og_fct(d, qflx_anti, QTRC0, DENS0, DENS, qflx_hi, qflx_lo, mflx_hi, RCDZ, RCDX, RCDY,
               G4(GSQRT, I_XYZ), MAPF_XY, dtl, FLAG_FCT_ALONG_STREAM);
        const double *aZ = qflx_anti, *aX = qflx_anti + N3, *aY = qflx_anti + 2 * N3;
        /* :188-210 */
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i)
                for (int k = KS; k <= KE; ++k)
                    QTRCo[I3(k, i, j)] = (QTRC0[I3(k, i, j)] * DENS0[I3(k, i, j)]
                                          + dtl * (-((hZ[I3(k, i, j)] - aZ[I3(k, i, j)] - hZ[I3(k - 1, i, j)] + aZ[I3(k - 1, i, j)]) * RCDZ[k - 1]
                                                     + (hX[I3(k, i, j)] - aX[I3(k, i, j)] - hX[I3(k, i - 1, j)] + aX[I3(k, i - 1, j)]) * RCDX[i - 1]
                                                     + (hY[I3(k, i, j)] - aY[I3(k, i, j)] - hY[I3(k, i, j - 1)] + aY[I3(k, i, j - 1)]) * RCDY[j - 1])
                                                       * M1(i, j) * M2(i, j) / GXYZ(k, i, j)
                                                   + RHOQ_t[I3(k, i, j)]))
                                         / DENS[I3(k, i, j)];
    } else {
        /* :214-236 */
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i)
                for (int k = KS; k <= KE; ++k)
                    QTRCo[I3(k, i, j)] = (QTRC0[I3(k, i, j)] * DENS0[I3(k, i, j)]
                                          + dtl * (-((hZ[I3(k, i, j)] - hZ[I3(k - 1, i, j)]) * RCDZ[k - 1]
                                                     + (hX[I3(k, i, j)] - hX[I3(k, i - 1, j)]) * RCDX[i - 1]
                                                     + (hY[I3(k, i, j)] - hY[I3(k, i, j - 1)]) * RCDY[j - 1])
                                                       * M1(i, j) * M2(i, j) / GXYZ(k, i, j)
                                                   + RHOQ_t[I3(k, i, j)]))
                                         / DENS[I3(k, i, j)];
    }
#undef M1
#undef M2
#undef GXYZ
    free(qflx_hi); free(qflx_lo); free(qflx_anti);
    return 0;
}

int og_tinteg_tracer_rk3(
    const og_dims *d, int scheme,
    double *QTRC, const double *QTRC0, const double *RHOQ_t,
    const double *DENS0, const double *DENS, const double *mflx_hi, const double *num_diff_q,
    const double *GSQRT, const double *MAPF_XY,
    const double *CDZ, const double *RCDZ, const double *RCDX, const double *RCDY,
    double dtl, int FLAG_FCT_TRACER, int FLAG_FCT_ALONG_STREAM)
{
    OG_DIMS(d);
    double *DENS_RK = og_alloc_undef(N3), *RK1 = og_alloc_undef(N3), *RK2 = og_alloc_undef(N3);
    int rc = -1;
    if (!DENS_RK || !RK1 || !RK2) goto out;
    /* :140-147 */
    for (int j = JS - 1; j <= JE + 1; ++j)
        for (int i = IS - 1; i <= IE + 1; ++i)
            for (int k = KS; k <= KE; ++k)
                DENS_RK[I3(k, i, j)] = DENS0[I3(k, i, j)] + (DENS[I3(k, i, j)] - DENS0[I3(k, i, j)]) / 3.0;
    rc = og_tstep_tracer_fvm_heve(d, scheme, RK1, QTRC, QTRC0, RHOQ_t, DENS0, DENS_RK, mflx_hi, num_diff_q,
                                  GSQRT, MAPF_XY, CDZ, RCDZ, RCDX, RCDY, dtl / 3.0, 0, FLAG_FCT_ALONG_STREAM);
    if (rc) goto out;
    og_halo_periodic(d, RK1, 1);
    /* :168-175 */
    for (int j = JS - 1; j <= JE + 1; ++j)
        for (int i = IS - 1; i <= IE + 1; ++i)
            for (int k = KS; k <= KE; ++k)
                DENS_RK[I3(k, i, j)] = DENS0[I3(k, i, j)] + (DENS[I3(k, i, j)] - DENS0[I3(k, i, j)]) * 0.5;
    rc = og_tstep_tracer_fvm_heve(d, scheme, RK2, RK1, QTRC0, RHOQ_t, DENS0, DENS_RK, mflx_hi, num_diff_q,
                                  GSQRT, MAPF_XY, CDZ, RCDZ, RCDX, RCDY, dtl / 2.0, 0, FLAG_FCT_ALONG_STREAM);
    if (rc) goto out;
    og_halo_periodic(d, RK2, 1);
    /* :196-206; QTRCo may alias QTRC0 (the large step passes the same array) */
    rc = og_tstep_tracer_fvm_heve(d, scheme, QTRC, RK2, QTRC0, RHOQ_t, DENS0, DENS, mflx_hi, num_diff_q,
                                  GSQRT, MAPF_XY, CDZ, RCDZ, RCDX, RCDY, dtl, FLAG_FCT_TRACER, FLAG_FCT_ALONG_STREAM);
out:
    free(DENS_RK); free(RK1); free(RK2);
    return rc;
}

/* Large step, tstep_large_fvm_heve.F90:171-1130. Restated subset: periodic lateral
 * boundaries, DAMP_alpha = 0 (no nudging), ND_COEF_Q = 0, USE_AVERAGE off,
 * FLAG_TRACER_SPLIT_TEND off, EULER large-step integrator (Llast = .true., QTRC0 = QTRC). */
/* the registered short step of the large step (ATMOS_DYN_Tstep_short_regist): 0 HEVI, 1 HEVE */
static int og_short = 0;
void og_short_type(int type) { og_short = type; }
int og_short_type_get(void) { return og_short; }
/* the registered short integrator (ATMOS_DYN_TINTEG_SHORT_TYPE): 0 RK4, 1 RK3, 2 RK3WS2002 */
static int og_tinteg = 0;
void og_tinteg_short_type(int type) { og_tinteg = type; }
int og_tinteg_short_type_get(void) { return og_tinteg; }

int og_tstep_large(
    const og_dims *d, int scheme, int scheme_tracer,
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT, double *QTRC, int QA,
    double *mflx_hi, double *tflx_hi, double *num_diff,
    const double *DENS_tp, const double *MOMZ_tp, const double *MOMX_tp, const double *MOMY_tp,
    const double *RHOT_tp, const double *RHOQ_tp,
    const double *CORIOLI,
    const double *CDZ, const double *CDX, const double *CDY, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY, const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, double J33G, const double *MAPF,
    const double *AQ_R, const double *AQ_CV, const double *AQ_CP, const double *AQ_MASS,
    const double *REF_dens, const double *REF_pott, const double *REF_pres,
    double ND_COEF, int ND_ORDER, double ND_SFC_FACT, int ND_USE_RS,
    const double *wdamp_coef, double divdmp_coef,
    int FLAG_FCT_TRACER, int FLAG_FCT_ALONG_STREAM,
    double DTLS, double DTSS)
{
    OG_DIMS(d);
    const double P0 = OG_PRE00, Rdry = OG_RDRY, CPdry = OG_CPDRY, CVdry = OG_CPDRY - OG_RDRY;
    double dts = DTSS, dtl = DTLS;
    const int nstep = (int)ceil((dtl - OG_EPS) / dts);
    dts = dtl / nstep;

    double *DENS00 = og_alloc(N3), *DPRES0 = og_alloc_undef(N3), *RT2P = og_alloc_undef(N3), *REF_rhot = og_alloc_undef(N3);
    double *tend = og_alloc(5 * N3), *DDIV = og_alloc(N3), *mflx_av = (double *)calloc(3 * N3, sizeof(double));
    double *ndq = (double *)calloc(3 * N3, sizeof(double));
    int rc = -1;
    if (!DENS00 || !DPRES0 || !RT2P || !REF_rhot || !tend || !DDIV || !mflx_av || !ndq) goto out;
    memcpy(DENS00, DENS, N3 * sizeof(double));

    /* RT2P / DPRES0 / REF_rhot, :428-470 (moist form) */
#pragma omp parallel for collapse(2)
    for (int j = 1; j <= JA; ++j)
        for (int i = 1; i <= IA; ++i) {
            for (int k = KS; k <= KE; ++k) {
                double Rtot = 0.0, CVtot = 0.0, CPtot = 0.0, QDRY = 1.0;
                for (int iq = 0; iq < QA; ++iq) {
                    double q = QTRC[I3(k, i, j) + (size_t)iq * N3];
                    Rtot = Rtot + AQ_R[iq] * q;
                    CVtot = CVtot + AQ_CV[iq] * q;
                    CPtot = CPtot + AQ_CP[iq] * q;
                    QDRY = QDRY - q * AQ_MASS[iq];
                }
                Rtot = Rtot + Rdry * QDRY;
                CVtot = CVtot + CVdry * QDRY;
                CPtot = CPtot + CPdry * QDRY;
                double PRES = P0 * pow(Rtot * RHOT[I3(k, i, j)] / P0, CPtot / CVtot);
                RT2P[I3(k, i, j)] = CPtot / CVtot * PRES / RHOT[I3(k, i, j)];
                DPRES0[I3(k, i, j)] = PRES - REF_pres[I3(k, i, j)];
                REF_rhot[I3(k, i, j)] = RHOT[I3(k, i, j)];
            }
            DPRES0[I3(KS - 1, i, j)] = DPRES0[I3(KS + 1, i, j)] + (REF_pres[I3(KS + 1, i, j)] - REF_pres[I3(KS - 1, i, j)]);
            DPRES0[I3(KE + 1, i, j)] = DPRES0[I3(KE - 1, i, j)] + (REF_pres[I3(KE - 1, i, j)] - REF_pres[I3(KE + 1, i, j)]);
        }

    for (int step = 1; step <= nstep; ++step) {
        /* tendencies :606-839 with DAMP_alpha = 0: *_t = *_tp in the interior, zero in the k-halo */
        const double *tp[5] = {DENS_tp, MOMZ_tp, MOMX_tp, MOMY_tp, RHOT_tp};
        for (int v = 0; v < 5; ++v) {
            double *t = tend + (size_t)v * N3;
            const int kz = (v == 1) ? KE : KE + 1; /* MOMZ_t(KE:KA) = 0 */
            const int ke = (v == 1) ? KE - 1 : KE;
#pragma omp parallel for collapse(2)
            for (int j = JS; j <= JE; ++j)
                for (int i = IS; i <= IE; ++i) {
                    for (int k = KS; k <= ke; ++k) t[I3(k, i, j)] = tp[v][I3(k, i, j)];
                    for (int k = 1; k <= KS - 1; ++k) t[I3(k, i, j)] = 0.0;
                    for (int k = kz; k <= KA; ++k) t[I3(k, i, j)] = 0.0;
                }
            og_halo_periodic(d, t, 1);
        }
        /* numerical filter :847-858 */
        if (ND_COEF == 0.0) memset(num_diff, 0, 15 * N3 * sizeof(double));
        else if ((rc = og_numfilter_coef(d, num_diff, DENS, MOMZ, MOMX, MOMY, RHOT, CDZ, CDX, CDY, FDZ, FDX, FDY, dts,
                                         REF_dens, REF_pott, ND_COEF, ND_ORDER, ND_SFC_FACT, ND_USE_RS)))
            goto out;
        /* divergence :860-874 */
        if (divdmp_coef > 0.0)
            og_divergence(d, DDIV, MOMZ, MOMX, MOMY, GSQRT, J13G, J23G, J33G, MAPF, RCDZ, RCDX, RCDY, RFDZ, FDZ);
        else
            memset(DDIV, 0, N3 * sizeof(double));
        /* short step :880-894 */
        /* ATMOS_DYN_tinteg_short: the registered integrator and short step */
        if (og_tinteg)
            rc = og_tinteg_short_rk3(d, scheme, og_tinteg == 2, DENS, MOMZ, MOMX, MOMY, RHOT, mflx_hi, tflx_hi,
                                     tend, tend + N3, tend + 2 * N3, tend + 3 * N3, tend + 4 * N3,
                                     DPRES0, RT2P, CORIOLI, num_diff, wdamp_coef, divdmp_coef, DDIV,
                                     CDZ, FDZ, FDX, FDY, RCDZ, RCDX, RCDY, RFDZ, RFDX, RFDY,
                                     PHI, GSQRT, J13G, J23G, J33G, MAPF, REF_dens, REF_rhot, dts);
        else
            rc = (og_short ? og_tinteg_short_rk4_heve : og_tinteg_short_rk4)(
                d, scheme, DENS, MOMZ, MOMX, MOMY, RHOT, mflx_hi, tflx_hi,
                tend, tend + N3, tend + 2 * N3, tend + 3 * N3, tend + 4 * N3,
                DPRES0, RT2P, CORIOLI, num_diff, wdamp_coef, divdmp_coef, DDIV,
                CDZ, FDZ, FDX, FDY, RCDZ, RCDX, RCDY, RFDZ, RFDX, RFDY,
                PHI, GSQRT, J13G, J23G, J33G, MAPF, REF_dens, REF_rhot, dts);
        if (rc) goto out;
        /* vertical boundary fill :910-926 */
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i) {
                for (int k = 1; k <= KS - 1; ++k) {
                    DENS[I3(k, i, j)] = DENS[I3(KS, i, j)];
                    MOMZ[I3(k, i, j)] = 0.0;
                    MOMX[I3(k, i, j)] = MOMX[I3(KS, i, j)];
                    MOMY[I3(k, i, j)] = MOMY[I3(KS, i, j)];
                    RHOT[I3(k, i, j)] = RHOT[I3(KS, i, j)];
                }
                for (int k = KE + 1; k <= KA; ++k) {
                    DENS[I3(k, i, j)] = DENS[I3(KE, i, j)];
                    MOMZ[I3(k, i, j)] = 0.0;
                    MOMX[I3(k, i, j)] = MOMX[I3(KE, i, j)];
                    MOMY[I3(k, i, j)] = MOMY[I3(KE, i, j)];
                    RHOT[I3(k, i, j)] = RHOT[I3(KE, i, j)];
                }
            }
        og_halo_periodic(d, DENS, 1); og_halo_periodic(d, MOMZ, 1); og_halo_periodic(d, MOMX, 1);
        og_halo_periodic(d, MOMY, 1); og_halo_periodic(d, RHOT, 1);
        /* mass-flux accumulation for tracers :960-967 */
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i)
                for (int k = KS; k <= KE; ++k)
                    for (int n = 0; n < 3; ++n)
                        mflx_av[I3(k, i, j) + (size_t)n * N3] = mflx_av[I3(k, i, j) + (size_t)n * N3] + mflx_hi[I3(k, i, j) + (size_t)n * N3];
    }

    rc = 0;
    if (QA > 0) {
        /* :1012-1026 */
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i)
                for (int k = KS; k <= KE; ++k)
                    for (int n = 0; n < 3; ++n)
                        mflx_hi[I3(k, i, j) + (size_t)n * N3] = mflx_av[I3(k, i, j) + (size_t)n * N3] / nstep;
        og_halo_periodic(d, mflx_hi, 3);
        /* :1036-1120 (ND_COEF_Q = 0 -> num_diff_q = 0) */
        for (int iq = 0; iq < QA; ++iq) {
            double *q = QTRC + (size_t)iq * N3;
            if ((rc = og_tinteg_tracer_rk3(d, scheme_tracer, q, q, RHOQ_tp + (size_t)iq * N3, DENS00, DENS, mflx_hi, ndq,
                                           GSQRT, MAPF, CDZ, RCDZ, RCDX, RCDY, dtl, FLAG_FCT_TRACER, FLAG_FCT_ALONG_STREAM)))
                goto out;
            og_halo_periodic(d, q, 1);
        }
    }
out:
    free(DENS00); free(DPRES0); free(RT2P); free(REF_rhot); free(tend); free(DDIV); free(mflx_av); free(ndq);
    return rc;
}

/* sum over the interior of var*CDZ*CDX*CDY (check_mass, scale_atmos_dyn.F90:530-688),
 * accumulated per column then over columns in a fixed order */
double og_domain_sum(const og_dims *d, const double *var, const double *CDZ, const double *CDX, const double *CDY)
{
    OG_DIMS(d);
    double total = 0.0;
    for (int j = JS; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i)
            for (int k = KS; k <= KE; ++k) total += var[I3(k, i, j)] * CDZ[k - 1] * CDX[i - 1] * CDY[j - 1];
    return total;
}

/* Dry-air energy totals [J]: totals[0..3] = ENGT, ENGP, ENGK, ENGI over the
 * interior, each cell weighted by CDZ*CDX*CDY; per-cell values as
 * scale-rm/src/atmos/mod_atmos_vars.F90:2097-2171 (ENGP = DENS*GRAV*CZ,
 * ENGK = 0.5*DENS*(W**2+U**2+V**2), ENGI = DENS*QDRY*TEMP*CVdry with QDRY = 1,
 * ENGT = ENGP+ENGK+ENGI), the cell-centre velocities of
 * ATMOS_DIAGNOSTIC_CARTESC_get_vel on flat terrain
 * (scalelib/src/atmosphere/common/scale_atmos_diagnostic_cartesC.F90:88-135:
 * W(KS) = momws*0.5 with momws = MOMZ(KS), W(KE) = 0.5*MOMZ(KE-1)/DENS) and the
 * temperature of ATMOS_THERMODYN_rhot2temp_pres (scale_atmos_thermodyn.F90:791-792). */
void og_energy_sum(const og_dims *d, const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY,
                   const double *RHOT, const double *CZ, const double *CDZ, const double *CDX, const double *CDY,
                   double *totals)
{
    OG_DIMS(d);
    const double CVdry = OG_CPDRY - OG_RDRY;
    double tot[4] = {0.0, 0.0, 0.0, 0.0};
    for (int j = JS; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i) {
            double col[4] = {0.0, 0.0, 0.0, 0.0};
            for (int k = KS; k <= KE; ++k) {
                const double dn = DENS[I3(k, i, j)];
                double w;
                if (k == KS) w = MOMZ[I3(KS, i, j)] * 0.5;
                else if (k == KE) w = 0.5 * (MOMZ[I3(KE - 1, i, j)]) / dn;
                else w = 0.5 * (MOMZ[I3(k - 1, i, j)] + MOMZ[I3(k, i, j)]) / dn;
                const double u = 0.5 * (MOMX[I3(k, i - 1, j)] + MOMX[I3(k, i, j)]) / dn;
                const double v = 0.5 * (MOMY[I3(k, i, j - 1)] + MOMY[I3(k, i, j)]) / dn;
                const double pres = OG_PRE00 * pow(RHOT[I3(k, i, j)] * OG_RDRY / OG_PRE00, OG_CPDRY / CVdry);
                const double temp = pres / (dn * OG_RDRY);
                const double engp = dn * OG_GRAV * CZ[k - 1];
                const double engk = 0.5 * dn * (w * w + u * u + v * v);
                const double engi = dn * 1.0 * temp * CVdry;
                const double engt = engp + engk + engi;
                const double e[4] = {engt, engp, engk, engi};
                for (int q = 0; q < 4; ++q) col[q] += e[q] * CDZ[k - 1] * CDX[i - 1] * CDY[j - 1];
            }
            for (int q = 0; q < 4; ++q) tot[q] += col[q];
        }
    for (int q = 0; q < 4; ++q) totals[q] = tot[q];
}

