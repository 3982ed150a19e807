/*
 * CPU oracle for the HEVI short-step hot path of SCALE-RM (test infrastructure).
 *
 * This is a line-by-line FP64 restatement, in C99 + OpenMP, of the Fortran
 * reference routines named in each function's comment. It is the CHECKER for
 * the CUDA product path, never part of it: only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it.
 *
 * Pinning status: the reference ships no golden vectors for this path and no
 * Fortran compiler exists in the build image, so the restatement cannot be run
 * against the Fortran build. It is pinned only by the reference's own property
 * tests (scalelib/test/unit/test_atmos_dyn.f90: constancy, conservation,
 * consistency with continuity, FCT min/max, no UNDEF leak) and the DEBUG solver
 * residual check (scale_atmos_dyn_tstep_short_fvm_hevi.F90:1131-1271), all
 * re-run in tests/. Bit-level agreement with the Fortran build is therefore
 * "parity unpinned".
 *
 * Conventions
 *   - Arrays are Fortran column-major (KA,IA,JA) with k fastest; all indices in
 *     the code below are the reference's 1-based indices.
 *   - Arithmetic follows the Fortran evaluation order (left to right inside a
 *     precedence level, parentheses honoured) and is compiled with
 *     -ffp-contract=off, matching the reference's GNU build flags
 *     (sysdep/Makedef.Linux64-gnu-ompi: -O3, no -ffast-math, no FMA target).
 *   - Fortran SIGN(a,b) is copysign(|a|,b); MAX/MIN are plain comparisons.
 */
#ifndef SCALE_ORACLE_H
#define SCALE_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* grid index set, scale_atmos_grid_cartesC_index.F90:256-268 */
typedef struct {
    int KA, IA, JA;
    int KS, KE, IS, IE, JS, JE;
    int KMAX, IMAX, JMAX;
    int IHALO, JHALO;
    int IEH, JEH;
} og_dims;

/* flux scheme ids (scale_atmos_dyn_fvm_flux.F90:276 setup by name) */
enum { OG_UD3 = 1, OG_CD4 = 2, OG_KOREN = 3, OG_CD2 = 4, OG_UD5 = 5, OG_CD6 = 6 }; /* OG_KOREN: UD3KOREN1993;
 * OG_UD5 and OG_CD6 need IHALO = JHALO = 3 */

/* physical constants, scale_const.F90 */
#define OG_GRAV   9.80665
#define OG_RDRY   287.04
#define OG_CPDRY  1004.64
#define OG_PRE00  100000.0
#define OG_EPS    2.220446049250313080847263336181640625e-16

/* ---- one HEVI stage: scale_atmos_dyn_tstep_short_fvm_hevi.F90:128-1089 ---- */
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
    double dtrk);

/* ---- RK4 short integrator: scale_atmos_dyn_tinteg_short_rk4.F90:199-650 ---- */
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
    double dt);

/* ---- one HEVE stage (fully explicit; no momentum/theta FCT):
 *      scale_atmos_dyn_tstep_short_fvm_heve.F90:109-1518 ---- */
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
    double dtrk);

/* ---- the RK4 short integrator with the HEVE stage ---- */
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
    double dt);

/* ---- RK3 short integrator: scale_atmos_dyn_tinteg_short_rk3.F90:188-576, with the
 *      registered short step; ws2002 = 1 for RK3WS2002, 0 for RK3 (Heun) ---- */
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
    double dt);

/* ---- the short step and short integrator that og_tstep_large and og_tinteg_short_rk3 run
 *      (ATMOS_DYN_Tstep_short_regist, ATMOS_DYN_TINTEG_SHORT_TYPE): short 0 HEVI (default),
 *      1 HEVE; integrator 0 RK4 (default), 1 RK3, 2 RK3WS2002 ---- */
void og_short_type(int type);
void og_tinteg_short_type(int type);

/* ---- periodic 8-neighbour halo fill, scale_comm_cartesC.F90 (COMM_vars8 on a periodic 1x1 grid) ---- */
void og_halo_periodic(const og_dims *d, double *var, int nfields);
/* ---- a decomposed domain (the tests' ranks): while fn is set, every halo fill of the
 *      oracle, og_halo_periodic included, calls fn(var, nfields, user) instead, with
 *      nfields consecutive (KA,IA,JA) arrays at var; NULL restores the periodic fill ---- */
typedef int (*og_halo_fn)(double *var, int nfields, void *user);
void og_set_halo_exchange(og_halo_fn fn, void *user);

/* ---- numerical filter: scale_atmos_dyn_common.F90:385-985 (ND_ORDER=1 path) + filter_setup :100-330 ---- */
int og_numfilter_coef(
    const og_dims *d, double *num_diff,
    const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY, const double *RHOT,
    const double *CDZ, const double *CDX, const double *CDY,
    const double *FDZ, const double *FDX, const double *FDY, double DT,
    const double *REF_dens, const double *REF_pott,
    double ND_COEF, int ND_ORDER, double ND_SFC_FACT, int ND_USE_RS);

/* ---- 3-D divergence: scale_atmos_dyn_common.F90:1437-1515 ---- */
void og_divergence(
    const og_dims *d, double *DDIV,
    const double *MOMZ, const double *MOMX, const double *MOMY,
    const double *GSQRT, const double *J13G, const double *J23G, double J33G, const double *MAPF,
    const double *RCDZ, const double *RCDX, const double *RCDY, const double *RFDZ, const double *FDZ);

/* ---- tracer step: scale_atmos_dyn_tstep_tracer_fvm_heve.F90:72-240 ---- */
int og_tstep_tracer_fvm_heve(
    const og_dims *d, int scheme,
    double *QTRCo, const double *QTRC, const double *QTRC0, const double *RHOQ_t,
    const double *DENS0, const double *DENS, const double *mflx_hi, const double *num_diff_q,
    const double *GSQRT, const double *MAPF_XY,
    const double *CDZ, const double *RCDZ, const double *RCDX, const double *RCDY,
    double dtl, int FLAG_FCT_TRACER, int FLAG_FCT_ALONG_STREAM);

/* ---- tracer RK3 (Wicker-Skamarock 2002): scale_atmos_dyn_tinteg_tracer_rk3.F90:92-210 ---- */
int og_tinteg_tracer_rk3(
    const og_dims *d, int scheme,
    double *QTRC, const double *QTRC0, const double *RHOQ_t,
    const double *DENS0, const double *DENS, const double *mflx_hi, const double *num_diff_q,
    const double *GSQRT, const double *MAPF_XY,
    const double *CDZ, const double *RCDZ, const double *RCDX, const double *RCDY,
    double dtl, int FLAG_FCT_TRACER, int FLAG_FCT_ALONG_STREAM);

/* ---- large step around the short step: scale_atmos_dyn_tstep_large_fvm_heve.F90:171-1130
 * (periodic, no lateral damping, USE_AVERAGE off, ND_COEF_Q = 0, FLAG_TRACER_SPLIT_TEND off).
 * QTRC(KA,IA,JA,QA) is advanced in place; AQ_* describe the tracers. */
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
    double DTLS, double DTSS);

/* ---- DEBUG residual check of the implicit solve: scale_atmos_dyn_tstep_short_fvm_hevi.F90:1131-1271.
 * Runs one stage and returns the maximum relative residual over DENS, MOMZ and RHOT. */
double og_hevi_max_residual(
    const og_dims *d, int scheme,
    const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY, const double *RHOT,
    const double *DPRES0, const double *RT2P, const double *num_diff,
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY,
    const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *REF_dens, const double *REF_rhot, double dtrk);

/* ---- FP64 domain budget: sum over the interior of field*CDZ*CDX*CDY (check_mass, scale_atmos_dyn.F90:530-688) ---- */
double og_domain_sum(const og_dims *d, const double *var, const double *CDZ, const double *CDX, const double *CDY);
/* ---- FP64 energy budget of dry air: totals ENGT, ENGP, ENGK, ENGI (mod_atmos_vars.F90:2097-2171) ---- */
void og_energy_sum(const og_dims *d, const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY,
                   const double *RHOT, const double *CZ, const double *CDZ, const double *CDX, const double *CDY,
                   double *totals);

int og_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
