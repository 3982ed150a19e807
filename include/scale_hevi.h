/*
 * scale_hevi.h -- C-ABI of the B200 implementation of SCALE-RM's HEVI short
 * time step (libscale_hevi.so).
 *
 * Every entry point replaces one procedure of the reference dynamical core
 * (hisashiyashiro/scale, SCALE 5.3.6) and keeps its argument list and order so
 * that scale-rm's Fortran driver can bind it with ISO_C_BINDING.
 * Conventions follow what gfortran passes for those dummies:
 *   - arrays are double* in Fortran column-major order with k fastest:
 *     a (KA,IA,JA) field is element (k,i,j) at (k-1) + KA*((i-1) + IA*(j-1));
 *   - intent(in) scalars are passed by reference (const double*, const int*);
 *   - LOGICAL is a 4-byte int (0 = .false., nonzero = .true.).
 * Entry points without the _dev suffix take HOST arrays: the library copies the
 * inputs to the GPU, runs, and copies the outputs back before returning.
 * Entry points with the _dev suffix take DEVICE pointers for every 2-D/3-D
 * array and host pointers for the 1-D grid vectors and scalars; they enqueue
 * work on the library's stream and return without synchronising.
 *
 * Every entry returns 0 on success or one of the SCALE_HEVI_ERR_* codes below;
 * scale_hevi_last_error() then describes the failure. A Fortran shim maps a
 * nonzero status to PRC_abort, as the reference aborts on errors.
 *
 * Supported configuration (checked, otherwise SCALE_HEVI_ERR_UNSUPPORTED):
 * periodic lateral boundaries (BND_* = .false.); terrain-following metrics
 * (GSQRT, J13G, J23G, MAPF not those of flat terrain, classified once per set
 * of metric arrays) in the FP64 HEVI and HEVE stage, RK4, RK3, large-step,
 * tracer and divergence entries of one domain, where they select the
 * general-metric stage (PHI is read) or the metric forms of the tracer and
 * divergence kernels;
 * flat terrain (GSQRT = 1, J13G = J23G = 0, MAPF = 1) in every other entry; the default
 * IBLOCK/JBLOCK (whole domain), flux schemes "UD3", "CD4", "CD2",
 * "UD3KOREN1993", "UD5" and "CD6", ND_ORDER >= 1 (above 1 on the FP64 path of
 * one domain with KMAX >= 6), 4 <= KMAX <= 256 (5 for UD5/CD6), KHALO = 2 and IHALO = JHALO
 * = 2 or 3 (3 for UD5/CD6). No additional prognostic variables (VA = 0).
 *
 * Concurrency: one library state per process (like the reference's module
 * variables); calls are not re-entrant and must come from one host thread.
 */
#ifndef SCALE_HEVI_H
#define SCALE_HEVI_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SCALE_HEVI_OK                0
#define SCALE_HEVI_ERR_ARG           1  /* inconsistent sizes or invalid argument       */
#define SCALE_HEVI_ERR_NOT_SETUP     2  /* scale_hevi_setup() was not called            */
#define SCALE_HEVI_ERR_CUDA          3  /* CUDA runtime error                            */
#define SCALE_HEVI_ERR_NONFINITE     4  /* a prognostic output became NaN or Inf        */
#define SCALE_HEVI_ERR_UNSUPPORTED   5  /* option outside the supported configuration   */
#define SCALE_HEVI_ERR_ALLOC         6  /* device or pinned host allocation failed      */

/* Index set of the local domain, the module variables of
 * scalelib/src/atmosphere/grid/scale_atmos_grid_cartesC_index.F90:40-45,256-279 */
typedef struct scale_hevi_index {
    int KA, IA, JA;
    int KS, KE, IS, IE, JS, JE;
    int KMAX, IMAX, JMAX;
    int KHALO, IHALO, JHALO;
    int IBLOCK, JBLOCK;
} scale_hevi_index;

/* ---------------------------------------------------------------------------
 * Library state
 * ------------------------------------------------------------------------- */

/* Setup of the index set and the flux schemes; replaces the module state set
 * by ATMOS_GRID_CARTESC_INDEX_setup and ATMOS_DYN_FVM_flux_setup
 * (scalelib/src/atmos-rm/dynamics/scale_atmos_dyn_fvm_flux.F90:276) for the
 * HEVI short step (ATMOS_DYN_Tstep_short_fvm_hevi_setup,
 * scale_atmos_dyn_tstep_short_fvm_hevi.F90:118). flux_type and
 * flux_tracer_type are the ATMOS_DYN_FVM_FLUX_TYPE / _TRACER_TYPE names
 * ("UD3", "CD4", "CD2", "UD3KOREN1993", "UD5" or "CD6":
 * scale_atmos_dyn_fvm_flux_ud3.F90, _cd4.F90, _cd2.F90, _ud3Koren1993.F90,
 * _ud5.F90, _cd6.F90; UD3KOREN1993 is the reference's default tracer flux;
 * UD5 and CD6 need IHALO = JHALO = 3, as scale_atmos_dyn_fvm_flux.F90:742-749
 * requires). device is the CUDA ordinal to use. */
int scale_hevi_setup(const scale_hevi_index *idx, const char *flux_type, const char *flux_tracer_type, int device);
/* Frees every device buffer and the stream. */
int scale_hevi_finalize(void);
/* Text of the last error (empty when none). */
const char *scale_hevi_last_error(void);
/* The cudaStream_t the _dev entries enqueue on (as void*). It is a blocking
 * stream: work on the legacy default stream is ordered with it both ways, so
 * arrays produced or consumed there need no further synchronisation; a caller
 * on another stream orders its work with events. */
void *scale_hevi_stream(void);
/* Waits for the stream and returns SCALE_HEVI_ERR_NONFINITE if any kernel
 * since the last check saw a non-finite prognostic value (the device-side
 * counterpart of the reference's UNDEF/NaN checks, scale_debug.F90:53-76). */
int scale_hevi_check(void);
/* Number of this library's kernels launched since setup (for profiling). */
long long scale_hevi_kernel_launches(void);
/* Bytes copied host->device and device->host by the host-array entries since
 * setup (the staging copies of inputs and results). No counterpart in the
 * reference; used to report the transfer volume of an end-to-end call. */
int scale_hevi_transfer_bytes(long long *h2d_bytes, long long *d2h_bytes);

/* ---------------------------------------------------------------------------
 * One HEVI stage. Replaces ATMOS_DYN_Tstep_short_fvm_hevi
 * (scalelib/src/atmos-rm/dynamics/scale_atmos_dyn_tstep_short_fvm_hevi.F90:128-1089),
 * the target of the ATMOS_DYN_Tstep_short procedure pointer
 * (scale_atmos_dyn_tstep_short.F90:38-128,134). Same dummy arguments, same
 * order. Outputs are written on the cells the reference writes; other cells of
 * the output arrays keep their contents. PROG_RK/PROG0/PROG (VA = 0) and
 * FLAG_FCT_* (unused by HEVI) are accepted and ignored; `last` only gates the
 * reference's HIST_TEND output and is ignored.
 * ------------------------------------------------------------------------- */
#define SCALE_HEVI_TSTEP_SHORT_ARGS                                                                         \
    double *DENS_RK, double *MOMZ_RK, double *MOMX_RK, double *MOMY_RK, double *RHOT_RK,                       \
    double *PROG_RK, double *mflx_hi, double *tflx_hi,                                                         \
    const double *DENS0, const double *MOMZ0, const double *MOMX0, const double *MOMY0, const double *RHOT0,   \
    const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY, const double *RHOT,        \
    const double *DENS_t, const double *MOMZ_t, const double *MOMX_t, const double *MOMY_t, const double *RHOT_t, \
    const double *PROG0, const double *PROG,                                                                   \
    const double *DPRES0, const double *RT2P, const double *CORIOLI,                                           \
    const double *num_diff, const double *wdamp_coef, const double *divdmp_coef, const double *DDIV,           \
    const int *FLAG_FCT_MOMENTUM, const int *FLAG_FCT_T, const int *FLAG_FCT_ALONG_STREAM,                     \
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,                                \
    const double *RCDZ, const double *RCDX, const double *RCDY,                                                \
    const double *RFDZ, const double *RFDX, const double *RFDY,                                                \
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, const double *J33G,        \
    const double *MAPF, const double *REF_dens, const double *REF_rhot,                                        \
    const int *BND_W, const int *BND_E, const int *BND_S, const int *BND_N,                                    \
    const double *dtrk, const int *last

int ATMOS_DYN_Tstep_short_fvm_hevi_b200(SCALE_HEVI_TSTEP_SHORT_ARGS);
int ATMOS_DYN_Tstep_short_fvm_hevi_b200_dev(SCALE_HEVI_TSTEP_SHORT_ARGS);

/* ---------------------------------------------------------------------------
 * One HEVE stage, the fully explicit short step. Replaces
 * ATMOS_DYN_Tstep_short_fvm_heve (scale_atmos_dyn_tstep_short_fvm_heve.F90:109-1518),
 * the other target of ATMOS_DYN_Tstep_short. Same arguments as the HEVI
 * stage. FLAG_FCT_MOMENTUM and FLAG_FCT_T must be .false. (the momentum and
 * theta FCT branches, :386-447, :716-1309, :1388-1515, are not provided);
 * FP64 only. Terrain-following metrics select the general-metric HEVE stage.
 * ------------------------------------------------------------------------- */
int ATMOS_DYN_Tstep_short_fvm_heve_b200(SCALE_HEVI_TSTEP_SHORT_ARGS);
int ATMOS_DYN_Tstep_short_fvm_heve_b200_dev(SCALE_HEVI_TSTEP_SHORT_ARGS);

/* Registers the short step that the RK4 entries and the large step run, as
 * ATMOS_DYN_Tstep_short_regist does for ATMOS_DYN_TSTEP_SHORT_TYPE
 * (scale_atmos_dyn_tstep_short.F90:153-215): "HEVI" (the default after setup)
 * or "HEVE". The mixed-precision and differentiated entries take HEVI only. */
int scale_hevi_short_type(const char *type);

/* ---------------------------------------------------------------------------
 * One short time step with the four-stage Runge-Kutta integrator. Replaces
 * ATMOS_DYN_tinteg_short_rk4 (scale_atmos_dyn_tinteg_short_rk4.F90:199-650),
 * target of ATMOS_DYN_Tinteg_short (scale_atmos_dyn_tinteg_short.F90:32-108).
 * Same arguments in the same order (the reference names positions 21 and 48-49
 * CVtot, REF_pres and REF_dens although the large step passes RT2P, REF_dens
 * and REF_rhot; they are named here for what they receive). DENS..RHOT are
 * updated in place on the interior; mflx_hi and tflx_hi receive the RK4
 * averaged fluxes. The RK stage buffers stay on the device and the halo
 * exchange between stages is done on the device.
 * ------------------------------------------------------------------------- */
#define SCALE_HEVI_TINTEG_SHORT_ARGS                                                                           \
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT, double *PROG,                        \
    double *mflx_hi, double *tflx_hi,                                                                          \
    const double *DENS_t, const double *MOMZ_t, const double *MOMX_t, const double *MOMY_t, const double *RHOT_t, \
    const double *DPRES0, const double *RT2P, const double *CORIOLI,                                           \
    const double *num_diff, const double *wdamp_coef, const double *divdmp_coef, const double *DDIV,           \
    const int *FLAG_FCT_MOMENTUM, const int *FLAG_FCT_T, const int *FLAG_FCT_ALONG_STREAM,                     \
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,                                \
    const double *RCDZ, const double *RCDX, const double *RCDY,                                                \
    const double *RFDZ, const double *RFDX, const double *RFDY,                                                \
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, const double *J33G,        \
    const double *MAPF, const double *REF_dens, const double *REF_rhot,                                        \
    const int *BND_W, const int *BND_E, const int *BND_S, const int *BND_N,                                    \
    const double *dt

int ATMOS_DYN_Tinteg_short_rk4_b200(SCALE_HEVI_TINTEG_SHORT_ARGS);
int ATMOS_DYN_Tinteg_short_rk4_b200_dev(SCALE_HEVI_TINTEG_SHORT_ARGS);

/* ---------------------------------------------------------------------------
 * One short time step with a three-stage Runge-Kutta integrator. Replaces
 * ATMOS_DYN_tinteg_short_rk3 (scale_atmos_dyn_tinteg_short_rk3.F90:188-576),
 * the other target of ATMOS_DYN_Tinteg_short. Same arguments as the RK4 step.
 * The variant is the registered one (scale_hevi_tinteg_short_type), as the
 * reference fixes it in ATMOS_DYN_Tinteg_short_rk3_setup (:89-184): "RK3",
 * Heun's method, stages at dt/3, 2dt/3, dt and the state
 * (r1*3 + r3*3 - phi_n*2)/4, fluxes (F1 + F3*3)/4; or "RK3WS2002" (Wicker and
 * Skamarock 2002), stages at dt/3, dt/2, dt and the third stage kept. With RK4
 * registered both entries return SCALE_HEVI_ERR_UNSUPPORTED.
 * ------------------------------------------------------------------------- */
int ATMOS_DYN_Tinteg_short_rk3_b200(SCALE_HEVI_TINTEG_SHORT_ARGS);
int ATMOS_DYN_Tinteg_short_rk3_b200_dev(SCALE_HEVI_TINTEG_SHORT_ARGS);

/* ---------------------------------------------------------------------------
 * Halo exchange hook for a domain decomposed over ranks. Replaces the
 * periodic self-exchange of COMM_vars8/COMM_wait
 * (scale_comm_cartesC.F90:1600-2043, 2787-3023) that the library does on one
 * rank. When fn is set, every lateral halo fill of the short step and the
 * large step (the RK stage buffers, the state, num_diff, mflx_hi, the
 * tracers and their RK stages, the FCT limiter's R+/R-
 * (scale_atmos_dyn_common.F90:2558-2561) and the work arrays of the filter at
 * ND_ORDER > 1 (:1557-1563)) calls fn instead: fn receives the device
 * addresses of nfields (KA,IA,JA) fields with elements of elem_bytes (8 or 4)
 * and must have filled their lateral halos (IHALO columns, JHALO rows,
 * corners included) when it returns 0 (a nonzero return is reported as an
 * error). The library's stream is idle during the call. NULL restores the
 * periodic fill. One domain only; the persistent short step does not take it.
 * ------------------------------------------------------------------------- */
typedef int (*scale_hevi_halo_fn)(void *const *fields, int nfields, int elem_bytes, void *user);
int scale_hevi_set_halo_exchange(scale_hevi_halo_fn fn, void *user);

/* Registers the short integrator of the large step and the RK3 entries, as
 * ATMOS_DYN_Tinteg_short_setup does for ATMOS_DYN_TINTEG_SHORT_TYPE
 * (scale_atmos_dyn_tinteg_short.F90:146-159): "RK4" (the default after
 * setup), "RK3" or "RK3WS2002". The differentiated entries take RK4 only. */
int scale_hevi_tinteg_short_type(const char *type);

/* ---------------------------------------------------------------------------
 * Mixed-precision RK4 short step (device arrays). No counterpart in the
 * reference, which is either all FP64 or, built with -DSINGLE, all FP32. Flux
 * and divergence arithmetic runs in FP32. The state (DENS..RHOT), DPRES0, RT2P,
 * REF_dens, REF_rhot, the deviations from the base state, the right-hand side
 * and the tridiagonal solve stay FP64. The flux-like arrays are FP32 buffers:
 * mflx_hi, tflx_hi, the tendencies DENS_t..RHOT_t, num_diff and DDIV. The
 * arguments are otherwise those of ATMOS_DYN_Tinteg_short_rk4_b200_dev.
 * ------------------------------------------------------------------------- */
#define SCALE_HEVI_TINTEG_SHORT_MIXED_ARGS                                                                     \
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT, double *PROG,                        \
    float *mflx_hi, float *tflx_hi,                                                                            \
    const float *DENS_t, const float *MOMZ_t, const float *MOMX_t, const float *MOMY_t, const float *RHOT_t,   \
    const double *DPRES0, const double *RT2P, const double *CORIOLI,                                           \
    const float *num_diff, const double *wdamp_coef, const double *divdmp_coef, const float *DDIV,             \
    const int *FLAG_FCT_MOMENTUM, const int *FLAG_FCT_T, const int *FLAG_FCT_ALONG_STREAM,                     \
    const double *CDZ, const double *FDZ, const double *FDX, const double *FDY,                                \
    const double *RCDZ, const double *RCDX, const double *RCDY,                                                \
    const double *RFDZ, const double *RFDX, const double *RFDY,                                                \
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, const double *J33G,        \
    const double *MAPF, const double *REF_dens, const double *REF_rhot,                                        \
    const int *BND_W, const int *BND_E, const int *BND_S, const int *BND_N,                                    \
    const double *dt

int ATMOS_DYN_Tinteg_short_rk4_b200_mixed_dev(SCALE_HEVI_TINTEG_SHORT_MIXED_ARGS);

/* Numerical filter of the mixed-precision path: as
 * ATMOS_DYN_numfilter_coef_b200_dev, with num_diff an FP32 device array. */
#define SCALE_HEVI_NUMFILTER_MIXED_ARGS                                                                        \
    float *num_diff,                                                                                           \
    const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY, const double *RHOT,        \
    const double *CDZ, const double *CDX, const double *CDY, const double *FDZ, const double *FDX,             \
    const double *FDY, const double *DT, const double *REF_dens, const double *REF_pott,                       \
    const double *ND_COEF, const int *ND_ORDER, const double *ND_SFC_FACT, const int *ND_USE_RS

int ATMOS_DYN_numfilter_coef_b200_mixed_dev(SCALE_HEVI_NUMFILTER_MIXED_ARGS);

/* ---------------------------------------------------------------------------
 * Numerical filter coefficients. Replaces ATMOS_DYN_numfilter_coef
 * (scalelib/src/atmos-rm/dynamics/scale_atmos_dyn_common.F90:385-985),
 * including the halo exchange of the fifteen num_diff components.
 * num_diff is (KA,IA,JA,5,3). ND_ORDER 1..8; above 1 the differences are
 * iterated with calc_diff4 (scale_atmos_dyn_common.F90:1518-1573, 1810-1918).
 * ------------------------------------------------------------------------- */
#define SCALE_HEVI_NUMFILTER_ARGS                                                                              \
    double *num_diff,                                                                                          \
    const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY, const double *RHOT,        \
    const double *CDZ, const double *CDX, const double *CDY, const double *FDZ, const double *FDX,             \
    const double *FDY, const double *DT, const double *REF_dens, const double *REF_pott,                       \
    const double *ND_COEF, const int *ND_ORDER, const double *ND_SFC_FACT, const int *ND_USE_RS

int ATMOS_DYN_numfilter_coef_b200(SCALE_HEVI_NUMFILTER_ARGS);
int ATMOS_DYN_numfilter_coef_b200_dev(SCALE_HEVI_NUMFILTER_ARGS);

/* ---------------------------------------------------------------------------
 * Tracer advection. Replaces ATMOS_DYN_Tstep_tracer_fvm_heve
 * (scalelib/src/atmos-rm/dynamics/scale_atmos_dyn_tstep_tracer_fvm_heve.F90:72-240,
 * target of ATMOS_DYN_Tstep_tracer, scale_atmos_dyn_tstep_tracer.F90:32-68)
 * and the three-stage integrator ATMOS_DYN_tinteg_tracer_rk3
 * (scale_atmos_dyn_tinteg_tracer_rk3.F90:92-210), with the flux-corrected
 * transport limiter ATMOS_DYN_fct (scale_atmos_dyn_common.F90:1922-2734).
 * num_diff is (KA,IA,JA,3); GSQRT (KA,IA,JA,7); MAPF (IA,JA,2) at (x,y).
 * QTRCo may be the same array as QTRC0. num_diff may be NULL for ND_COEF_Q = 0.
 * ------------------------------------------------------------------------- */
#define SCALE_HEVI_TSTEP_TRACER_ARGS                                                                           \
    double *QTRCo, const double *QTRC, const double *QTRC0, const double *RHOQ_t,                              \
    const double *DENS0, const double *DENS, const double *mflx_hi, const double *num_diff,                    \
    const double *GSQRT, const double *MAPF,                                                                   \
    const double *CDZ, const double *RCDZ, const double *RCDX, const double *RCDY,                             \
    const double *dtl, const int *FLAG_FCT_TRACER, const int *FLAG_FCT_ALONG_STREAM

int ATMOS_DYN_Tstep_tracer_fvm_heve_b200(SCALE_HEVI_TSTEP_TRACER_ARGS);
int ATMOS_DYN_Tstep_tracer_fvm_heve_b200_dev(SCALE_HEVI_TSTEP_TRACER_ARGS);

#define SCALE_HEVI_TINTEG_TRACER_ARGS                                                                          \
    double *QTRC, const double *QTRC0, const double *RHOQ_t,                                                   \
    const double *DENS0, const double *DENS, const double *mflx_hi, const double *num_diff,                    \
    const double *GSQRT, const double *MAPF,                                                                   \
    const double *CDZ, const double *RCDZ, const double *RCDX, const double *RCDY,                             \
    const int *BND_W, const int *BND_E, const int *BND_S, const int *BND_N,                                    \
    const double *dtl, const int *FLAG_FCT_TRACER, const int *FLAG_FCT_ALONG_STREAM

int ATMOS_DYN_Tinteg_tracer_rk3_b200(SCALE_HEVI_TINTEG_TRACER_ARGS);
int ATMOS_DYN_Tinteg_tracer_rk3_b200_dev(SCALE_HEVI_TINTEG_TRACER_ARGS);

/* The same tracer RK3 (scale_atmos_dyn_tinteg_tracer_rk3.F90:92-210) on the
 * mixed-precision path: the high- and low-order fluxes and the FCT limiter
 * (scale_atmos_dyn_common.F90:1922-2734) in FP32, with FP32 mass fluxes,
 * tracer num_diff and tendency (the arrays of the mixed short step); the
 * tracer, its RK stage values, the densities and the update stay FP64. The
 * limiter's zero tests use the FP32 epsilon. Flat terrain; device pointers. */
#define SCALE_HEVI_TINTEG_TRACER_MIXED_ARGS                                                                    \
    double *QTRC, const double *QTRC0, const float *RHOQ_t,                                                    \
    const double *DENS0, const double *DENS, const float *mflx_hi, const float *num_diff,                      \
    const double *GSQRT, const double *MAPF,                                                                   \
    const double *CDZ, const double *RCDZ, const double *RCDX, const double *RCDY,                             \
    const int *BND_W, const int *BND_E, const int *BND_S, const int *BND_N,                                    \
    const double *dtl, const int *FLAG_FCT_TRACER, const int *FLAG_FCT_ALONG_STREAM
int ATMOS_DYN_Tinteg_tracer_rk3_b200_mixed_dev(SCALE_HEVI_TINTEG_TRACER_MIXED_ARGS);

/* ---------------------------------------------------------------------------
 * Periodic halo exchange of nfields consecutive (KA,IA,JA) device fields on
 * one GPU. Replaces COMM_vars8 + COMM_wait of a periodic single-rank domain
 * (scalelib/src/communication/scale_comm_cartesC.F90:345-397).
 * ------------------------------------------------------------------------- */
int COMM_vars8_b200_dev(double *var, const int *nfields);

/* ---------------------------------------------------------------------------
 * 3-D divergence of the momentum for divergence damping. Replaces
 * ATMOS_DYN_divergence (scale_atmos_dyn_common.F90:1437-1515), same arguments in
 * the same order. DDIV is written on k = KS-1..KE+1, i = IS..IE+1, j = JS..JE+1;
 * other cells keep their contents. Terrain-following metrics select the
 * metric form of the divergence (its J13G/J23G/GSQRT/MAPF terms).
 * ------------------------------------------------------------------------- */
#define SCALE_HEVI_DIVERGENCE_ARGS                                                                             \
    double *DDIV, const double *MOMZ, const double *MOMX, const double *MOMY,                                  \
    const double *GSQRT, const double *J13G, const double *J23G, const double *J33G, const double *MAPF,       \
    const double *RCDZ, const double *RCDX, const double *RCDY, const double *RFDZ, const double *FDZ

int ATMOS_DYN_divergence_b200(SCALE_HEVI_DIVERGENCE_ARGS);
int ATMOS_DYN_divergence_b200_dev(SCALE_HEVI_DIVERGENCE_ARGS);

/* ---------------------------------------------------------------------------
 * One large step of the dynamics on device-resident state. Replaces the
 * dynamics part of ATMOS_DYN_Tstep_large_fvm_heve
 * (scale_atmos_dyn_tstep_large_fvm_heve.F90:171-1130) for the supported
 * configuration: no lateral damping (DAMP_alpha = 0), ND_COEF_Q = 0,
 * USE_AVERAGE off, FLAG_TRACER_SPLIT_TEND off, EULER large-step integrator
 * (QTRC0 = QTRC). Per large step: RT2P, DPRES0 and REF_rhot from the moist
 * thermodynamics (:428-470); nstep = ceiling((DTLS-EPS)/DTSS) short steps, each
 * numfilter + divergence for the damping term when divdmp_coef > 0 (:860-871)
 * + RK4 short step + vertical boundary values + halo exchange;
 * then the RK3 tracer advection of every tracer with the short-step-averaged
 * mass flux. Arrays are device pointers; QTRC and RHOQ_tp are (KA,IA,JA,QA),
 * AQ_* are host arrays of length QA (QA <= 8). mflx_hi, tflx_hi and num_diff
 * are outputs, as in the reference.
 * ------------------------------------------------------------------------- */
int ATMOS_DYN_Tstep_large_fvm_heve_b200_dev(
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT, double *QTRC, const int *QA,
    double *mflx_hi, double *tflx_hi, double *num_diff,
    const double *DENS_tp, const double *MOMZ_tp, const double *MOMX_tp, const double *MOMY_tp,
    const double *RHOT_tp, const double *RHOQ_tp,
    const double *CORIOLI,
    const double *CDZ, const double *CDX, const double *CDY, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY, const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, const double *J33G, const double *MAPF,
    const double *AQ_R, const double *AQ_CV, const double *AQ_CP, const double *AQ_MASS,
    const double *REF_dens, const double *REF_pott, const double *REF_pres,
    const double *ND_COEF, const int *ND_ORDER, const double *ND_SFC_FACT, const int *ND_USE_RS,
    const double *wdamp_coef, const double *divdmp_coef,
    const int *FLAG_FCT_TRACER, const int *FLAG_FCT_ALONG_STREAM,
    const double *DTLS, const double *DTSS);

/* Host-array variant of the large step: copies the state in, runs, copies the
 * state, QTRC, mflx_hi, tflx_hi and num_diff back. Same arguments and results
 * as the device entry. The copies run on a second stream, inputs in the order
 * of first use and each output group as soon as it is final, so that with
 * page-locked host arrays they overlap the kernels; the call returns when all
 * copies have landed. Not capturable in a CUDA graph (rejected while a capture
 * is open). */
int ATMOS_DYN_Tstep_large_fvm_heve_b200(
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT, double *QTRC, const int *QA,
    double *mflx_hi, double *tflx_hi, double *num_diff,
    const double *DENS_tp, const double *MOMZ_tp, const double *MOMX_tp, const double *MOMY_tp,
    const double *RHOT_tp, const double *RHOQ_tp,
    const double *CORIOLI,
    const double *CDZ, const double *CDX, const double *CDY, const double *FDZ, const double *FDX, const double *FDY,
    const double *RCDZ, const double *RCDX, const double *RCDY, const double *RFDZ, const double *RFDX, const double *RFDY,
    const double *PHI, const double *GSQRT, const double *J13G, const double *J23G, const double *J33G, const double *MAPF,
    const double *AQ_R, const double *AQ_CV, const double *AQ_CP, const double *AQ_MASS,
    const double *REF_dens, const double *REF_pott, const double *REF_pres,
    const double *ND_COEF, const int *ND_ORDER, const double *ND_SFC_FACT, const int *ND_USE_RS,
    const double *wdamp_coef, const double *divdmp_coef,
    const int *FLAG_FCT_TRACER, const int *FLAG_FCT_ALONG_STREAM,
    const double *DTLS, const double *DTSS);

/* ---------------------------------------------------------------------------
 * Boundary values after a short step: the vertical boundary copy of
 * scale_atmos_dyn_tstep_large_fvm_heve.F90:910-926 followed by the periodic
 * halo exchange of the five prognostic fields (:929-944). Device arrays.
 * ------------------------------------------------------------------------- */
int scale_hevi_boundary_dev(double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT);

/* ---------------------------------------------------------------------------
 * Section timers, the counterpart of PROF_rapstart/PROF_rapend
 * (scalelib/src/common/scale_prof.F90:156,209): when enabled, CUDA events on
 * the library stream bracket each kernel section (hevi_horiz, hevi_column,
 * numfilter, halo, boundary, tracer, tracer_fct, large_prep, mflx_average).
 * scale_hevi_profile(1) enables and resets, scale_hevi_profile(0) disables;
 * the report is a JSON object {"section": [launches, total_ms], ...} and
 * synchronises the stream.
 * ------------------------------------------------------------------------- */
int scale_hevi_profile(int enable);
const char *scale_hevi_profile_report(void);

/* ---------------------------------------------------------------------------
 * Ensembles; no counterpart in the reference, where each member is a separate
 * run. n members of possibly different sizes (each its own index set, same
 * flux schemes) share one library state; every kernel of the short step then
 * advances all members in one launch. After scale_hevi_ensemble_setup the
 * short-step _dev entries (ATMOS_DYN_Tstep_short_fvm_hevi_b200_dev,
 * ATMOS_DYN_Tinteg_short_rk4_b200[_mixed]_dev,
 * ATMOS_DYN_numfilter_coef_b200[_mixed]_dev, scale_hevi_boundary_dev,
 * COMM_vars8_b200_dev) take POOLED arrays:
 *   - a 3-D field holds member m's (KA,IA,JA) array at point cell0[m]; a
 *     multi-component array (num_diff(...,15), mflx_hi(...,3), GSQRT(...,7))
 *     holds component q of member m at q*cell0[n] + cell0[m];
 *   - a 2-D field (CORIOLI) holds member m's (IA,JA) array at col0[m]
 *     (MAPF: component q at q*col0[n] + col0[m]);
 *   - a 1-D z vector (CDZ, FDZ, RCDZ, RFDZ, wdamp_coef) holds member m's KA
 *     values at z0[m] (FDZ/RFDZ use KA-1 of the KA slots); x and y vectors
 *     likewise at x0[m] (IA slots) and y0[m] (JA slots).
 * The time step and the filter and damping coefficients are common to all
 * members; divergence damping, the tracer, large-step, divergence and
 * domain-sum entries and the host-array entries need a single domain
 * (SCALE_HEVI_ERR_UNSUPPORTED otherwise). scale_hevi_setup(idx, ...) is
 * scale_hevi_ensemble_setup(1, idx, ...). At most 64 members.
 * scale_hevi_ensemble_layout fills arrays of n+1 entries with those offsets;
 * entry n holds the pooled totals. Any pointer may be NULL.
 * ------------------------------------------------------------------------- */
int scale_hevi_ensemble_setup(int n, const scale_hevi_index *idx, const char *flux_type,
                              const char *flux_tracer_type, int device);
int scale_hevi_ensemble_layout(long long *cell0, long long *col0, long long *z0, long long *x0, long long *y0);

/* ---------------------------------------------------------------------------
 * One short step of the large step's loop as ONE persistent launch; no
 * counterpart in the reference. The numerical filter of the state
 * (ATMOS_DYN_numfilter_coef, scale_atmos_dyn_common.F90:385-985, ND_ORDER 1,
 * ND_USE_RS, DT = dt), the RK4 short step of HEVI stages
 * (ATMOS_DYN_tinteg_short_rk4, scale_atmos_dyn_tinteg_short_rk4.F90:199-666),
 * the vertical boundary values and the lateral halo of the state
 * (scale_atmos_dyn_tstep_large_fvm_heve.F90:847-944): the same results, bit
 * for bit, as ATMOS_DYN_numfilter_coef_b200_dev,
 * ATMOS_DYN_Tinteg_short_rk4_b200_dev (tile width 16) and
 * scale_hevi_boundary_dev called in turn, for one domain or every member of
 * an ensemble (pooled arrays as above). Flat terrain (J33G = 1), no
 * divergence damping, no halo exchange hook; SCALE_HEVI_ERR_UNSUPPORTED when
 * the registered short step is not RK4 of HEVI stages.
 *
 * The launch is cooperative: as many CTAs as the GPU holds at once, which take
 * the blocks of each phase in turn and meet at a grid barrier between phases.
 * Every barrier waits at most a time limit (2 s unless
 * scale_hevi_persistent_wait says otherwise); on expiry the launch ends and
 * the next scale_hevi_check reports SCALE_HEVI_ERR_CUDA. The call can be
 * captured in a CUDA graph (scale_hevi_capture_begin). The _mixed form takes
 * the FP32 flux-like arrays of the mixed-precision path.
 *
 * scale_hevi_persistent_wait sets the barrier time limit (0 < seconds <= 60)
 * and, for a test of that limit, extra_arrivals = 1 makes every barrier wait
 * for one CTA more than the grid has, so that it expires. scale_hevi_persistent_grid
 * gives the CTA count of the last launch.
 * ------------------------------------------------------------------------- */
#define SCALE_HEVI_SHORT_STEP_ARGS                                                                             \
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT,                                      \
    double *mflx_hi, double *tflx_hi, double *num_diff,                                                        \
    const double *DENS_t, const double *MOMZ_t, const double *MOMX_t, const double *MOMY_t, const double *RHOT_t, \
    const double *DPRES0, const double *RT2P, const double *CORIOLI, const double *wdamp_coef,                 \
    const double *CDZ, const double *CDX, const double *CDY, const double *FDZ, const double *FDX,             \
    const double *FDY, const double *RCDZ, const double *RCDX, const double *RCDY,                             \
    const double *RFDZ, const double *RFDX, const double *RFDY,                                                \
    const double *REF_dens, const double *REF_pott, const double *REF_rhot,                                    \
    const double *ND_COEF, const double *ND_SFC_FACT, const double *dt
#define SCALE_HEVI_SHORT_STEP_MIXED_ARGS                                                                       \
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT,                                      \
    float *mflx_hi, float *tflx_hi, float *num_diff,                                                           \
    const float *DENS_t, const float *MOMZ_t, const float *MOMX_t, const float *MOMY_t, const float *RHOT_t,   \
    const double *DPRES0, const double *RT2P, const double *CORIOLI, const double *wdamp_coef,                 \
    const double *CDZ, const double *CDX, const double *CDY, const double *FDZ, const double *FDX,             \
    const double *FDY, const double *RCDZ, const double *RCDX, const double *RCDY,                             \
    const double *RFDZ, const double *RFDX, const double *RFDY,                                                \
    const double *REF_dens, const double *REF_pott, const double *REF_rhot,                                    \
    const double *ND_COEF, const double *ND_SFC_FACT, const double *dt

/* The numerical filter's form for one domain (no counterpart in the
 * reference): 1, the default after setup, forms num_diff from tiles of the
 * filtered quantities staged in shared memory by bulk tensor copies wherever
 * the arrays admit tensor maps (16-byte aligned bases and strides); 0 keeps the
 * column kernel. The results are identical. */
int scale_hevi_numfilter_form(int tiled);

/* The form of the FCT-limited tracer stage (ATMOS_DYN_fct inside
 * ATMOS_DYN_Tstep_tracer_fvm_heve, scale_atmos_dyn_common.F90:1922-2734; no
 * counterpart switch in the reference): 1, the default after setup, runs the
 * limiter fused with the fluxes (one kernel forms phi_lo, the anti-diffusive
 * fluxes and R+/R- from QTRC0 rows staged by bulk tensor copies, a second
 * limits and updates) wherever QTRC0 admits a tensor map (16-byte aligned
 * base, even KA); 0 keeps the three-kernel form (phi_lo and the
 * anti-diffusive fluxes through HBM). The FP64 results are identical. */
int scale_hevi_tracer_fct_form(int fused);

int scale_hevi_short_step_persistent_dev(SCALE_HEVI_SHORT_STEP_ARGS);
int scale_hevi_short_step_persistent_mixed_dev(SCALE_HEVI_SHORT_STEP_MIXED_ARGS);
int scale_hevi_persistent_wait(const double *seconds, const int *extra_arrivals);
int scale_hevi_persistent_grid(int *ctas);

/* ---------------------------------------------------------------------------
 * Launch shape of the stage kernel; no counterpart in the reference. A CTA
 * owns 16 columns as a tile of tile_x x (16/tile_x) columns (tile_x one of
 * 16, 8, 4) and CTAs are issued in raster groups of `raster` tile rows.
 * 0 selects the default (16, 16). The shape changes the speed only: results
 * are identical for every shape.
 * ------------------------------------------------------------------------- */
int scale_hevi_stage_shape(int tile_x, int raster);
/* Autotuner of that shape. With enable != 0, the next short-step call of each
 * path (FP64, mixed precision) outside a graph capture first times every
 * compiled tile width at raster heights 4, 16 and 64 on its own inputs (a
 * plain stage per candidate, outputs to library scratch; the caller's arrays
 * are not written) and keeps the fastest. scale_hevi_stage_shape() replaces
 * the choice and turns the tuner off. */
int scale_hevi_stage_autotune(int enable);
/* The shape in use on the FP64 (mixed = 0) or mixed-precision path. */
int scale_hevi_stage_shape_get(int *tile_x, int *raster, int mixed);
/* JSON record of the last tuning: {"path", "chosen": [tile_x, raster, ms],
 * "candidates": [[tile_x, raster, ms], ...]}; empty before one ran. */
const char *scale_hevi_autotune_report(void);

/* ---------------------------------------------------------------------------
 * Differentiated short step; no counterpart in the reference. The model is one
 * short step of a single flat-terrain domain as ATMOS_DYN_Tstep_large_fvm_heve
 * runs it (scale_atmos_dyn_tstep_large_fvm_heve.F90:847-944): the numerical
 * filter (ND_ORDER = 1) of the step's start state, the RK4 short integrator of
 * four HEVI stages without divergence damping, then the vertical boundary
 * values and the periodic halo. The large-step quantities (DPRES0, RT2P,
 * REF_rhot) and the base state are fixed parameters and the tendencies are
 * zero. A state X is one device buffer of 5*KA*IA*JA doubles: DENS, MOMZ,
 * MOMX, MOMY, RHOT.
 *   scale_hevi_adjoint_setup      parameters (device arrays, kept by pointer;
 *                                 1-D vectors and scalars on the host, copied)
 *   scale_hevi_short_step_dev     forward: X advanced one step (the fused kernels)
 *   scale_hevi_short_step_passes_dev
 *                                 the same step through the pass form the
 *                                 tangent-linear and adjoint linearise
 *   scale_hevi_short_step_tlm_dev X and its tangent dX advanced one step
 *   scale_hevi_short_step_adjoint_dev
 *                                 lam, the adjoint of the state after a step
 *                                 from X, replaced by the adjoint of X
 *   scale_hevi_boundary_adjoint_dev
 *                                 adjoint of scale_hevi_boundary_dev (on the
 *                                 5 fields of lam)
 *   scale_hevi_short_step_dd_dev  the pass-form step in double-double
 *                                 arithmetic (about 32 significant digits): the
 *                                 state is X_hi + X_lo. A finite-difference
 *                                 check of the adjoint runs it so that the
 *                                 rounding of the forward model stays far below
 *                                 the perturbation's effect
 * ------------------------------------------------------------------------- */
int scale_hevi_adjoint_setup(const double *DPRES0, const double *RT2P, const double *REF_rhot, const double *REF_dens,
                             const double *REF_pott, const double *PHI, const double *CORIOLI, const double *CDZ,
                             const double *CDX, const double *CDY, const double *FDZ, const double *FDX,
                             const double *FDY, const double *RCDZ, const double *RCDX, const double *RCDY,
                             const double *RFDZ, const double *RFDX, const double *RFDY, const double *wdamp_coef,
                             const double *dt, const double *ND_COEF, const double *ND_SFC_FACT, const double *J33G);
int scale_hevi_short_step_dev(double *X);
int scale_hevi_short_step_passes_dev(double *X);
int scale_hevi_short_step_tlm_dev(double *X, double *dX);
int scale_hevi_short_step_dd_dev(double *X_hi, double *X_lo);
int scale_hevi_short_step_adjoint_dev(const double *X, double *lam);
int scale_hevi_boundary_adjoint_dev(double *lam);

/* ---------------------------------------------------------------------------
 * CUDA graph of a call sequence on the library's stream; no counterpart in the
 * reference. Between scale_hevi_capture_begin() and scale_hevi_capture_end()
 * the _dev entries are recorded instead of run; scale_hevi_replay(&n) then
 * launches the recorded sequence n times. The entries must have run once
 * eagerly with the same arguments before the capture, so that their one-time
 * checks and table uploads (which synchronise) are already done. A new capture
 * replaces the previous graph; the graph keeps the pointers it was recorded
 * with.
 * ------------------------------------------------------------------------- */
int scale_hevi_capture_begin(void);
int scale_hevi_capture_end(void);
int scale_hevi_replay(const int *n);

/* ---------------------------------------------------------------------------
 * FP64 domain budget: total = sum over the interior of var*CDZ*CDX*CDY, the
 * mass total of check_mass (scalelib/src/atmos-rm/dynamics/scale_atmos_dyn.F90:530-688)
 * computed on the device with a fixed reduction order. var is a device
 * pointer, CDZ/CDX/CDY host arrays, total a host pointer. Synchronises.
 * ------------------------------------------------------------------------- */
int scale_hevi_domain_sum_dev(const double *var, const double *CDZ, const double *CDX, const double *CDY, double *total);

/* ---------------------------------------------------------------------------
 * FP64 energy budget of dry air: totals[0..3] = the domain totals of ENGT,
 * ENGP, ENGK and ENGI [J], the energies that scale-rm's monitor reports
 * (scale-rm/src/atmos/mod_atmos_vars.F90:768-778 registration, :2097-2171 the
 * per-cell values): ENGP = DENS*GRAV*CZ, ENGK = 0.5*DENS*(W^2+U^2+V^2) with the
 * cell-centre velocities of ATMOS_DIAGNOSTIC_CARTESC_get_vel (flat terrain),
 * ENGI = DENS*TEMP*CVdry with TEMP from rho*theta
 * (ATMOS_THERMODYN_rhot2temp_pres), ENGT = ENGP+ENGK+ENGI, each cell weighted
 * by CDZ*CDX*CDY and summed on the device in a fixed order. The state arrays
 * are device pointers, CZ/CDZ/CDX/CDY host arrays (KA, KA, IA, JA), totals a
 * host array of 4. One domain. Synchronises.
 * ------------------------------------------------------------------------- */
int scale_hevi_energy_sum_dev(const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY,
                              const double *RHOT, const double *CZ, const double *CDZ, const double *CDX,
                              const double *CDY, double *totals);

/* ---------------------------------------------------------------------------
 * One HEVI stage that allocates no device memory. This entry has no
 * counterpart in the reference. It exists for callers that cannot let a
 * library allocate GPU memory: a host model that owns the whole device budget
 * and hands out pieces of it, where a library cudaMalloc in the middle of a
 * run could fail or break its accounting, or a caller that cannot call
 * scale_hevi_setup.
 *
 * Arguments: the index set (halo 2) and the flux scheme, the cudaStream_t to
 * run on (as void*), then the argument list of
 * ATMOS_DYN_Tstep_short_fvm_hevi_b200_dev (device pointers for the 2-D/3-D
 * arrays, host pointers for the 1-D vectors and scalars). It computes what
 * that entry computes, bit for bit, for the 4-point schemes (UD3, CD4,
 * UD3KOREN1993, CD2; the 6-point schemes need a halo of 3) on flat terrain.
 * Terrain-following metrics are refused with SCALE_HEVI_ERR_UNSUPPORTED: the
 * general-metric stage needs work arrays. A metric set (device and the four
 * pointers) found flat once is remembered in host memory and not checked
 * again, which assumes its contents do not change.
 *
 * Scratch: one fixed device array of SCALE_HEVI_NOALLOC_SCRATCH_BYTES inside
 * the library holds the status words, three per-level fields of the column
 * solve and the 1-D grid tables: 256 + 8*(3*KA*IA*JA + 7*KA + 4*IA + 4*JA)
 * bytes. A larger domain is rejected with SCALE_HEVI_ERR_ARG. Every call looks
 * the array up with the caller's device current; the first lookup on a device
 * can load the module, so make the first call before any stream capture. The
 * entry synchronises the stream before it returns, so it cannot itself be
 * captured. All calls on a device share the array, so calls that overlap in
 * time race.
 * ------------------------------------------------------------------------- */
#define SCALE_HEVI_NOALLOC_SCRATCH_BYTES (32UL * 1024UL * 1024UL)
int ATMOS_DYN_Tstep_short_fvm_hevi_b200_noalloc(const scale_hevi_index *idx, const char *flux_type, void *stream,
                                                SCALE_HEVI_TSTEP_SHORT_ARGS);

#ifdef __cplusplus
}
#endif
#endif /* SCALE_HEVI_H */
