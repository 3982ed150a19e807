/* Internal helpers of the CPU oracle (test infrastructure only). */
#ifndef OG_INTERNAL_H
#define OG_INTERNAL_H

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "scale_oracle.h"

/* Unpack the index set into locals named as in the reference. */
#define OG_DIMS(d)                                                        \
    const int KA = (d)->KA, IA = (d)->IA, JA = (d)->JA;                   \
    const int KS = (d)->KS, KE = (d)->KE, IS = (d)->IS, IE = (d)->IE;     \
    const int JS = (d)->JS, JE = (d)->JE, KMAX = (d)->KMAX;               \
    const int IEH = (d)->IEH, JEH = (d)->JEH;                             \
    const size_t N3 = (size_t)KA * (size_t)IA * (size_t)JA;               \
    (void)KA; (void)IA; (void)JA; (void)KS; (void)KE; (void)IS; (void)IE; \
    (void)JS; (void)JE; (void)KMAX; (void)IEH; (void)JEH; (void)N3

/* 1-based Fortran (k,i,j) -> linear offset, k fastest */
#define I3(k, i, j) ((size_t)((k) - 1) + (size_t)KA * ((size_t)((i) - 1) + (size_t)IA * (size_t)((j) - 1)))
/* (i,j) plane offset for arrays declared (IA,JA,...) */
#define I2(i, j) ((size_t)((i) - 1) + (size_t)IA * (size_t)((j) - 1))

/* staggering ids, scale_atmos_grid_cartesC_index.F90:90-101 */
enum { I_XYZ = 1, I_XYW, I_UYW, I_XVW, I_UYZ, I_XVZ, I_UVZ };
enum { I_XY = 1, I_UY, I_XV, I_UV };
/* variable ids, scale_index.F90:28-32; directions ZDIR=1,XDIR=2,YDIR=3 */
enum { I_DENS = 1, I_MOMZ, I_MOMX, I_MOMY, I_RHOT };
enum { ZDIR = 1, XDIR, YDIR };

/* slices of the 4-D/5-D reference arrays */
#define G4(a, idx) ((a) + (size_t)((idx) - 1) * N3)                  /* GSQRT(:,:,:,idx) */
#define ND(nd, v, dir) ((nd) + N3 * (size_t)(((v) - 1) + 5 * ((dir) - 1))) /* num_diff(:,:,:,v,dir) */
#define MAPF4(m, b) ((m) + (size_t)IA * (size_t)JA * 2 * (size_t)((b) - 1)) /* MAPF(:,:,:,b) */
#define MP(m, i, j, a) (m)[I2(i, j) + (size_t)IA * (size_t)JA * (size_t)((a) - 1)] /* MAPF(i,j,a) of a slice */

static inline double og_sign(double a, double b) { return copysign(fabs(a), b); }
static inline double og_max(double a, double b) { return a > b ? a : b; }
static inline double og_min(double a, double b) { return a < b ? a : b; }

/* Koren (1993) limiter of UD3KOREN1993, scale_atmos_dyn_fvm_flux_ud3Koren1993.F90:1690-1710 */
static inline double og_koren_phi(double v1, double v2, double v3)
{
    const double EPS = OG_EPS;
    const double zerosw1 = EPS - og_sign(EPS, fabs(v1 - v2) - EPS);
    const double zerosw2 = EPS - og_sign(EPS, fabs(v2 - v3) - EPS);
    const double r2 = 2.0 * (v1 - v2 + zerosw1 * zerosw2) / (v2 - v3 + zerosw2);
    return og_max(0.0, og_min(r2, og_min((1.0 + r2) / 3.0, 2.0)));
}

/* flux scheme kernels (UD3: scale_atmos_dyn_fvm_flux_ud3.F90:84-89,124-149;
 * CD4: scale_atmos_dyn_fvm_flux_cd4.F90:87-88,123-142; CD2: ..._cd2.F90, the
 * same F2*(v0+vp1) at every face; UD3KOREN1993: the limited upwind value of
 * ..._ud3Koren1993.F90:200-206 (interior), :236-241 (above KS), :243-249
 * (below KE)). The face lies between v0 and vp1; vm1/vp2 are the outer points. */
#define F2_  0.5
#define F31 (-1.0 / 12.0)
#define F32 (7.0 / 12.0)
#define F33 (3.0 / 12.0)
#define F41 (7.0 / 12.0)
#define F42 (-1.0 / 12.0)

static inline double og_ip4(int scheme, double vel, double vm1, double v0, double vp1, double vp2)
{
    if (scheme == OG_UD3)
        return (F31 * (vp2 + vm1) + F32 * (vp1 + v0)) - (F31 * (vp2 - vm1) + F33 * (vp1 - v0)) * og_sign(1.0, vel);
    if (scheme == OG_CD2)
        return F2_ * (vp1 + v0);
    if (scheme == OG_KOREN)
        return (v0 + 0.5 * og_koren_phi(vp1, v0, vm1) * (v0 - vm1)) * (0.5 + og_sign(0.5, vel))
               + (vp1 + 0.5 * og_koren_phi(v0, vp1, vp2) * (vp1 - vp2)) * (0.5 - og_sign(0.5, vel));
    return F41 * (vp1 + v0) + F42 * (vp2 + vm1);
}
/* one-sided value at the KS face from val(KS), val(KS+1), val(KS+2) */
static inline double og_ipL(int scheme, double vel, double v0, double v1, double v2)
{
    if (scheme == OG_UD3 || scheme == OG_UD5)
        return F2_ * (v1 + v0) * (0.5 + og_sign(0.5, vel)) + (2.0 * v0 + 5.0 * v1 - v2) / 6.0 * (0.5 - og_sign(0.5, vel));
    if (scheme == OG_KOREN)
        return v0 * (0.5 + og_sign(0.5, vel)) + (v1 + 0.5 * og_koren_phi(v0, v1, v2) * (v1 - v2)) * (0.5 - og_sign(0.5, vel));
    return F2_ * (v1 + v0);
}
/* one-sided value at the KE-1 face from val(KE), val(KE-1), val(KE-2) */
static inline double og_ipH(int scheme, double vel, double vE, double vE1, double vE2)
{
    if (scheme == OG_UD3 || scheme == OG_UD5)
        return (2.0 * vE + 5.0 * vE1 - vE2) / 6.0 * (0.5 + og_sign(0.5, vel)) + F2_ * (vE + vE1) * (0.5 - og_sign(0.5, vel));
    if (scheme == OG_KOREN)
        return (vE1 + 0.5 * og_koren_phi(vE2, vE1, vE) * (vE1 - vE)) * (0.5 + og_sign(0.5, vel)) + vE * (0.5 - og_sign(0.5, vel));
    return F2_ * (vE + vE1);
}

/* ---- 6-point schemes (scale_atmos_dyn_fvm_flux_ud5.F90, ..._cd6.F90; one
 * generator template, scale_atmos_dyn_fvm_flux_udcd.F90.erb). The interior face
 * value uses two points more on each side (IHALO = JHALO = 3); in z, where the
 * halo is 2, the faces KS+1 and KE-2 take the forms og_ipL2/og_ipH2 and the
 * faces KS and KE-1 the UD3 (UD5) or F2 (CD6) forms of og_ipL/og_ipH. */
#define F51 (1.0 / 60.0)
#define F52 (-8.0 / 60.0)
#define F53 (37.0 / 60.0)
#define F54 (-5.0 / 60.0)
#define F55 (10.0 / 60.0)
#define F61 (37.0 / 60.0)
#define F62 (-8.0 / 60.0)
#define F63 (1.0 / 60.0)

static inline int og_wide(int scheme) { return scheme == OG_UD5 || scheme == OG_CD6; }

/* ud5.F90:92-96,133-138 ; cd6.F90:89-91,130-132. The face lies between v0 and vp1. */
static inline double og_ip6(int scheme, double vel, double vm2, double vm1, double v0, double vp1, double vp2,
                            double vp3)
{
    if (scheme == OG_UD5)
        return (F51 * (vp3 + vm2) + F52 * (vp2 + vm1) + F53 * (vp1 + v0))
               - (F51 * (vp3 - vm2) + F54 * (vp2 - vm1) + F55 * (vp1 - v0)) * og_sign(1.0, vel);
    if (scheme == OG_CD6)
        return F61 * (vp1 + v0) + F62 * (vp2 + vm1) + F63 * (vp3 + vm2);
    return og_ip4(scheme, vel, vm1, v0, vp1, vp2);
}
/* the KS+1 face from val(KS..KS+4): ud5.F90:171-177, cd6.F90:159-160 */
static inline double og_ipL2(int scheme, double vel, double v0, double v1, double v2, double v3, double v4)
{
    if (scheme == OG_UD5)
        return (2.0 * v2 + 5.0 * v1 - v0) / 6.0 * (0.5 + og_sign(0.5, vel))
               + (-3.0 * v0 + 27.0 * v1 + 47.0 * v2 - 13.0 * v3 + 2.0 * v4) / 60.0 * (0.5 - og_sign(0.5, vel));
    return F41 * (v2 + v1) + F42 * (v3 + v0);
}
/* the KE-2 face from val(KE), val(KE-1), ..., val(KE-4): ud5.F90:179-185, cd6.F90:161-162 */
static inline double og_ipH2(int scheme, double vel, double vE, double vE1, double vE2, double vE3, double vE4)
{
    if (scheme == OG_UD5)
        return (-3.0 * vE + 27.0 * vE1 + 47.0 * vE2 - 13.0 * vE3 + 2.0 * vE4) / 60.0 * (0.5 + og_sign(0.5, vel))
               + (2.0 * vE2 + 5.0 * vE1 - vE) / 6.0 * (0.5 - og_sign(0.5, vel));
    return F41 * (vE1 + vE2) + F42 * (vE + vE3);
}

/* Face value between p[0] and p[s] along a horizontal direction of stride s:
 * the 4-point value from p[-s..2s], or the 6-point one from p[-2s..3s]. */
static inline double og_hface(int scheme, double vel, const double *p, long s)
{
    if (og_wide(scheme)) return og_ip6(scheme, vel, p[-2 * s], p[-s], p[0], p[s], p[2 * s], p[3 * s]);
    return og_ip4(scheme, vel, p[-s], p[0], p[s], p[2 * s]);
}

/* Face value at the w-level m (between levels m and m+1) of a column whose
 * level l is col[l-1], with the near-wall forms of the scheme: og_ipL at KS,
 * og_ipH at KE-1, and for the 6-point schemes og_ipL2 at KS+1, og_ipH2 at KE-2
 * (the k-loops KS+1..KE-2 of ud3.F90 and KS+2..KE-3 of ud5.F90/cd6.F90). */
static inline double og_zface(int scheme, double vel, const double *col, int m, int KS, int KE)
{
#define V_(l) col[(l) - 1]
    if (m == KS) return og_ipL(scheme, vel, V_(KS), V_(KS + 1), V_(KS + 2));
    if (m == KE - 1) return og_ipH(scheme, vel, V_(KE), V_(KE - 1), V_(KE - 2));
    if (og_wide(scheme)) {
        if (m == KS + 1) return og_ipL2(scheme, vel, V_(KS), V_(KS + 1), V_(KS + 2), V_(KS + 3), V_(KS + 4));
        if (m == KE - 2) return og_ipH2(scheme, vel, V_(KE), V_(KE - 1), V_(KE - 2), V_(KE - 3), V_(KE - 4));
        return og_ip6(scheme, vel, V_(m - 2), V_(m - 1), V_(m), V_(m + 1), V_(m + 2), V_(m + 3));
    }
    return og_ip4(scheme, vel, V_(m - 1), V_(m), V_(m + 1), V_(m + 2));
#undef V_
}

/* ---- work arrays and the stage bodies (og_hevi.c, og_heve.c) ---- */
typedef struct {
    double *POTT, *DPRES, *qflx_hi, *qflx_J13, *qflx_J23, *Sr, *Sw, *St;
} og_stage_work;
int og_stage_work_alloc(og_stage_work *w, size_t N3);
int og_short_type_get(void);        /* the registered short step: 0 HEVI, 1 HEVE */
int og_tinteg_short_type_get(void); /* the registered short integrator: 0 RK4, 1 RK3, 2 RK3WS2002 */
void og_stage_work_free(og_stage_work *w);
typedef int (*og_stage_fn)(
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
    double dtrk);
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
    double dtrk);

/* ---- flux family (19 routines), one generic restatement per reference routine ---- */
typedef struct {
    int IIS, IIE, JJS, JJE;
} og_blk;

void og_valueW_Z(const og_dims *d, int scheme, double *valW, const double *mflx, const double *val);
void og_fluxZ_XYZ(const og_dims *d, int scheme, double *flux, const double *mflx, const double *val,
                  const double *GSQRT, const double *nd, og_blk b);
void og_fluxX_XYZ(const og_dims *d, int scheme, double *flux, const double *mflx, const double *val,
                  const double *GSQRT, const double *nd, og_blk b);
void og_fluxY_XYZ(const og_dims *d, int scheme, double *flux, const double *mflx, const double *val,
                  const double *GSQRT, const double *nd, og_blk b);
void og_fluxZ_XYW(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, double J33G, const double *nd, og_blk b);
void og_fluxJ13_XYW(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *J13G, const double *MAPF, og_blk b);
void og_fluxJ23_XYW(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *J23G, const double *MAPF, og_blk b);
void og_fluxX_XYW(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd,
                  const double *CDZ, og_blk b);
void og_fluxY_XYW(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd,
                  const double *CDZ, og_blk b);
void og_fluxZ_UYZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, double J33G, const double *nd,
                  const double *CDZ, og_blk b);
void og_fluxJ13_UYZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *GSQRT, const double *J13G, const double *MAPF,
                    const double *CDZ, og_blk b);
void og_fluxJ23_UYZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *GSQRT, const double *J23G, const double *MAPF,
                    const double *CDZ, og_blk b);
void og_fluxX_UYZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd, og_blk b);
void og_fluxY_UYZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd, og_blk b);
void og_fluxZ_XVZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, double J33G, const double *nd,
                  const double *CDZ, og_blk b);
void og_fluxJ13_XVZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *GSQRT, const double *J13G, const double *MAPF,
                    const double *CDZ, og_blk b);
void og_fluxJ23_XVZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *GSQRT, const double *J23G, const double *MAPF,
                    const double *CDZ, og_blk b);
void og_fluxX_XVZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd, og_blk b);
void og_fluxY_XVZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd, og_blk b);

/* donor-cell (UD1) tracer fluxes, scale_atmos_dyn_fvm_flux_ud1.F90:135-294 */
void og_fluxZ_XYZ_ud1(const og_dims *d, double *flux, const double *mflx, const double *val, og_blk b);
void og_fluxX_XYZ_ud1(const og_dims *d, double *flux, const double *mflx, const double *val, og_blk b);
void og_fluxY_XYZ_ud1(const og_dims *d, double *flux, const double *mflx, const double *val, og_blk b);

/* FCT limiter, scale_atmos_dyn_common.F90:1922-2734 */
void og_fct(const og_dims *d, double *qflx_anti, const double *phi_in, const double *DENS0, const double *DENS,
            const double *qflx_hi, const double *qflx_lo, const double *mflx_hi,
            const double *RDZ, const double *RDX, const double *RDY,
            const double *GSQRT, const double *MAPF, double dt, int flag_vect);

static inline double *og_alloc(size_t n)
{
    double *p = (double *)malloc(n * sizeof(double));
    return p;
}
/* fill with a NaN sentinel so that any read of a cell the reference leaves
 * undefined shows up in the parity tests (the reference DEBUG build fills UNDEF) */
static inline double *og_alloc_undef(size_t n)
{
    double *p = og_alloc(n);
    if (p) for (size_t q = 0; q < n; ++q) p[q] = NAN;
    return p;
}

#endif
