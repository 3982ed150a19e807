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
    if (scheme == OG_UD3)
        return F2_ * (v1 + v0) * (0.5 + og_sign(0.5, vel)) + (2.0 * v0 + 5.0 * v1 - v2) / 6.0 * (0.5 - og_sign(0.5, vel));
    if (scheme == OG_KOREN)
        return v0 * (0.5 + og_sign(0.5, vel)) + (v1 + 0.5 * og_koren_phi(v0, v1, v2) * (v1 - v2)) * (0.5 - og_sign(0.5, vel));
    return F2_ * (v1 + v0);
}
/* one-sided value at the KE-1 face from val(KE), val(KE-1), val(KE-2) */
static inline double og_ipH(int scheme, double vel, double vE, double vE1, double vE2)
{
    if (scheme == OG_UD3)
        return (2.0 * vE + 5.0 * vE1 - vE2) / 6.0 * (0.5 + og_sign(0.5, vel)) + F2_ * (vE + vE1) * (0.5 - og_sign(0.5, vel));
    if (scheme == OG_KOREN)
        return (vE1 + 0.5 * og_koren_phi(vE2, vE1, vE) * (vE1 - vE)) * (0.5 + og_sign(0.5, vel)) + vE * (0.5 - og_sign(0.5, vel));
    return F2_ * (vE + vE1);
}

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
