/*
 * Oracle restatement of the FVM flux family used by the HEVI short step.
 *
 * Each routine follows the loop bounds, index shifts and arithmetic of the
 * reference routine of the same name in
 *   scalelib/src/atmos-rm/dynamics/scale_atmos_dyn_fvm_flux_ud3.F90 (UD3)
 *   scalelib/src/atmos-rm/dynamics/scale_atmos_dyn_fvm_flux_cd4.F90 (CD4)
 *   ..._cd2.F90, ..._ud5.F90, ..._cd6.F90 (CD2, UD5, CD6)
 *   ..._ud3Koren1993.F90 (UD3KOREN1993)
 * The UD/CD files are generated from one template (scale_atmos_dyn_fvm_flux_udcd.F90.erb)
 * and differ only in the face interpolation and the near-wall formulas: og_hface
 * along x and y, og_zface along z (og_internal.h). Each z routine loops over all
 * its faces; the reference's separate statements at KS and KE-1 (and, for the
 * 6-point schemes, KS+1 and KE-2) use the same velocity formula as its interior
 * loop and differ only in the face value, which og_zface selects by level.
 * Line numbers cite the UD3 file.
 */
#include "og_internal.h"

/* F2H(k,p): cell-to-face weight, scale_atmos_dyn_fvm_flux_ud3.F90:75 (GSQRT is the
 * 3-D slice passed to the routine) */
#define F2H(k, p) (CDZ[(k) + (p) - 2] * GSQRT[I3((k) + (p) - 1, i, j)] / \
                   (CDZ[(k) - 1] * GSQRT[I3(k, i, j)] + CDZ[(k)] * GSQRT[I3((k) + 1, i, j)]))

/* ud3.F90:98-153 */
void og_valueW_Z(const og_dims *d, int scheme, double *valW, const double *mflx, const double *val)
{
    const int KS = d->KS, KE = d->KE;
    for (int m = KS; m <= KE - 1; ++m) valW[m - 1] = og_zface(scheme, mflx[m - 1], val, m, KS, KE);
}

/* ud3.F90:157-247 */
void og_fluxZ_XYZ(const og_dims *d, int scheme, double *flux, const double *mflx, const double *val,
                  const double *GSQRT, const double *nd, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double vel = mflx[I3(k, i, j)];
                flux[I3(k, i, j)] = vel * og_zface(scheme, vel, &val[I3(1, i, j)], k, KS, KE)
                                    + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
            flux[I3(KS - 1, i, j)] = 0.0;
            flux[I3(KE, i, j)] = 0.0;
        }
}

/* ud3.F90:251-300 */
void og_fluxX_XYZ(const og_dims *d, int scheme, double *flux, const double *mflx, const double *val,
                  const double *GSQRT, const double *nd, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS - 1; i <= b.IIE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double vel = mflx[I3(k, i, j)];
                flux[I3(k, i, j)] = vel * og_hface(scheme, vel, &val[I3(k, i, j)], (long)KA)
                                    + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
}

/* ud3.F90:304-353 */
void og_fluxY_XYZ(const og_dims *d, int scheme, double *flux, const double *mflx, const double *val,
                  const double *GSQRT, const double *nd, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS - 1; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double vel = mflx[I3(k, i, j)];
                flux[I3(k, i, j)] = vel * og_hface(scheme, vel, &val[I3(k, i, j)], (long)KA * IA)
                                    + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
}

/* ud3.F90:358-452 (z-index of the result is shifted by -1) */
void og_fluxZ_XYW(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, double J33G, const double *nd, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            /* flux(k-1) for k = KS+1..KE-1: the KS face (ud3.F90:424-432) and the
             * interior loop (:376-402) share the same velocity formula */
            for (int k = KS + 1; k <= KE - 1; ++k) {
                double vel = (0.5 * (mom[I3(k - 1, i, j)] + mom[I3(k, i, j)])) / DENS[I3(k, i, j)];
                flux[I3(k - 1, i, j)] = J33G * vel * og_zface(scheme, vel, &val[I3(1, i, j)], k - 1, KS, KE)
                                        + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
            flux[I3(KS - 1, i, j)] = 0.0;
            flux[I3(KE - 1, i, j)] = 0.0;
            flux[I3(KE, i, j)] = 0.0;
        }
}

/* ud3.F90:457-523 */
void og_fluxJ13_XYW(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *J13G, const double *MAPF, og_blk b)
{
    OG_DIMS(d);
    /* 4-point schemes: flux(k-1) for k = KS+2..KE-1 (ud3.F90); 6-point ones: for
     * k = KS+2..KE-2 from val(k-3..k+2), and at KE-2 the 3-point form of the KE-1
     * face one level lower (ud5.F90:604-657, cd6.F90) */
    const int wide = og_wide(scheme), kend = wide ? KE - 2 : KE - 1;
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            for (int k = KS + 2; k <= kend; ++k) {
                double vel = (0.5 * (mom[I3(k, i, j)] + mom[I3(k, i - 1, j)])) / DENS[I3(k, i, j)];
                vel = vel * J13G[I3(k, i, j)];
                const double q = wide ? og_ip6(scheme, vel, val[I3(k - 3, i, j)], val[I3(k - 2, i, j)], val[I3(k - 1, i, j)],
                                               val[I3(k, i, j)], val[I3(k + 1, i, j)], val[I3(k + 2, i, j)])
                                      : og_ip4(scheme, vel, val[I3(k - 2, i, j)], val[I3(k - 1, i, j)],
                                               val[I3(k, i, j)], val[I3(k + 1, i, j)]);
                flux[I3(k - 1, i, j)] = vel / MP(MAPF, i, j, 2) * q;
            }
            flux[I3(KS - 1, i, j)] = 0.0;
            double vel = ((0.5 * (mom[I3(KS + 1, i, j)] + mom[I3(KS + 1, i - 1, j)])) / DENS[I3(KS + 1, i, j)]
                          + (0.5 * (mom[I3(KS, i, j)] + mom[I3(KS, i - 1, j)])) / DENS[I3(KS, i, j)]) * 0.5;
            vel = vel * J13G[I3(KS + 1, i, j)];
            flux[I3(KS, i, j)] = vel / MP(MAPF, i, j, 2)
                                 * og_ipL(scheme, vel, val[I3(KS, i, j)], val[I3(KS + 1, i, j)], val[I3(KS + 2, i, j)]);
            if (wide) {
                vel = (0.5 * (mom[I3(KE - 1, i, j)] + mom[I3(KE - 1, i - 1, j)])) / DENS[I3(KE - 1, i, j)];
                vel = vel * J13G[I3(KE - 1, i, j)];
                flux[I3(KE - 2, i, j)] = vel / MP(MAPF, i, j, 2)
                                         * og_ipH(scheme, vel, val[I3(KE - 1, i, j)], val[I3(KE - 2, i, j)], val[I3(KE - 3, i, j)]);
            }
            flux[I3(KE - 1, i, j)] = 0.0;
        }
}

/* ud3.F90:527-593 */
void og_fluxJ23_XYW(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *J23G, const double *MAPF, og_blk b)
{
    OG_DIMS(d);
    /* 4-point schemes: flux(k-1) for k = KS+2..KE-1 (ud3.F90); 6-point ones: for
     * k = KS+2..KE-2 from val(k-3..k+2), and at KE-2 the 3-point form of the KE-1
     * face one level lower (ud5.F90:604-657, cd6.F90) */
    const int wide = og_wide(scheme), kend = wide ? KE - 2 : KE - 1;
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            for (int k = KS + 2; k <= kend; ++k) {
                double vel = (0.5 * (mom[I3(k, i, j)] + mom[I3(k, i, j - 1)])) / DENS[I3(k, i, j)];
                vel = vel * J23G[I3(k, i, j)];
                const double q = wide ? og_ip6(scheme, vel, val[I3(k - 3, i, j)], val[I3(k - 2, i, j)], val[I3(k - 1, i, j)],
                                               val[I3(k, i, j)], val[I3(k + 1, i, j)], val[I3(k + 2, i, j)])
                                      : og_ip4(scheme, vel, val[I3(k - 2, i, j)], val[I3(k - 1, i, j)],
                                               val[I3(k, i, j)], val[I3(k + 1, i, j)]);
                flux[I3(k - 1, i, j)] = vel / MP(MAPF, i, j, 1) * q;
            }
            flux[I3(KS - 1, i, j)] = 0.0;
            double vel = ((0.5 * (mom[I3(KS + 1, i, j)] + mom[I3(KS + 1, i, j - 1)])) / DENS[I3(KS + 1, i, j)]
                          + (0.5 * (mom[I3(KS, i, j)] + mom[I3(KS, i, j - 1)])) / DENS[I3(KS, i, j)]) * 0.5;
            vel = vel * J23G[I3(KS + 1, i, j)];
            flux[I3(KS, i, j)] = vel / MP(MAPF, i, j, 1)
                                 * og_ipL(scheme, vel, val[I3(KS, i, j)], val[I3(KS + 1, i, j)], val[I3(KS + 2, i, j)]);
            if (wide) {
                vel = (0.5 * (mom[I3(KE - 1, i, j)] + mom[I3(KE - 1, i, j - 1)])) / DENS[I3(KE - 1, i, j)];
                vel = vel * J23G[I3(KE - 1, i, j)];
                flux[I3(KE - 2, i, j)] = vel / MP(MAPF, i, j, 1)
                                         * og_ipH(scheme, vel, val[I3(KE - 1, i, j)], val[I3(KE - 2, i, j)], val[I3(KE - 3, i, j)]);
            }
            flux[I3(KE - 1, i, j)] = 0.0;
        }
}

/* ud3.F90:598-671 */
void og_fluxX_XYW(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd,
                  const double *CDZ, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS - 1; i <= b.IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double vel = (F2H(k, 1) * mom[I3(k + 1, i, j)] + F2H(k, 2) * mom[I3(k, i, j)])
                             / (F2H(k, 1) * 0.5 * (DENS[I3(k + 1, i, j)] + DENS[I3(k + 1, i + 1, j)])
                                + F2H(k, 2) * 0.5 * (DENS[I3(k, i, j)] + DENS[I3(k, i + 1, j)]));
                flux[I3(k, i, j)] = GSQRT[I3(k, i, j)] / MP(MAPF, i, j, 2) * vel
                                    * og_hface(scheme, vel, &val[I3(k, i, j)], (long)KA)
                                    + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
            flux[I3(KE, i, j)] = 0.0;
        }
}

/* ud3.F90:675-748 */
void og_fluxY_XYW(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd,
                  const double *CDZ, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS - 1; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double vel = (F2H(k, 1) * mom[I3(k + 1, i, j)] + F2H(k, 2) * mom[I3(k, i, j)])
                             / (F2H(k, 1) * 0.5 * (DENS[I3(k + 1, i, j)] + DENS[I3(k + 1, i, j + 1)])
                                + F2H(k, 2) * 0.5 * (DENS[I3(k, i, j)] + DENS[I3(k, i, j + 1)]));
                flux[I3(k, i, j)] = GSQRT[I3(k, i, j)] / MP(MAPF, i, j, 1) * vel
                                    * og_hface(scheme, vel, &val[I3(k, i, j)], (long)KA * IA)
                                    + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
            flux[I3(KE, i, j)] = 0.0;
        }
}

/* denominator shared by the UYZ routines: face-weighted density at (u,y,w) */
#define DEN_UYZ(k) (F2H(k, 1) * 0.5 * (DENS[I3((k) + 1, i, j)] + DENS[I3((k) + 1, i + 1, j)]) \
                    + F2H(k, 2) * 0.5 * (DENS[I3(k, i, j)] + DENS[I3(k, i + 1, j)]))
#define DEN_XVZ(k) (F2H(k, 1) * 0.5 * (DENS[I3((k) + 1, i, j)] + DENS[I3((k) + 1, i, j + 1)]) \
                    + F2H(k, 2) * 0.5 * (DENS[I3(k, i, j)] + DENS[I3(k, i, j + 1)]))

/* ud3.F90:753-859 */
void og_fluxZ_UYZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, double J33G, const double *nd,
                  const double *CDZ, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double vel = (0.5 * (mom[I3(k, i, j)] + mom[I3(k, i + 1, j)])) / DEN_UYZ(k);
                flux[I3(k, i, j)] = J33G * vel * og_zface(scheme, vel, &val[I3(1, i, j)], k, KS, KE)
                                    + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
            flux[I3(KS - 1, i, j)] = 0.0;
            flux[I3(KE, i, j)] = 0.0;
        }
}

/* ud3.F90:863-954 */
void og_fluxJ13_UYZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *GSQRT, const double *J13G, const double *MAPF,
                    const double *CDZ, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double vel = (F2H(k, 1) * mom[I3(k + 1, i, j)] + F2H(k, 2) * mom[I3(k, i, j)]) / DEN_UYZ(k);
                vel = vel * J13G[I3(k, i, j)];
                flux[I3(k, i, j)] = vel / MP(MAPF, i, j, 2)
                                    * og_zface(scheme, vel, &val[I3(1, i, j)], k, KS, KE);
            }
            flux[I3(KS - 1, i, j)] = 0.0;
            flux[I3(KE, i, j)] = 0.0;
        }
}

/* 4-point average of a v-point field onto a u-point, as written in ud3.F90:988-990 */
#define AVG4_UV(m, k) (0.25 * ((m)[I3(k, i, j)] + (m)[I3(k, i + 1, j)] + (m)[I3(k, i, j - 1)] + (m)[I3(k, i + 1, j - 1)]))

/* ud3.F90:958-1049 */
void og_fluxJ23_UYZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *GSQRT, const double *J23G, const double *MAPF,
                    const double *CDZ, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double vel = (F2H(k, 1) * AVG4_UV(mom, k + 1) + F2H(k, 2) * AVG4_UV(mom, k)) / DEN_UYZ(k);
                vel = vel * J23G[I3(k, i, j)];
                flux[I3(k, i, j)] = vel / MP(MAPF, i, j, 1)
                                    * og_zface(scheme, vel, &val[I3(1, i, j)], k, KS, KE);
            }
            flux[I3(KS - 1, i, j)] = 0.0;
            flux[I3(KE, i, j)] = 0.0;
        }
}

/* ud3.F90:1053-1109 (x-index of the result is shifted by -1) */
void og_fluxX_UYZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE + 1; ++i)
            for (int k = KS; k <= KE; ++k) {
                double vel = (0.5 * (mom[I3(k, i, j)] + mom[I3(k, i - 1, j)])) / (DENS[I3(k, i, j)]);
                flux[I3(k, i - 1, j)] = GSQRT[I3(k, i, j)] / MP(MAPF, i, j, 2) * vel
                                        * og_hface(scheme, vel, &val[I3(k, i - 1, j)], (long)KA)
                                        + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
}

/* ud3.F90:1113-1167 */
void og_fluxY_UYZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS - 1; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double vel = (0.5 * (mom[I3(k, i, j)] + mom[I3(k, i + 1, j)]))
                             / (0.25 * (DENS[I3(k, i, j)] + DENS[I3(k, i + 1, j)] + DENS[I3(k, i, j + 1)] + DENS[I3(k, i + 1, j + 1)]));
                flux[I3(k, i, j)] = GSQRT[I3(k, i, j)] / MP(MAPF, i, j, 1) * vel
                                    * og_hface(scheme, vel, &val[I3(k, i, j)], (long)KA * IA)
                                    + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
}

/* ud3.F90:1173-1279 */
void og_fluxZ_XVZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, double J33G, const double *nd,
                  const double *CDZ, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double vel = (0.5 * (mom[I3(k, i, j)] + mom[I3(k, i, j + 1)])) / DEN_XVZ(k);
                flux[I3(k, i, j)] = J33G * vel * og_zface(scheme, vel, &val[I3(1, i, j)], k, KS, KE)
                                    + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
            flux[I3(KS - 1, i, j)] = 0.0;
            flux[I3(KE, i, j)] = 0.0;
        }
}

#define AVG4_XV(m, k) (0.25 * ((m)[I3(k, i, j)] + (m)[I3(k, i - 1, j)] + (m)[I3(k, i, j + 1)] + (m)[I3(k, i - 1, j + 1)]))

/* ud3.F90:1283-1374 */
void og_fluxJ13_XVZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *GSQRT, const double *J13G, const double *MAPF,
                    const double *CDZ, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double vel = (F2H(k, 1) * AVG4_XV(mom, k + 1) + F2H(k, 2) * AVG4_XV(mom, k)) / DEN_XVZ(k);
                vel = vel * J13G[I3(k, i, j)];
                flux[I3(k, i, j)] = vel / MP(MAPF, i, j, 2)
                                    * og_zface(scheme, vel, &val[I3(1, i, j)], k, KS, KE);
            }
            flux[I3(KS - 1, i, j)] = 0.0;
            flux[I3(KE, i, j)] = 0.0;
        }
}

/* ud3.F90:1378-1469 */
void og_fluxJ23_XVZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                    const double *DENS, const double *GSQRT, const double *J23G, const double *MAPF,
                    const double *CDZ, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double vel = (F2H(k, 1) * mom[I3(k + 1, i, j)] + F2H(k, 2) * mom[I3(k, i, j)]) / DEN_XVZ(k);
                vel = vel * J23G[I3(k, i, j)];
                flux[I3(k, i, j)] = vel / MP(MAPF, i, j, 1)
                                    * og_zface(scheme, vel, &val[I3(1, i, j)], k, KS, KE);
            }
            flux[I3(KS - 1, i, j)] = 0.0;
            flux[I3(KE, i, j)] = 0.0;
        }
}

/* ud3.F90:1473-1527 */
void og_fluxX_XVZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS - 1; i <= b.IIE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double vel = (0.5 * (mom[I3(k, i, j)] + mom[I3(k, i, j + 1)]))
                             / (0.25 * (DENS[I3(k, i, j)] + DENS[I3(k, i + 1, j)] + DENS[I3(k, i, j + 1)] + DENS[I3(k, i + 1, j + 1)]));
                flux[I3(k, i, j)] = GSQRT[I3(k, i, j)] / MP(MAPF, i, j, 2) * vel
                                    * og_hface(scheme, vel, &val[I3(k, i, j)], (long)KA)
                                    + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
}

/* ud3.F90:1531-1587 (y-index of the result is shifted by -1) */
void og_fluxY_XVZ(const og_dims *d, int scheme, double *flux, const double *mom, const double *val,
                  const double *DENS, const double *GSQRT, const double *MAPF, const double *nd, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE + 1; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double vel = (0.5 * (mom[I3(k, i, j)] + mom[I3(k, i, j - 1)])) / (DENS[I3(k, i, j)]);
                flux[I3(k, i, j - 1)] = GSQRT[I3(k, i, j)] / MP(MAPF, i, j, 1) * vel
                                        * og_hface(scheme, vel, &val[I3(k, i, j - 1)], (long)KA * IA)
                                        + GSQRT[I3(k, i, j)] * nd[I3(k, i, j)];
            }
}

/* ---- donor cell, scale_atmos_dyn_fvm_flux_ud1.F90:84 (F1=0.5), :135-294 ---- */
#define UD1(vel, a, b) ((vel) * (0.5 * ((b) + (a)) - og_sign(0.5, vel) * ((b) - (a))))

void og_fluxZ_XYZ_ud1(const og_dims *d, double *flux, const double *mflx, const double *val, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double vel = mflx[I3(k, i, j)];
                flux[I3(k, i, j)] = UD1(vel, val[I3(k, i, j)], val[I3(k + 1, i, j)]);
            }
            flux[I3(KS - 1, i, j)] = 0.0;
            flux[I3(KE, i, j)] = 0.0;
        }
}

void og_fluxX_XYZ_ud1(const og_dims *d, double *flux, const double *mflx, const double *val, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS; j <= b.JJE; ++j)
        for (int i = b.IIS - 1; i <= b.IIE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double vel = mflx[I3(k, i, j)];
                flux[I3(k, i, j)] = UD1(vel, val[I3(k, i, j)], val[I3(k, i + 1, j)]);
            }
}

void og_fluxY_XYZ_ud1(const og_dims *d, double *flux, const double *mflx, const double *val, og_blk b)
{
    OG_DIMS(d);
#pragma omp parallel for collapse(2)
    for (int j = b.JJS - 1; j <= b.JJE; ++j)
        for (int i = b.IIS; i <= b.IIE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double vel = mflx[I3(k, i, j)];
                flux[I3(k, i, j)] = UD1(vel, val[I3(k, i, j)], val[I3(k, i, j + 1)]);
            }
}
