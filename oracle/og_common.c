/*
 * Oracle restatement of the dynamics helpers in
 * scalelib/src/atmos-rm/dynamics/scale_atmos_dyn_common.F90:
 *   ATMOS_DYN_filter_setup (CNZ3/CNX3/CNY3, CNZ4/CNX4/CNY4) :100-330
 *   ATMOS_DYN_numfilter_coef                 :385-985
 *   calc_numdiff / calc_diff3 / calc_diff4   :1518-1918
 *   ATMOS_DYN_divergence                     :1437-1515
 *   ATMOS_DYN_fct / get_fact_fct             :1922-2734
 */
#include "og_internal.h"

/* real ** integer as gfortran lowers it (libgcc __powidf2: square-and-multiply) */
static double og_powi(double x, int m)
{
    unsigned n = m < 0 ? -(unsigned)m : (unsigned)m;
    double y = (n % 2) ? x : 1.0;
    while (n >>= 1) {
        x = x * x;
        if (n % 2) y = y * x;
    }
    return m < 0 ? 1.0 / y : y;
}

/* ---------------- filter_setup: third-order difference coefficients ---------------- */
typedef struct {
    double *CNZ3, *CNX3, *CNY3; /* (3,KA,2) (3,IA,2) (3,JA,2), 1-based */
    double *CNZ4, *CNX4, *CNY4; /* (5,KA,2) (5,IA,2) (5,JA,2) */
} cn3_t;
#define CZ3(c, n, k, s) (c).CNZ3[((n) - 1) + 3 * ((size_t)((k) - 1) + (size_t)KA * ((s) - 1))]
#define CX3(c, n, i, s) (c).CNX3[((n) - 1) + 3 * ((size_t)((i) - 1) + (size_t)IA * ((s) - 1))]
#define CY3(c, n, j, s) (c).CNY3[((n) - 1) + 3 * ((size_t)((j) - 1) + (size_t)JA * ((s) - 1))]
#define CZ4(c, n, k, s) (c).CNZ4[((n) - 1) + 5 * ((size_t)((k) - 1) + (size_t)KA * ((s) - 1))]
#define CX4(c, n, i, s) (c).CNX4[((n) - 1) + 5 * ((size_t)((i) - 1) + (size_t)IA * ((s) - 1))]
#define CY4(c, n, j, s) (c).CNY4[((n) - 1) + 5 * ((size_t)((j) - 1) + (size_t)JA * ((s) - 1))]

static int cn3_setup(const og_dims *d, cn3_t *c, const double *CDZ, const double *CDX, const double *CDY,
                     const double *FDZ, const double *FDX, const double *FDY)
{
    OG_DIMS(d);
    c->CNZ3 = og_alloc_undef(3 * (size_t)KA * 2);
    c->CNX3 = og_alloc_undef(3 * (size_t)IA * 2);
    c->CNY3 = og_alloc_undef(3 * (size_t)JA * 2);
    c->CNZ4 = og_alloc_undef(5 * (size_t)KA * 2);
    c->CNX4 = og_alloc_undef(5 * (size_t)IA * 2);
    c->CNY4 = og_alloc_undef(5 * (size_t)JA * 2);
    if (!c->CNZ3 || !c->CNX3 || !c->CNY3 || !c->CNZ4 || !c->CNX4 || !c->CNY4) return -1;
    cn3_t C = *c;
#define cdz(k) CDZ[(k) - 1]
#define fdz(k) FDZ[(k) - 1]
#define cdx(i) CDX[(i) - 1]
#define fdx(i) FDX[(i) - 1]
#define cdy(j) CDY[(j) - 1]
#define fdy(j) FDY[(j) - 1]
    /* z, :203-250 */
    for (int k = KS + 1; k <= KE - 1; ++k) {
        CZ3(C, 1, k, 1) = 1.0 / (fdz(k) * cdz(k) * fdz(k - 1));
        CZ3(C, 2, k, 1) = 1.0 / (fdz(k) * cdz(k) * fdz(k - 1)) + 1.0 / (fdz(k - 1) * cdz(k) * fdz(k - 1))
                          + 1.0 / (fdz(k - 1) * cdz(k - 1) * fdz(k - 1));
    }
    for (int k = KS + 2; k <= KE; ++k)
        CZ3(C, 3, k, 1) = 1.0 / (fdz(k - 1) * cdz(k) * fdz(k - 1)) + 1.0 / (fdz(k - 1) * cdz(k - 1) * fdz(k - 1))
                          + 1.0 / (fdz(k - 1) * cdz(k - 1) * fdz(k - 2));
    CZ3(C, 1, KS - 1, 1) = 1.0 / (fdz(KS) * cdz(KS + 1) * fdz(KS));
    CZ3(C, 1, KS, 1) = 1.0 / (fdz(KS) * cdz(KS) * fdz(KS));
    CZ3(C, 2, KS, 1) = 1.0 / (fdz(KS) * cdz(KS) * fdz(KS)) + 1.0 / (fdz(KS) * cdz(KS) * fdz(KS))
                       + 1.0 / (fdz(KS) * cdz(KS + 1) * fdz(KS));
    CZ3(C, 3, KS, 1) = 1.0 / (fdz(KS) * cdz(KS) * fdz(KS)) + 1.0 / (fdz(KS) * cdz(KS + 1) * fdz(KS))
                       + 1.0 / (fdz(KS) * cdz(KS + 1) * fdz(KS + 1));
    CZ3(C, 3, KS + 1, 1) = 1.0 / (fdz(KS) * cdz(KS + 1) * fdz(KS)) + 1.0 / (fdz(KS) * cdz(KS) * fdz(KS))
                           + 1.0 / (fdz(KS) * cdz(KS) * fdz(KS));
    CZ3(C, 1, KE, 1) = 1.0 / (fdz(KE - 1) * cdz(KE) * fdz(KE - 1));
    CZ3(C, 2, KE, 1) = 1.0 / (fdz(KE - 1) * cdz(KE) * fdz(KE - 1)) + 1.0 / (fdz(KE - 1) * cdz(KE) * fdz(KE - 1))
                       + 1.0 / (fdz(KE - 1) * cdz(KE - 1) * fdz(KE - 1));
    CZ3(C, 1, KE + 1, 1) = 1.0 / (fdz(KE - 2) * cdz(KE - 1) * fdz(KE - 1));
    CZ3(C, 2, KE + 1, 1) = 1.0 / (fdz(KE - 2) * cdz(KE - 1) * fdz(KE - 1)) + 1.0 / (fdz(KE - 1) * cdz(KE - 1) * fdz(KE - 1))
                           + 1.0 / (fdz(KE - 1) * cdz(KE) * fdz(KE - 1));
    CZ3(C, 3, KE + 1, 1) = 1.0 / (fdz(KE - 1) * cdz(KE + 1) * fdz(KE - 1)) + 1.0 / (fdz(KE - 1) * cdz(KE) * fdz(KE - 1))
                           + 1.0 / (fdz(KE - 1) * cdz(KE) * fdz(KE - 1));
    /* :259-305 */
    for (int k = KS + 1; k <= KE - 1; ++k) {
        CZ3(C, 1, k, 2) = 1.0 / (cdz(k + 1) * fdz(k) * cdz(k));
        CZ3(C, 2, k, 2) = 1.0 / (cdz(k + 1) * fdz(k) * cdz(k)) + 1.0 / (cdz(k) * fdz(k) * cdz(k))
                          + 1.0 / (cdz(k) * fdz(k - 1) * cdz(k));
        CZ3(C, 3, k, 2) = 1.0 / (cdz(k) * fdz(k) * cdz(k)) + 1.0 / (cdz(k) * fdz(k - 1) * cdz(k))
                          + 1.0 / (cdz(k) * fdz(k - 1) * cdz(k - 1));
    }
    CZ3(C, 1, KS - 1, 2) = 1.0 / (cdz(KS) * fdz(KS) * cdz(KS));
    CZ3(C, 1, KS, 2) = 1.0 / (cdz(KS + 1) * fdz(KS) * cdz(KS));
    CZ3(C, 2, KS, 2) = 1.0 / (cdz(KS + 1) * fdz(KS) * cdz(KS)) + 1.0 / (cdz(KS) * fdz(KS) * cdz(KS))
                       + 1.0 / (cdz(KS) * fdz(KS) * cdz(KS));
    CZ3(C, 3, KS, 2) = 1.0 / (cdz(KS) * fdz(KS) * cdz(KS)) + 1.0 / (cdz(KS) * fdz(KS) * cdz(KS))
                       + 1.0 / (cdz(KS) * fdz(KS) * cdz(KS + 1));
    CZ3(C, 1, KE, 2) = 1.0 / (cdz(KE - 1) * fdz(KE - 1) * cdz(KE));
    CZ3(C, 2, KE, 2) = 1.0 / (cdz(KE - 1) * fdz(KE - 1) * cdz(KE)) + 1.0 / (cdz(KE) * fdz(KE - 1) * cdz(KE))
                       + 1.0 / (cdz(KE) * fdz(KE - 1) * cdz(KE));
    CZ3(C, 3, KE, 2) = 1.0 / (cdz(KE) * fdz(KE - 1) * cdz(KE)) + 1.0 / (cdz(KE) * fdz(KE - 1) * cdz(KE))
                       + 1.0 / (cdz(KE) * fdz(KE - 1) * cdz(KE - 1));
    CZ3(C, 1, KE + 1, 2) = 1.0 / (cdz(KE - 2) * fdz(KE - 2) * cdz(KE - 1));
    CZ3(C, 2, KE + 1, 2) = 1.0 / (cdz(KE - 2) * fdz(KE - 2) * cdz(KE - 1)) + 1.0 / (cdz(KE - 1) * fdz(KE - 2) * cdz(KE - 1))
                           + 1.0 / (cdz(KE - 1) * fdz(KE - 1) * cdz(KE - 1));
    CZ3(C, 3, KE + 1, 2) = 1.0 / (cdz(KE - 1) * fdz(KE - 2) * cdz(KE - 1)) + 1.0 / (cdz(KE - 1) * fdz(KE - 1) * cdz(KE - 1))
                           + 1.0 / (cdz(KE - 1) * fdz(KE - 1) * cdz(KE));
    /* x, :318-346 */
    CX3(C, 1, IS - 1, 1) = 1.0 / (fdx(IS - 1) * cdx(IS - 1) * fdx(IS - 2));
    for (int i = IS; i <= IE + 1; ++i) {
        CX3(C, 1, i, 1) = 1.0 / (fdx(i) * cdx(i) * fdx(i - 1));
        CX3(C, 2, i, 1) = 1.0 / (fdx(i) * cdx(i) * fdx(i - 1)) + 1.0 / (fdx(i - 1) * cdx(i) * fdx(i - 1))
                          + 1.0 / (fdx(i - 1) * cdx(i - 1) * fdx(i - 1));
        CX3(C, 3, i, 1) = 1.0 / (fdx(i - 1) * cdx(i) * fdx(i - 1)) + 1.0 / (fdx(i - 1) * cdx(i - 1) * fdx(i - 1))
                          + 1.0 / (fdx(i - 1) * cdx(i - 1) * fdx(i - 2));
    }
    for (int i = IS - 1; i <= IE + 1; ++i) {
        CX3(C, 1, i, 2) = 1.0 / (cdx(i + 1) * fdx(i) * cdx(i));
        CX3(C, 2, i, 2) = 1.0 / (cdx(i + 1) * fdx(i) * cdx(i)) + 1.0 / (cdx(i) * fdx(i) * cdx(i))
                          + 1.0 / (cdx(i) * fdx(i - 1) * cdx(i));
        CX3(C, 3, i, 2) = 1.0 / (cdx(i) * fdx(i) * cdx(i)) + 1.0 / (cdx(i) * fdx(i - 1) * cdx(i))
                          + 1.0 / (cdx(i) * fdx(i - 1) * cdx(i - 1));
    }
    /* y */
    CY3(C, 1, JS - 1, 1) = 1.0 / (fdy(JS - 1) * cdy(JS - 1) * fdy(JS - 2));
    for (int j = JS; j <= JE + 1; ++j) {
        CY3(C, 1, j, 1) = 1.0 / (fdy(j) * cdy(j) * fdy(j - 1));
        CY3(C, 2, j, 1) = 1.0 / (fdy(j) * cdy(j) * fdy(j - 1)) + 1.0 / (fdy(j - 1) * cdy(j) * fdy(j - 1))
                          + 1.0 / (fdy(j - 1) * cdy(j - 1) * fdy(j - 1));
        CY3(C, 3, j, 1) = 1.0 / (fdy(j - 1) * cdy(j) * fdy(j - 1)) + 1.0 / (fdy(j - 1) * cdy(j - 1) * fdy(j - 1))
                          + 1.0 / (fdy(j - 1) * cdy(j - 1) * fdy(j - 2));
    }
    for (int j = JS - 1; j <= JE + 1; ++j) {
        CY3(C, 1, j, 2) = 1.0 / (cdy(j + 1) * fdy(j) * cdy(j));
        CY3(C, 2, j, 2) = 1.0 / (cdy(j + 1) * fdy(j) * cdy(j)) + 1.0 / (cdy(j) * fdy(j) * cdy(j))
                          + 1.0 / (cdy(j) * fdy(j - 1) * cdy(j));
        CY3(C, 3, j, 2) = 1.0 / (cdy(j) * fdy(j) * cdy(j)) + 1.0 / (cdy(j) * fdy(j - 1) * cdy(j))
                          + 1.0 / (cdy(j) * fdy(j - 1) * cdy(j - 1));
    }
    /* fourth-order coefficients (:186-193, :253-263, :281-297, :309-317): the
     * second kind of z, x and y divides by FDZ/FDX/FDY, the first by CDZ/CDX/CDY */
    for (int s = 1; s <= 2; ++s)
        for (int k = KS; k <= KE - 1; ++k) {
            const double den = s == 1 ? cdz(k) : fdz(k);
            CZ4(C, 1, k, s) = (CZ3(C, 1, k + 1, s)) / den;
            CZ4(C, 2, k, s) = (CZ3(C, 2, k + 1, s) + CZ3(C, 1, k, s)) / den;
            CZ4(C, 3, k, s) = (CZ3(C, 3, k + 1, s) + CZ3(C, 2, k, s)) / den;
            CZ4(C, 4, k, s) = (CZ3(C, 1, k, s) + CZ3(C, 3, k, s)) / den;
            CZ4(C, 5, k, s) = (CZ3(C, 1, k - 1, s)) / den;
        }
    for (int s = 1; s <= 2; ++s)
        for (int i = IS; i <= IE; ++i) {
            const double den = s == 1 ? cdx(i) : fdx(i);
            CX4(C, 1, i, s) = (CX3(C, 1, i + 1, s)) / den;
            CX4(C, 2, i, s) = (CX3(C, 2, i + 1, s) + CX3(C, 1, i, s)) / den;
            CX4(C, 3, i, s) = (CX3(C, 3, i + 1, s) + CX3(C, 2, i, s)) / den;
            CX4(C, 4, i, s) = (CX3(C, 1, i, s) + CX3(C, 3, i, s)) / den;
            CX4(C, 5, i, s) = (CX3(C, 1, i - 1, s)) / den;
        }
    for (int s = 1; s <= 2; ++s)
        for (int j = JS; j <= JE; ++j) {
            const double den = s == 1 ? cdy(j) : fdy(j);
            CY4(C, 1, j, s) = (CY3(C, 1, j + 1, s)) / den;
            CY4(C, 2, j, s) = (CY3(C, 2, j + 1, s) + CY3(C, 1, j, s)) / den;
            CY4(C, 3, j, s) = (CY3(C, 3, j + 1, s) + CY3(C, 2, j, s)) / den;
            CY4(C, 4, j, s) = (CY3(C, 1, j, s) + CY3(C, 3, j, s)) / den;
            CY4(C, 5, j, s) = (CY3(C, 1, j - 1, s)) / den;
        }
#undef cdz
#undef fdz
#undef cdx
#undef fdx
#undef cdy
#undef fdy
    return 0;
}
static void cn3_free(cn3_t *c)
{
    free(c->CNZ3); free(c->CNX3); free(c->CNY3);
    free(c->CNZ4); free(c->CNX4); free(c->CNY4);
}

/* calc_diff3, :1600-1760; diff is (KA,IA,JA,3) */
static void calc_diff3(const og_dims *d, const cn3_t *c, double *diff, const double *phi, int KO, int IO, int JO)
{
    OG_DIMS(d);
    const cn3_t C = *c;
    double *dZ = diff, *dX = diff + N3, *dY = diff + 2 * N3;
    const int KEE = KE - KO;
    if (KO == 0) {
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i)
                for (int k = KS + 1; k <= KE - 2; ++k)
                    dZ[I3(k, i, j)] = (+CZ3(C, 1, k + 1, 1) * phi[I3(k + 2, i, j)] - CZ3(C, 2, k + 1, 1) * phi[I3(k + 1, i, j)]
                                       + CZ3(C, 3, k + 1, 1) * phi[I3(k, i, j)] - CZ3(C, 1, k, 1) * phi[I3(k - 1, i, j)]);
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i) {
                dZ[I3(KS, i, j)] = (+CZ3(C, 1, KS + 1, 1) * phi[I3(KS + 2, i, j)] - CZ3(C, 2, KS + 1, 1) * phi[I3(KS + 1, i, j)]
                                    + CZ3(C, 3, KS + 1, 1) * phi[I3(KS, i, j)] - CZ3(C, 1, KS, 1) * phi[I3(KS + 1, i, j)]);
                dZ[I3(KS - 1, i, j)] = -dZ[I3(KS, i, j)];
                dZ[I3(KS - 2, i, j)] = -dZ[I3(KS + 1, i, j)];
                dZ[I3(KE - 1, i, j)] = (+CZ3(C, 1, KE, 1) * phi[I3(KE - 1, i, j)] - CZ3(C, 2, KE, 1) * phi[I3(KE, i, j)]
                                        + CZ3(C, 3, KE, 1) * phi[I3(KE - 1, i, j)] - CZ3(C, 1, KE - 1, 1) * phi[I3(KE - 2, i, j)]);
                dZ[I3(KE, i, j)] = -dZ[I3(KE - 1, i, j)];
                dZ[I3(KE + 1, i, j)] = -dZ[I3(KE - 2, i, j)];
                dZ[I3(KE + 2, i, j)] = 0.0;
            }
    } else {
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i)
                for (int k = KS + 2; k <= KE - 2; ++k)
                    dZ[I3(k, i, j)] = (+CZ3(C, 1, k, 2) * phi[I3(k + 1, i, j)] - CZ3(C, 2, k, 2) * phi[I3(k, i, j)]
                                       + CZ3(C, 3, k, 2) * phi[I3(k - 1, i, j)] - CZ3(C, 1, k - 1, 2) * phi[I3(k - 2, i, j)]);
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i) {
                dZ[I3(KS + 1, i, j)] = (+CZ3(C, 1, KS + 1, 2) * phi[I3(KS + 2, i, j)] - CZ3(C, 2, KS + 1, 2) * phi[I3(KS + 1, i, j)]
                                        + CZ3(C, 3, KS + 1, 2) * phi[I3(KS, i, j)] - CZ3(C, 1, KS, 2) * phi[I3(KS + 1, i, j)]);
                dZ[I3(KS, i, j)] = -dZ[I3(KS + 1, i, j)];
                dZ[I3(KS - 1, i, j)] = -dZ[I3(KS + 2, i, j)];
                dZ[I3(KS - 2, i, j)] = -dZ[I3(KS + 3, i, j)];
                dZ[I3(KE - 1, i, j)] = (-CZ3(C, 2, KE - 1, 2) * phi[I3(KE - 1, i, j)] + CZ3(C, 3, KE - 1, 2) * phi[I3(KE - 2, i, j)]
                                        - CZ3(C, 1, KE - 2, 2) * phi[I3(KE - 3, i, j)]);
                dZ[I3(KE, i, j)] = (+CZ3(C, 1, KE, 2) * phi[I3(KE - 1, i, j)] + CZ3(C, 3, KE, 2) * phi[I3(KE - 1, i, j)]
                                    - CZ3(C, 1, KE - 1, 2) * phi[I3(KE - 2, i, j)]);
                dZ[I3(KE + 1, i, j)] = -dZ[I3(KE, i, j)];
                dZ[I3(KE + 2, i, j)] = -dZ[I3(KE - 1, i, j)];
            }
    }
#pragma omp parallel for collapse(2)
    for (int j = JS; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i) {
            for (int k = KS; k <= KEE; ++k) {
                if (IO == 0)
                    dX[I3(k, i, j)] = (+CX3(C, 1, i + 1, 1) * phi[I3(k, i + 2, j)] - CX3(C, 2, i + 1, 1) * phi[I3(k, i + 1, j)]
                                       + CX3(C, 3, i + 1, 1) * phi[I3(k, i, j)] - CX3(C, 1, i, 1) * phi[I3(k, i - 1, j)]);
                else
                    dX[I3(k, i, j)] = (+CX3(C, 1, i, 2) * phi[I3(k, i + 1, j)] - CX3(C, 2, i, 2) * phi[I3(k, i, j)]
                                       + CX3(C, 3, i, 2) * phi[I3(k, i - 1, j)] - CX3(C, 1, i - 1, 2) * phi[I3(k, i - 2, j)]);
            }
            for (int k = 1; k <= KS - 1; ++k) dX[I3(k, i, j)] = 0.0;
            for (int k = KE + 1; k <= KA; ++k) dX[I3(k, i, j)] = 0.0;
        }
#pragma omp parallel for collapse(2)
    for (int j = JS; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i) {
            for (int k = KS; k <= KEE; ++k) {
                if (JO == 0)
                    dY[I3(k, i, j)] = (+CY3(C, 1, j + 1, 1) * phi[I3(k, i, j + 2)] - CY3(C, 2, j + 1, 1) * phi[I3(k, i, j + 1)]
                                       + CY3(C, 3, j + 1, 1) * phi[I3(k, i, j)] - CY3(C, 1, j, 1) * phi[I3(k, i, j - 1)]);
                else
                    dY[I3(k, i, j)] = (+CY3(C, 1, j, 2) * phi[I3(k, i, j + 1)] - CY3(C, 2, j, 2) * phi[I3(k, i, j)]
                                       + CY3(C, 3, j, 2) * phi[I3(k, i, j - 1)] - CY3(C, 1, j - 1, 2) * phi[I3(k, i, j - 2)]);
            }
            for (int k = 1; k <= KS - 1; ++k) dY[I3(k, i, j)] = 0.0;
            for (int k = KE + 1; k <= KA; ++k) dY[I3(k, i, j)] = 0.0;
        }
}

/* calc_diff4, :1810-1918: out = fourth difference of in, z on KS..KE-1 with the
 * mirrored levels KS-1, KS-2, KE, KE+1, x and y on KS..K1; interior columns */
static void calc_diff4(const og_dims *d, const cn3_t *c, double *out, const double *in, int KO, int IO, int JO, int K1)
{
    OG_DIMS(d);
    const cn3_t C = *c;
    double *oZ = out, *oX = out + N3, *oY = out + 2 * N3;
    const double *iZ = in, *iX = in + N3, *iY = in + 2 * N3;
    const int sz = 1 + KO, sx = 1 + IO, sy = 1 + JO;
#pragma omp parallel for collapse(2)
    for (int j = JS; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i) {
            for (int k = KS; k <= KE - 1; ++k)
                oZ[I3(k, i, j)] = (CZ4(C, 1, k, sz) * iZ[I3(k + 2, i, j)] - CZ4(C, 2, k, sz) * iZ[I3(k + 1, i, j)]
                                   + CZ4(C, 3, k, sz) * iZ[I3(k, i, j)] - CZ4(C, 4, k, sz) * iZ[I3(k - 1, i, j)]
                                   + CZ4(C, 5, k, sz) * iZ[I3(k - 2, i, j)]);
            oZ[I3(KS - 1, i, j)] = -oZ[I3(KS, i, j)];
            oZ[I3(KS - 2, i, j)] = -oZ[I3(KS + 1, i, j)];
            oZ[I3(KE, i, j)] = -oZ[I3(KE - 1, i, j)];
            oZ[I3(KE + 1, i, j)] = -oZ[I3(KE - 2, i, j)];
            for (int k = KS; k <= K1; ++k) {
                oX[I3(k, i, j)] = (CX4(C, 1, i, sx) * iX[I3(k, i + 2, j)] - CX4(C, 2, i, sx) * iX[I3(k, i + 1, j)]
                                   + CX4(C, 3, i, sx) * iX[I3(k, i, j)] - CX4(C, 4, i, sx) * iX[I3(k, i - 1, j)]
                                   + CX4(C, 5, i, sx) * iX[I3(k, i - 2, j)]);
                oY[I3(k, i, j)] = (CY4(C, 1, j, sy) * iY[I3(k, i, j + 2)] - CY4(C, 2, j, sy) * iY[I3(k, i, j + 1)]
                                   + CY4(C, 3, j, sy) * iY[I3(k, i, j)] - CY4(C, 4, j, sy) * iY[I3(k, i, j - 1)]
                                   + CY4(C, 5, j, sy) * iY[I3(k, i, j - 2)]);
            }
        }
}

/* calc_numdiff, :1518-1573: calc_diff3, then nd_order-1 times the periodic halo
 * of the three components (COMM_vars8, one rank) and calc_diff4. Returns the
 * buffer (w1 or w2) that holds the result. */
static double *calc_numdiff(const og_dims *d, const cn3_t *c, double *w1, double *w2, const double *data, int nd_order,
                            int KO, int IO, int JO)
{
    calc_diff3(d, c, w1, data, KO, IO, JO);
    double *in = w1, *out = w2;
    for (int no = 2; no <= nd_order; ++no) {
        og_halo_periodic(d, in, 3);
        calc_diff4(d, c, out, in, KO, IO, JO, d->KE - KO);
        double *t = in;
        in = out;
        out = t;
    }
    return in;
}

/* numfilter_coef, :385-985, for any ND_ORDER >= 1. */
int og_numfilter_coef(
    const og_dims *d, double *num_diff,
    const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY, const double *RHOT,
    const double *CDZ, const double *CDX, const double *CDY,
    const double *FDZ, const double *FDX, const double *FDY, double DT,
    const double *REF_dens, const double *REF_pott,
    double ND_COEF, int ND_ORDER, double ND_SFC_FACT, int ND_USE_RS)
{
    OG_DIMS(d);
    if (ND_ORDER < 1) return -2;
    cn3_t cn;
    if (cn3_setup(d, &cn, CDZ, CDX, CDY, FDZ, FDX, FDY)) { cn3_free(&cn); return -1; }
    double *work = og_alloc_undef(3 * N3), *work2 = og_alloc_undef(3 * N3), *tmp = og_alloc_undef(N3),
           *tmp2 = og_alloc_undef(N3);
    double *ncz = og_alloc_undef(KA), *nfz = og_alloc_undef(KA), *ncx = og_alloc_undef(IA), *nfx = og_alloc_undef(IA);
    double *ncy = og_alloc_undef(JA), *nfy = og_alloc_undef(JA);
    if (!work || !work2 || !tmp || !tmp2 || !ncz || !nfz || !ncx || !nfx || !ncy || !nfy) {
        free(work); free(work2); free(tmp); free(tmp2); free(ncz); free(nfz); free(ncx); free(nfx); free(ncy); free(nfy);
        cn3_free(&cn);
        return -1;
    }
    const int nd_order4 = ND_ORDER * 4;
    const double DIFF4 = ND_COEF / ((double)og_powi(2.0, nd_order4) * DT);
    for (int k = KS - 1; k <= KE; ++k) ncz[k - 1] = DIFF4 * og_powi(CDZ[k - 1], nd_order4);
    for (int k = KS + 1; k <= KE - 1; ++k) nfz[k - 1] = DIFF4 * og_powi(FDZ[k - 1], nd_order4);
    for (int i = IS; i <= IE; ++i) {
        ncx[i - 1] = DIFF4 * og_powi(CDX[i - 1], nd_order4);
        nfx[i - 1] = DIFF4 * og_powi(FDX[i - 1], nd_order4);
    }
    for (int j = JS; j <= JE; ++j) {
        ncy[j - 1] = DIFF4 * og_powi(CDY[j - 1], nd_order4);
        nfy[j - 1] = DIFF4 * og_powi(FDY[j - 1], nd_order4);
    }
    double *wZ = work, *wX = work + N3, *wY = work + 2 * N3, *wres = work;
#define NUMDIFF(data, KO, IO, JO)                                                    \
    do {                                                                             \
        wres = calc_numdiff(d, &cn, work, work2, (data), ND_ORDER, (KO), (IO), (JO)); \
        wZ = wres; wX = wres + N3; wY = wres + 2 * N3;                               \
    } while (0)
#define NDF(v, dir) ND(num_diff, v, dir)
    /* lateral zeroing and surface factors shared by the x/y components */
#define SFC_TAIL(nd, kzero_top)                                                   \
    do {                                                                          \
        for (int k = 1; k <= KS - 1; ++k) (nd)[I3(k, i, j)] = 0.0;                \
        (nd)[I3(KS, i, j)] = (nd)[I3(KS, i, j)] * ND_SFC_FACT;                    \
        (nd)[I3(KS + 1, i, j)] = (nd)[I3(KS + 1, i, j)] * (1.0 + ND_SFC_FACT) * 0.5; \
        for (int k = (kzero_top); k <= KA; ++k) (nd)[I3(k, i, j)] = 0.0;          \
    } while (0)

    double *dens_diff = tmp, *pott_diff = tmp2;
    if (!ND_USE_RS) {
        /* :466-530 (19-point smoothed anomalies) */
        double *POTT = og_alloc_undef(N3);
        for (int j = JS - 2; j <= JE + 2; ++j)
            for (int i = IS - 2; i <= IE + 2; ++i)
                for (int k = KS; k <= KE; ++k) POTT[I3(k, i, j)] = RHOT[I3(k, i, j)] / DENS[I3(k, i, j)];
        const double *F[2] = {DENS, POTT};
        double *O[2] = {dens_diff, pott_diff};
        for (int v = 0; v < 2; ++v) {
            const double *f = F[v];
            double *o = O[v];
#pragma omp parallel for collapse(2)
            for (int j = JS; j <= JE; ++j)
                for (int i = IS; i <= IE; ++i) {
                    for (int k = KS + 1; k <= KE - 1; ++k)
                        o[I3(k, i, j)] = ((f[I3(k, i, j)]) * 3.0
                                          + (f[I3(k, i + 1, j)] + f[I3(k, i - 1, j)] + f[I3(k, i, j + 1)] + f[I3(k, i, j - 1)]) * 2.0
                                          + (f[I3(k, i + 2, j)] + f[I3(k, i - 2, j)] + f[I3(k, i, j + 2)] + f[I3(k, i, j - 2)])
                                          + (f[I3(k + 1, i, j)] + f[I3(k - 1, i, j)]) * 2.0) / 19.0;
                    o[I3(KS, i, j)] = ((f[I3(KS, i, j)]) * 3.0
                                       + (f[I3(KS, i + 1, j)] + f[I3(KS, i - 1, j)] + f[I3(KS, i, j + 1)] + f[I3(KS, i, j - 1)]) * 2.0
                                       + (f[I3(KS, i + 2, j)] + f[I3(KS, i - 2, j)] + f[I3(KS, i, j + 2)] + f[I3(KS, i, j - 2)])
                                       + (f[I3(KS + 1, i, j)]) * 2.0) / 17.0;
                    o[I3(KE, i, j)] = ((f[I3(KE, i, j)]) * 3.0
                                       + (f[I3(KE, i + 1, j)] + f[I3(KE, i - 1, j)] + f[I3(KE, i, j + 1)] + f[I3(KE, i, j - 1)]) * 2.0
                                       + (f[I3(KE, i + 2, j)] + f[I3(KE, i - 2, j)] + f[I3(KE, i, j + 2)] + f[I3(KE, i, j - 2)])
                                       + (f[I3(KE - 1, i, j)]) * 2.0) / 17.0;
                }
            og_halo_periodic(d, o, 1);
        }
        free(POTT);
    } else {
        /* :538-550 */
#pragma omp parallel for collapse(2)
        for (int j = JS - 1; j <= JE + 2; ++j)
            for (int i = IS - 1; i <= IE + 2; ++i)
                for (int k = KS; k <= KE; ++k) dens_diff[I3(k, i, j)] = DENS[I3(k, i, j)] - REF_dens[I3(k, i, j)];
    }

    /* ---- density :552-610 ---- */
    NUMDIFF(dens_diff, 0, 0, 0);
    {
        double *nz = NDF(I_DENS, ZDIR), *nx = NDF(I_DENS, XDIR), *ny = NDF(I_DENS, YDIR);
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i) {
                for (int k = KS - 1; k <= KE; ++k) nz[I3(k, i, j)] = wZ[I3(k, i, j)] * ncz[k - 1];
                for (int k = 1; k <= KS - 2; ++k) nz[I3(k, i, j)] = 0.0;
                for (int k = KE + 1; k <= KA; ++k) nz[I3(k, i, j)] = 0.0;
                for (int k = KS; k <= KE; ++k) nx[I3(k, i, j)] = wX[I3(k, i, j)] * ncx[i - 1];
                SFC_TAIL(nx, KE + 1);
                for (int k = KS; k <= KE; ++k) ny[I3(k, i, j)] = wY[I3(k, i, j)] * ncy[j - 1];
                SFC_TAIL(ny, KE + 1);
            }
        og_halo_periodic(d, nz, 1); og_halo_periodic(d, nx, 1); og_halo_periodic(d, ny, 1);
    }

    /* ---- z-momentum :613-700 ---- */
    {
        double *VELZ = tmp;
#pragma omp parallel for collapse(2)
        for (int j = JS - 2; j <= JE + 2; ++j)
            for (int i = IS - 2; i <= IE + 2; ++i)
                for (int k = KS; k <= KE - 1; ++k)
                    VELZ[I3(k, i, j)] = 2.0 * MOMZ[I3(k, i, j)] / (DENS[I3(k + 1, i, j)] + DENS[I3(k, i, j)]);
        NUMDIFF(VELZ, 1, 0, 0);
        double *nz = NDF(I_MOMZ, ZDIR), *nx = NDF(I_MOMZ, XDIR), *ny = NDF(I_MOMZ, YDIR);
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i) {
                for (int k = KS + 1; k <= KE - 1; ++k) nz[I3(k, i, j)] = wZ[I3(k, i, j)] * nfz[k - 1] * DENS[I3(k, i, j)];
                for (int k = 1; k <= KS; ++k) nz[I3(k, i, j)] = 0.0;
                for (int k = KE; k <= KA; ++k) nz[I3(k, i, j)] = 0.0;
                for (int k = KS; k <= KE - 1; ++k)
                    nx[I3(k, i, j)] = wX[I3(k, i, j)] * ncx[i - 1]
                                      * 0.25 * (DENS[I3(k + 1, i + 1, j)] + DENS[I3(k + 1, i, j)] + DENS[I3(k, i + 1, j)] + DENS[I3(k, i, j)]);
                SFC_TAIL(nx, KE);
                for (int k = KS; k <= KE - 1; ++k)
                    ny[I3(k, i, j)] = wY[I3(k, i, j)] * ncy[j - 1]
                                      * 0.25 * (DENS[I3(k + 1, i, j + 1)] + DENS[I3(k + 1, i, j)] + DENS[I3(k, i, j + 1)] + DENS[I3(k, i, j)]);
                SFC_TAIL(ny, KE);
            }
        og_halo_periodic(d, nz, 1); og_halo_periodic(d, nx, 1); og_halo_periodic(d, ny, 1);
    }

    /* ---- x-momentum :710-790 ---- */
    {
        double *VELX = tmp;
#pragma omp parallel for collapse(2)
        for (int j = JS - 2; j <= JE + 2; ++j)
            for (int i = IS - 2; i <= IE + 1; ++i)
                for (int k = KS; k <= KE; ++k)
                    VELX[I3(k, i, j)] = 2.0 * MOMX[I3(k, i, j)] / (DENS[I3(k, i + 1, j)] + DENS[I3(k, i, j)]);
        NUMDIFF(VELX, 0, 1, 0);
        double *nz = NDF(I_MOMX, ZDIR), *nx = NDF(I_MOMX, XDIR), *ny = NDF(I_MOMX, YDIR);
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i) {
                for (int k = KS; k <= KE - 1; ++k)
                    nz[I3(k, i, j)] = wZ[I3(k, i, j)] * ncz[k - 1]
                                      * 0.25 * (DENS[I3(k + 1, i + 1, j)] + DENS[I3(k + 1, i, j)] + DENS[I3(k, i + 1, j)] + DENS[I3(k, i, j)]);
                for (int k = 1; k <= KS - 1; ++k) nz[I3(k, i, j)] = 0.0;
                for (int k = KE; k <= KA; ++k) nz[I3(k, i, j)] = 0.0;
                for (int k = KS; k <= KE; ++k) nx[I3(k, i, j)] = wX[I3(k, i, j)] * nfx[i - 1] * DENS[I3(k, i, j)];
                SFC_TAIL(nx, KE + 1);
                for (int k = KS; k <= KE; ++k)
                    ny[I3(k, i, j)] = wY[I3(k, i, j)] * ncy[j - 1]
                                      * 0.25 * (DENS[I3(k, i + 1, j + 1)] + DENS[I3(k, i + 1, j)] + DENS[I3(k, i, j + 1)] + DENS[I3(k, i, j)]);
                SFC_TAIL(ny, KE + 1);
            }
        og_halo_periodic(d, nz, 1); og_halo_periodic(d, nx, 1); og_halo_periodic(d, ny, 1);
    }

    /* ---- y-momentum :793-870 ---- */
    {
        double *VELY = tmp;
#pragma omp parallel for collapse(2)
        for (int j = JS - 2; j <= JE + 1; ++j)
            for (int i = IS - 2; i <= IE + 2; ++i)
                for (int k = KS; k <= KE; ++k)
                    VELY[I3(k, i, j)] = 2.0 * MOMY[I3(k, i, j)] / (DENS[I3(k, i, j + 1)] + DENS[I3(k, i, j)]);
        NUMDIFF(VELY, 0, 0, 1);
        double *nz = NDF(I_MOMY, ZDIR), *nx = NDF(I_MOMY, XDIR), *ny = NDF(I_MOMY, YDIR);
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i) {
                for (int k = KS; k <= KE - 1; ++k)
                    nz[I3(k, i, j)] = wZ[I3(k, i, j)] * ncz[k - 1]
                                      * 0.25 * (DENS[I3(k + 1, i, j + 1)] + DENS[I3(k + 1, i, j)] + DENS[I3(k, i, j + 1)] + DENS[I3(k, i, j)]);
                for (int k = 1; k <= KS - 1; ++k) nz[I3(k, i, j)] = 0.0;
                for (int k = KE; k <= KA; ++k) nz[I3(k, i, j)] = 0.0;
                for (int k = KS; k <= KE; ++k)
                    nx[I3(k, i, j)] = wX[I3(k, i, j)] * ncx[i - 1]
                                      * 0.25 * (DENS[I3(k, i + 1, j + 1)] + DENS[I3(k, i, j + 1)] + DENS[I3(k, i + 1, j)] + DENS[I3(k, i, j)]);
                SFC_TAIL(nx, KE + 1);
                for (int k = KS; k <= KE; ++k) ny[I3(k, i, j)] = wY[I3(k, i, j)] * nfy[j - 1] * DENS[I3(k, i, j)];
                SFC_TAIL(ny, KE + 1);
            }
        og_halo_periodic(d, nz, 1); og_halo_periodic(d, nx, 1); og_halo_periodic(d, ny, 1);
    }

    /* ---- rho*theta :873-960 ---- */
    if (ND_USE_RS) {
#pragma omp parallel for collapse(2)
        for (int j = JS - 1; j <= JE + 2; ++j)
            for (int i = IS - 1; i <= IE + 2; ++i)
                for (int k = KS; k <= KE; ++k)
                    pott_diff[I3(k, i, j)] = RHOT[I3(k, i, j)] / DENS[I3(k, i, j)] - REF_pott[I3(k, i, j)];
    }
    NUMDIFF(pott_diff, 0, 0, 0);
    {
        double *nz = NDF(I_RHOT, ZDIR), *nx = NDF(I_RHOT, XDIR), *ny = NDF(I_RHOT, YDIR);
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i) {
                for (int k = KS; k <= KE - 1; ++k)
                    nz[I3(k, i, j)] = wZ[I3(k, i, j)] * ncz[k - 1] * 0.5 * (DENS[I3(k + 1, i, j)] + DENS[I3(k, i, j)]);
                for (int k = 1; k <= KS - 2; ++k) nz[I3(k, i, j)] = 0.0;
                nz[I3(KS - 1, i, j)] = wZ[I3(KS - 1, i, j)] * ncz[KS - 2] * DENS[I3(KS, i, j)];
                nz[I3(KE, i, j)] = wZ[I3(KE, i, j)] * ncz[KE - 1] * DENS[I3(KE, i, j)];
                for (int k = KE + 1; k <= KA; ++k) nz[I3(k, i, j)] = 0.0;
                for (int k = KS; k <= KE; ++k)
                    nx[I3(k, i, j)] = wX[I3(k, i, j)] * ncx[i - 1] * 0.5 * (DENS[I3(k, i + 1, j)] + DENS[I3(k, i, j)]);
                SFC_TAIL(nx, KE + 1);
                for (int k = KS; k <= KE; ++k)
                    ny[I3(k, i, j)] = wY[I3(k, i, j)] * ncy[j - 1] * 0.5 * (DENS[I3(k, i, j + 1)] + DENS[I3(k, i, j)]);
                SFC_TAIL(ny, KE + 1);
            }
        og_halo_periodic(d, nz, 1); og_halo_periodic(d, nx, 1); og_halo_periodic(d, ny, 1);
    }
#undef SFC_TAIL
#undef NDF
#undef NUMDIFF
    (void)wres;
    free(work); free(work2); free(tmp); free(tmp2); free(ncz); free(nfz); free(ncx); free(nfx); free(ncy); free(nfy);
    cn3_free(&cn);
    return 0;
}

/* ATMOS_DYN_divergence, :1437-1515 */
void og_divergence(
    const og_dims *d, double *DDIV,
    const double *MOMZ, const double *MOMX, const double *MOMY,
    const double *GSQRT, const double *J13G, const double *J23G, double J33G, const double *MAPF,
    const double *RCDZ, const double *RCDX, const double *RCDY, const double *RFDZ, const double *FDZ)
{
    OG_DIMS(d);
#define GS_(k, i, j, idx) GSQRT[I3(k, i, j) + ((size_t)(idx) - 1) * N3]
#define J13_(k, i, j) J13G[I3(k, i, j) + ((size_t)I_XYW - 1) * N3]
#define J23_(k, i, j) J23G[I3(k, i, j) + ((size_t)I_XYW - 1) * N3]
#define MF(i, j, a, b) MAPF[I2(i, j) + (size_t)IA * (size_t)JA * ((size_t)((a) - 1) + 2 * (size_t)((b) - 1))]
#pragma omp parallel for collapse(2)
    for (int j = JS; j <= JE + 1; ++j)
        for (int i = IS; i <= IE + 1; ++i)
            for (int k = KS - 1; k <= KE + 1; ++k)
                DDIV[I3(k, i, j)] = J33G * (MOMZ[I3(k, i, j)] - MOMZ[I3(k - 1, i, j)]) * RCDZ[k - 1]
                                    + ((MOMX[I3(k + 1, i, j)] + MOMX[I3(k + 1, i - 1, j)]) * J13_(k + 1, i, j)
                                       - (MOMX[I3(k - 1, i, j)] + MOMX[I3(k - 1, i - 1, j)]) * J13_(k - 1, i, j)
                                       + (MOMY[I3(k + 1, i, j)] + MOMY[I3(k + 1, i, j - 1)]) * J23_(k + 1, i, j)
                                       - (MOMY[I3(k - 1, i, j)] + MOMY[I3(k - 1, i, j - 1)]) * J23_(k - 1, i, j)) / (FDZ[k - 1] + FDZ[k - 2])
                                    + MF(i, j, 1, I_XY) * MF(i, j, 2, I_XY)
                                      * ((MOMX[I3(k, i, j)] * GS_(k, i, j, I_UYZ) / MF(i, j, 2, I_UY)
                                          - MOMX[I3(k, i - 1, j)] * GS_(k, i - 1, j, I_UYZ) / MF(i - 1, j, 2, I_UY)) * RCDX[i - 1]
                                         + (MOMY[I3(k, i, j)] * GS_(k, i, j, I_XVZ) / MF(i, j, 1, I_XV)
                                            - MOMY[I3(k, i, j - 1)] * GS_(k, i, j - 1, I_XVZ) / MF(i, j - 1, 1, I_XV)) * RCDY[j - 1]);
#pragma omp parallel for collapse(2)
    for (int j = JS; j <= JE + 1; ++j)
        for (int i = IS; i <= IE + 1; ++i) {
            DDIV[I3(KS, i, j)] = J33G * (MOMZ[I3(KS, i, j)]) * RCDZ[KS - 1]
                                 + ((MOMX[I3(KS + 1, i, j)] + MOMX[I3(KS + 1, i - 1, j)]) * J13_(KS + 1, i, j)
                                    - (MOMX[I3(KS - 1, i, j)] + MOMX[I3(KS, i - 1, j)]) * J13_(KS, i, j)
                                    + (MOMY[I3(KS + 1, i, j)] + MOMY[I3(KS + 1, i, j - 1)]) * J23_(KS + 1, i, j)
                                    - (MOMY[I3(KS, i, j)] + MOMY[I3(KS, i, j - 1)]) * J23_(KS, i, j)) * RFDZ[KS - 1]
                                 + MF(i, j, 1, I_XY) * MF(i, j, 2, I_XY)
                                   * ((MOMX[I3(KS, i, j)] * GS_(KS, i, j, I_UYZ) / MF(i, j, 2, I_UY)
                                       - MOMX[I3(KS, i - 1, j)] * GS_(KS, i - 1, j, I_UYZ) / MF(i - 1, j, 2, I_UY)) * RCDX[i - 1]
                                      + (MOMY[I3(KS, i, j)] * GS_(KS, i, j, I_XVZ) / MF(i, j, 1, I_XV)
                                         - MOMY[I3(KS, i, j - 1)] * GS_(KS, i, j - 1, I_XVZ) / MF(i, j - 1, 1, I_XV)) * RCDY[j - 1]);
            DDIV[I3(KE, i, j)] = J33G * (-MOMZ[I3(KE - 1, i, j)]) * RCDZ[KE - 1]
                                 + ((MOMX[I3(KE, i, j)] + MOMX[I3(KE, i - 1, j)]) * J13_(KE, i, j)
                                    - (MOMX[I3(KE - 1, i, j)] + MOMX[I3(KE - 1, i - 1, j)]) * J13_(KE - 1, i, j)
                                    + (MOMY[I3(KE, i, j)] + MOMY[I3(KE, i, j - 1)]) * J23_(KE, i, j)
                                    - (MOMY[I3(KE - 1, i, j)] + MOMY[I3(KE - 1, i, j - 1)]) * J23_(KE - 1, i, j)) * RFDZ[KE - 1]
                                 + MF(i, j, 1, I_XY) * MF(i, j, 2, I_XY)
                                   * ((MOMX[I3(KE, i, j)] * GS_(KE, i, j, I_UYZ) / MF(i, j, 2, I_UY)
                                       - MOMX[I3(KE, i - 1, j)] * GS_(KE, i - 1, j, I_UYZ) / MF(i - 1, j, 2, I_UY)) * RCDX[i - 1]
                                      + (MOMY[I3(KE, i, j)] * GS_(KE, i, j, I_XVZ) / MF(i, j, 1, I_XV)
                                         - MOMY[I3(KE, i, j - 1)] * GS_(KE, i, j - 1, I_XVZ) / MF(i, j - 1, 1, I_XV)) * RCDY[j - 1]);
        }
#undef GS_
#undef J13_
#undef J23_
#undef MF
}

/* get_fact_fct, :2676-2734. fact(0:1,-1:1,-1:1) stored as f[a][b+1][c+1] */
static void get_fact_fct(double f[2][3][3], double rw, double ru, double rv)
{
    const double EPSILON = OG_EPS;
    double ugev = og_sign(0.5, fabs(ru) - fabs(rv)) + 0.5;
    double ugew = og_sign(0.5, fabs(ru) - fabs(rw)) + 0.5;
    double vgew = og_sign(0.5, fabs(rv) - fabs(rw)) + 0.5;
    double uzero = og_sign(0.5, fabs(ru) - EPSILON) - 0.5;
    double vzero = og_sign(0.5, fabs(rv) - EPSILON) - 0.5;
    double wzero = og_sign(0.5, fabs(rw) - EPSILON) - 0.5;
    double sign_uv = og_sign(0.5, ru * rv) + 0.5;
    double sign_uw = og_sign(0.5, ru * rw) + 0.5;
    double sign_vw = og_sign(0.5, rv * rw) + 0.5;
    double wu = fabs(rw / (ru + uzero) * (1.0 + uzero));
    double vu = fabs(rv / (ru + uzero) * (1.0 + uzero));
    double uv = fabs(ru / (rv + vzero) * (1.0 + vzero));
    double wv = fabs(rw / (rv + vzero) * (1.0 + vzero));
    double uw = fabs(ru / (rw + wzero) * (1.0 + wzero));
    double vw = fabs(rv / (rw + wzero) * (1.0 + wzero));
    double umax = ugev * ugew * (1.0 + uzero);
    double vmax = (1.0 - ugev) * vgew;
    double wmax = 1.0 - ugev * ugew - vmax;
#define FF(a, b, c) f[a][(b) + 1][(c) + 1]
    FF(0, 0, 0) = -ugev * ugew * uzero;
    FF(1, 0, 0) = wmax * (1.0 - uw) * (1.0 - vw);
    FF(0, 1, 0) = umax * (1.0 - vu) * (1.0 - wu);
    FF(0, 0, 1) = vmax * (1.0 - uv) * (1.0 - wv);
    FF(1, 1, 1) = sign_uv * sign_uw * (umax * vu * wu + vmax * uv * wv + wmax * uw * vw);
    FF(1, -1, 1) = (1.0 - sign_uv) * (1.0 - sign_uw) * (umax * vu * wu + vmax * uv * wv + wmax * uw * vw);
    FF(1, 1, -1) = (1.0 - sign_uv) * sign_uw * (umax * vu * wu + vmax * uv * wv + wmax * uw * vw);
    FF(1, -1, -1) = sign_uv * (1.0 - sign_uw) * (umax * vu * wu + vmax * uv * wv + wmax * uw * vw);
    FF(1, 1, 0) = sign_uw * (1.0 - vmax) * (ugew * wu * (1.0 - vu) + (1.0 - ugew) * uw * (1.0 - vw));
    FF(1, -1, 0) = (1.0 - sign_uw) * (1.0 - vmax) * (ugew * wu * (1.0 - vu) + (1.0 - ugew) * uw * (1.0 - vw));
    FF(1, 0, 1) = sign_vw * (1.0 - umax) * (vgew * wv * (1.0 - uv) + (1.0 - vgew) * vw * (1.0 - uw));
    FF(1, 0, -1) = (1.0 - sign_vw) * (1.0 - umax) * (vgew * wv * (1.0 - uv) + (1.0 - vgew) * vw * (1.0 - uw));
    FF(0, 1, 1) = sign_uv * (1.0 - wmax) * (ugev * vu * (1.0 - wu) + (1.0 - ugev) * uv * (1.0 - wv));
    FF(0, 1, -1) = (1.0 - sign_uv) * (1.0 - wmax) * (ugev * vu * (1.0 - wu) + (1.0 - ugev) * uv * (1.0 - wv));
#undef FF
}

/* ATMOS_DYN_fct, :1922-2671, one block over the whole domain */
void og_fct(const og_dims *d, double *qflx_anti, const double *phi_in, const double *DENS0, const double *DENS,
            const double *qflx_hi, const double *qflx_lo, const double *mflx_hi,
            const double *RDZ, const double *RDX, const double *RDY,
            const double *GSQRT, const double *MAPF, double dt, int flag_vect)
{
    OG_DIMS(d);
    const double EPSILON = OG_EPS;
    double *phi_lo = og_alloc_undef(N3), *pjpls = og_alloc_undef(N3), *pjmns = og_alloc_undef(N3);
    double *qjpls = og_alloc_undef(N3), *qjmns = og_alloc_undef(N3), *rjpls = og_alloc_undef(N3), *rjmns = og_alloc_undef(N3);
    double *aZ = qflx_anti, *aX = qflx_anti + N3, *aY = qflx_anti + 2 * N3;
    const double *hZ = qflx_hi, *hX = qflx_hi + N3, *hY = qflx_hi + 2 * N3;
    const double *lZ = qflx_lo, *lX = qflx_lo + N3, *lY = qflx_lo + 2 * N3;
    const double *mZ = mflx_hi, *mX = mflx_hi + N3, *mY = mflx_hi + 2 * N3;
#define M1(i, j) MAPF[I2(i, j)]
#define M2(i, j) MAPF[I2(i, j) + (size_t)IA * (size_t)JA]

#pragma omp parallel for collapse(2)
    for (int j = JS; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) aZ[I3(k, i, j)] = hZ[I3(k, i, j)] - lZ[I3(k, i, j)];
            aZ[I3(KS - 1, i, j)] = 0.0;
            aZ[I3(KE, i, j)] = 0.0;
        }
#pragma omp parallel for collapse(2)
    for (int j = JS; j <= JE; ++j)
        for (int i = IS - 1; i <= IE; ++i)
            for (int k = KS; k <= KE; ++k) aX[I3(k, i, j)] = hX[I3(k, i, j)] - lX[I3(k, i, j)];
#pragma omp parallel for collapse(2)
    for (int j = JS - 1; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i)
            for (int k = KS; k <= KE; ++k) aY[I3(k, i, j)] = hY[I3(k, i, j)] - lY[I3(k, i, j)];

    /* update monotone scheme :2051-2073 */
#pragma omp parallel for collapse(2)
    for (int j = JS - 1; j <= JE + 1; ++j)
        for (int i = IS - 1; i <= IE + 1; ++i)
            for (int k = KS; k <= KE; ++k)
                phi_lo[I3(k, i, j)] = (phi_in[I3(k, i, j)] * DENS0[I3(k, i, j)]
                                       + dt * (-((lZ[I3(k, i, j)] - lZ[I3(k - 1, i, j)]) * RDZ[k - 1]
                                                 + (lX[I3(k, i, j)] - lX[I3(k, i - 1, j)]) * RDX[i - 1]
                                                 + (lY[I3(k, i, j)] - lY[I3(k, i, j - 1)]) * RDY[j - 1])
                                               * M1(i, j) * M2(i, j) / GSQRT[I3(k, i, j)]))
                                      / DENS[I3(k, i, j)];

#pragma omp parallel for collapse(2)
    for (int j = JS; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i)
            for (int k = KS; k <= KE; ++k) {
                pjpls[I3(k, i, j)] = dt * ((og_max(0.0, aZ[I3(k - 1, i, j)]) - og_min(0.0, aZ[I3(k, i, j)])) * RDZ[k - 1]
                                           + (og_max(0.0, aX[I3(k, i - 1, j)]) - og_min(0.0, aX[I3(k, i, j)])) * RDX[i - 1]
                                           + (og_max(0.0, aY[I3(k, i, j - 1)]) - og_min(0.0, aY[I3(k, i, j)])) * RDY[j - 1])
                                     * M1(i, j) * M2(i, j) / GSQRT[I3(k, i, j)];
                pjmns[I3(k, i, j)] = dt * ((og_max(0.0, aZ[I3(k, i, j)]) - og_min(0.0, aZ[I3(k - 1, i, j)])) * RDZ[k - 1]
                                           + (og_max(0.0, aX[I3(k, i, j)]) - og_min(0.0, aX[I3(k, i - 1, j)])) * RDX[i - 1]
                                           + (og_max(0.0, aY[I3(k, i, j)]) - og_min(0.0, aY[I3(k, i, j - 1)])) * RDY[j - 1])
                                     * M1(i, j) * M2(i, j) / GSQRT[I3(k, i, j)];
            }

#define PI_(k, i, j) phi_in[I3(k, i, j)]
#define PL_(k, i, j) phi_lo[I3(k, i, j)]
    if (flag_vect) {
        /* along-stream 14-point bound :2130-2369. The three k-cases (interior, KS, KE)
         * differ only in which k indices appear; ka/kb give the k used for the
         * (1,*,*) and (0,*,*) points of the qa (upstream) and qb (downstream) sums. */
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i)
                for (int k = KS; k <= KE; ++k) {
                    double rw, ru, rv;
                    int kap, kbm; /* k index replacing k+1 in qa and k-1 in qb */
                    if (k == KS) {
                        rw = (mZ[I3(KS, i, j)]) * RDZ[KS - 1];
                        kap = KS + 1; kbm = KS;
                    } else if (k == KE) {
                        rw = (mZ[I3(KE - 1, i, j)]) * RDZ[KE - 1];
                        kap = KE; kbm = KE - 1;
                    } else {
                        rw = (mZ[I3(k, i, j)] + mZ[I3(k - 1, i, j)]) * RDZ[k - 1];
                        kap = k + 1; kbm = k - 1;
                    }
                    ru = (mX[I3(k, i, j)] + mX[I3(k, i - 1, j)]) * RDX[i - 1];
                    rv = (mY[I3(k, i, j)] + mY[I3(k, i, j - 1)]) * RDY[j - 1];
                    double f[2][3][3];
                    get_fact_fct(f, rw, ru, rv);
#define FA(a, b, c) f[a][(b) + 1][(c) + 1]
                    double qa_in = FA(1, 1, 1) * PI_(kap, i + 1, j + 1) + FA(0, 1, 1) * PI_(k, i + 1, j + 1)
                                   + FA(1, 0, 1) * PI_(kap, i, j + 1) + FA(0, 0, 1) * PI_(k, i, j + 1)
                                   + FA(1, -1, 1) * PI_(kap, i - 1, j + 1) + FA(1, 1, 0) * PI_(kap, i + 1, j)
                                   + FA(0, 1, 0) * PI_(k, i + 1, j) + FA(1, 0, 0) * PI_(kap, i, j)
                                   + FA(1, -1, 0) * PI_(kap, i - 1, j) + FA(1, 1, -1) * PI_(kap, i + 1, j - 1)
                                   + FA(0, 1, -1) * PI_(k, i + 1, j - 1) + FA(1, 0, -1) * PI_(kap, i, j - 1)
                                   + FA(1, -1, -1) * PI_(kap, i - 1, j - 1) + FA(0, 0, 0) * PI_(k, i, j);
                    double qb_in = FA(1, 1, 1) * PI_(kbm, i - 1, j - 1) + FA(0, 1, 1) * PI_(k, i - 1, j - 1)
                                   + FA(1, 0, 1) * PI_(kbm, i, j - 1) + FA(0, 0, 1) * PI_(k, i, j - 1)
                                   + FA(1, -1, 1) * PI_(kbm, i + 1, j - 1) + FA(1, 1, 0) * PI_(kbm, i - 1, j)
                                   + FA(0, 1, 0) * PI_(k, i - 1, j) + FA(1, 0, 0) * PI_(kbm, i, j)
                                   + FA(1, -1, 0) * PI_(kbm, i + 1, j) + FA(1, 1, -1) * PI_(kbm, i - 1, j + 1)
                                   + FA(0, 1, -1) * PI_(k, i - 1, j - 1) + FA(1, 0, -1) * PI_(kbm, i, j - 1)
                                   + FA(1, -1, -1) * PI_(kbm, i + 1, j + 1) + FA(0, 0, 0) * PI_(k, i, j);
                    double qa_lo = FA(1, 1, 1) * PL_(kap, i + 1, j + 1) + FA(0, 1, 1) * PL_(k, i + 1, j + 1)
                                   + FA(1, 0, 1) * PL_(kap, i, j + 1) + FA(0, 0, 1) * PL_(k, i, j + 1)
                                   + FA(1, -1, 1) * PL_(kap, i - 1, j + 1) + FA(1, 1, 0) * PL_(kap, i + 1, j)
                                   + FA(0, 1, 0) * PL_(k, i + 1, j) + FA(1, 0, 0) * PL_(kap, i, j)
                                   + FA(1, -1, 0) * PL_(kap, i - 1, j) + FA(1, 1, -1) * PL_(kap, i + 1, j - 1)
                                   + FA(0, 1, -1) * PL_(k, i + 1, j - 1) + FA(1, 0, -1) * PL_(kap, i, j - 1)
                                   + FA(1, -1, -1) * PL_(kap, i - 1, j - 1) + FA(0, 0, 0) * PL_(k, i, j);
                    double qb_lo = FA(1, 1, 1) * PL_(kbm, i - 1, j - 1) + FA(0, 1, 1) * PL_(k, i - 1, j - 1)
                                   + FA(1, 0, 1) * PL_(kbm, i, j - 1) + FA(0, 0, 1) * PL_(k, i, j - 1)
                                   + FA(1, -1, 1) * PL_(kbm, i + 1, j - 1) + FA(1, 1, 0) * PL_(kbm, i - 1, j)
                                   + FA(0, 1, 0) * PL_(k, i - 1, j) + FA(1, 0, 0) * PL_(kbm, i, j)
                                   + FA(1, -1, 0) * PL_(kbm, i + 1, j) + FA(1, 1, -1) * PL_(kbm, i - 1, j + 1)
                                   + FA(0, 1, -1) * PL_(k, i - 1, j - 1) + FA(1, 0, -1) * PL_(kbm, i, j - 1)
                                   + FA(1, -1, -1) * PL_(kbm, i + 1, j + 1) + FA(0, 0, 0) * PL_(k, i, j);
#undef FA
                    double qmax = og_max(og_max(og_max(og_max(og_max(PI_(k, i, j), qa_in), qb_in), PL_(k, i, j)), qa_lo), qb_lo);
                    double qmin = og_min(og_min(og_min(og_min(og_min(PI_(k, i, j), qa_in), qb_in), PL_(k, i, j)), qa_lo), qb_lo);
                    qjpls[I3(k, i, j)] = (qmax - PL_(k, i, j)) * DENS[I3(k, i, j)];
                    qjmns[I3(k, i, j)] = (PL_(k, i, j) - qmin) * DENS[I3(k, i, j)];
                }
    } else {
        /* 7-point bound :2370-2515 */
#pragma omp parallel for collapse(2)
        for (int j = JS; j <= JE; ++j)
            for (int i = IS; i <= IE; ++i)
                for (int k = KS; k <= KE; ++k) {
                    double qmax, qmin;
                    if (k > KS && k < KE) {
                        qmax = og_max(og_max(og_max(og_max(og_max(og_max(og_max(og_max(og_max(og_max(og_max(og_max(og_max(
                                   PI_(k, i, j), PI_(k + 1, i, j)), PI_(k - 1, i, j)), PI_(k, i + 1, j)), PI_(k, i - 1, j)),
                                   PI_(k, i, j + 1)), PI_(k, i, j - 1)), PL_(k, i, j)), PL_(k + 1, i, j)), PL_(k - 1, i, j)),
                                   PL_(k, i + 1, j)), PL_(k, i - 1, j)), PL_(k, i, j + 1)), PL_(k, i, j - 1));
                        qmin = og_min(og_min(og_min(og_min(og_min(og_min(og_min(og_min(og_min(og_min(og_min(og_min(og_min(
                                   PI_(k, i, j), PI_(k + 1, i, j)), PI_(k - 1, i, j)), PI_(k, i - 1, j)), PI_(k, i + 1, j)),
                                   PI_(k, i, j + 1)), PI_(k, i, j - 1)), PL_(k, i, j)), PL_(k + 1, i, j)), PL_(k - 1, i, j)),
                                   PL_(k, i - 1, j)), PL_(k, i + 1, j)), PL_(k, i, j + 1)), PL_(k, i, j - 1));
                    } else {
                        const int kn = (k == KS) ? KS + 1 : KE - 1;
                        qmax = og_max(og_max(og_max(og_max(og_max(og_max(og_max(og_max(og_max(og_max(og_max(
                                   PI_(k, i, j), PI_(kn, i, j)), PI_(k, i + 1, j)), PI_(k, i - 1, j)), PI_(k, i, j + 1)),
                                   PI_(k, i, j - 1)), PL_(k, i, j)), PL_(kn, i, j)), PL_(k, i + 1, j)), PL_(k, i - 1, j)),
                                   PL_(k, i, j + 1)), PL_(k, i, j - 1));
                        qmin = og_min(og_min(og_min(og_min(og_min(og_min(og_min(og_min(og_min(og_min(og_min(
                                   PI_(k, i, j), PI_(kn, i, j)), PI_(k, i + 1, j)), PI_(k, i - 1, j)), PI_(k, i, j + 1)),
                                   PI_(k, i, j - 1)), PL_(k, i, j)), PL_(kn, i, j)), PL_(k, i + 1, j)), PL_(k, i - 1, j)),
                                   PL_(k, i, j + 1)), PL_(k, i, j - 1));
                    }
                    qjpls[I3(k, i, j)] = (qmax - PL_(k, i, j)) * DENS[I3(k, i, j)];
                    qjmns[I3(k, i, j)] = (PL_(k, i, j) - qmin) * DENS[I3(k, i, j)];
                }
    }
#undef PI_
#undef PL_

    /* flux limitation factors :2516-2553 */
#pragma omp parallel for collapse(2)
    for (int j = JS; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double zerosw = 0.5 - og_sign(0.5, pjpls[I3(k, i, j)] - EPSILON);
                rjpls[I3(k, i, j)] = og_min(1.0, qjpls[I3(k, i, j)] * (1.0 - zerosw) / (pjpls[I3(k, i, j)] - zerosw));
                zerosw = 0.5 - og_sign(0.5, pjmns[I3(k, i, j)] - EPSILON);
                rjmns[I3(k, i, j)] = og_min(1.0, qjmns[I3(k, i, j)] * (1.0 - zerosw) / (pjmns[I3(k, i, j)] - zerosw));
            }
    og_halo_periodic(d, rjpls, 1);
    og_halo_periodic(d, rjmns, 1);

    /* limit the anti-diffusive fluxes :2560-2660 */
#pragma omp parallel for collapse(2)
    for (int j = JS; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i) {
            for (int k = KS; k <= KE - 1; ++k) {
                double a = aZ[I3(k, i, j)];
                double dirsw = 0.5 + og_sign(0.5, a);
                aZ[I3(k, i, j)] = a * (1.0 - og_min(rjpls[I3(k + 1, i, j)], rjmns[I3(k, i, j)]) * (dirsw)
                                       - og_min(rjpls[I3(k, i, j)], rjmns[I3(k + 1, i, j)]) * (1.0 - dirsw));
            }
            aZ[I3(KS - 1, i, j)] = 0.0;
            aZ[I3(KE, i, j)] = 0.0;
        }
#pragma omp parallel for collapse(2)
    for (int j = JS; j <= JE; ++j)
        for (int i = IS - 1; i <= IE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double a = aX[I3(k, i, j)];
                double dirsw = 0.5 + og_sign(0.5, a);
                aX[I3(k, i, j)] = a * (1.0 - og_min(rjpls[I3(k, i + 1, j)], rjmns[I3(k, i, j)]) * (dirsw)
                                       - og_min(rjpls[I3(k, i, j)], rjmns[I3(k, i + 1, j)]) * (1.0 - dirsw));
            }
#pragma omp parallel for collapse(2)
    for (int j = JS - 1; j <= JE; ++j)
        for (int i = IS; i <= IE; ++i)
            for (int k = KS; k <= KE; ++k) {
                double a = aY[I3(k, i, j)];
                double dirsw = 0.5 + og_sign(0.5, a);
                aY[I3(k, i, j)] = a * (1.0 - og_min(rjpls[I3(k, i, j + 1)], rjmns[I3(k, i, j)]) * (dirsw)
                                       - og_min(rjpls[I3(k, i, j)], rjmns[I3(k, i, j + 1)]) * (1.0 - dirsw));
            }
#undef M1
#undef M2
    free(phi_lo); free(pjpls); free(pjmns); free(qjpls); free(qjmns); free(rjpls); free(rjmns);
}
