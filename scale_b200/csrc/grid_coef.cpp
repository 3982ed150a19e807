// Host-side coefficient tables for the device kernels.
//
// These are set-up computations the reference performs once per run or per
// call on the host: the cell-to-face weights F2H of the flux routines and the
// third-difference coefficients of the numerical filter. They are computed in
// FP64 with the reference's expressions (no FMA contraction) so the device
// kernels see the same coefficients the reference uses.
#include <cmath>
#include <vector>
#include "grid_coef.h"

namespace hevi {

// F2H(k,p) = CDZ(k+p-1)*GSQRT(k+p-1) / (CDZ(k)*GSQRT(k) + CDZ(k+1)*GSQRT(k+1))
// (scale_atmos_dyn_fvm_flux_ud3.F90:75) with GSQRT = 1.
void build_f2h(int KA, const double *CDZ, double *F2H1, double *F2H2)
{
    for (int k = 1; k <= KA - 1; ++k) {
        const double den = CDZ[k - 1] * 1.0 + CDZ[k] * 1.0;
        F2H1[k - 1] = CDZ[k - 1] * 1.0 / den;
        F2H2[k - 1] = CDZ[k] * 1.0 / den;
    }
    F2H1[KA - 1] = 0.0;
    F2H2[KA - 1] = 0.0;
}

// real ** integer as gfortran evaluates it (square and multiply)
static double powi(double x, int m)
{
    unsigned n = m < 0 ? -(unsigned)m : (unsigned)m;
    double y = (n % 2) ? x : 1.0;
    while (n >>= 1) {
        x = x * x;
        if (n % 2) y = y * x;
    }
    return m < 0 ? 1.0 / y : y;
}

// ATMOS_DYN_filter_setup (scale_atmos_dyn_common.F90:200-330): CNZ3, CNX3, CNY3,
// and the nd_coef_* vectors of ATMOS_DYN_numfilter_coef (:444-463).
void build_nd_tables(const NdGrid &gr, double DT, double ND_COEF, int ND_ORDER, NdTables &t)
{
    const int KA = gr.KA, IA = gr.IA, JA = gr.JA, KS = gr.KS, KE = gr.KE, IS = gr.IS, IE = gr.IE, JS = gr.JS, JE = gr.JE;
    t.CNZ3.assign(3 * (size_t)KA * 2, 0.0);
    t.CNX3.assign(3 * (size_t)IA * 2, 0.0);
    t.CNY3.assign(3 * (size_t)JA * 2, 0.0);
    auto cz = [&](int n, int k, int s) -> double & { return t.CNZ3[(n - 1) + 3 * ((size_t)(k - 1) + (size_t)KA * (s - 1))]; };
    auto cx = [&](int n, int i, int s) -> double & { return t.CNX3[(n - 1) + 3 * ((size_t)(i - 1) + (size_t)IA * (s - 1))]; };
    auto cy = [&](int n, int j, int s) -> double & { return t.CNY3[(n - 1) + 3 * ((size_t)(j - 1) + (size_t)JA * (s - 1))]; };
    auto CDZ = [&](int k) { return gr.CDZ[k - 1]; };
    auto FDZ = [&](int k) { return gr.FDZ[k - 1]; };
    auto CDX = [&](int i) { return gr.CDX[i - 1]; };
    auto FDX = [&](int i) { return gr.FDX[i - 1]; };
    auto CDY = [&](int j) { return gr.CDY[j - 1]; };
    auto FDY = [&](int j) { return gr.FDY[j - 1]; };

    // z, first kind (:203-250)
    for (int k = KS + 1; k <= KE - 1; ++k) {
        cz(1, k, 1) = 1.0 / (FDZ(k) * CDZ(k) * FDZ(k - 1));
        cz(2, k, 1) = 1.0 / (FDZ(k) * CDZ(k) * FDZ(k - 1)) + 1.0 / (FDZ(k - 1) * CDZ(k) * FDZ(k - 1))
                      + 1.0 / (FDZ(k - 1) * CDZ(k - 1) * FDZ(k - 1));
    }
    for (int k = KS + 2; k <= KE; ++k)
        cz(3, k, 1) = 1.0 / (FDZ(k - 1) * CDZ(k) * FDZ(k - 1)) + 1.0 / (FDZ(k - 1) * CDZ(k - 1) * FDZ(k - 1))
                      + 1.0 / (FDZ(k - 1) * CDZ(k - 1) * FDZ(k - 2));
    cz(1, KS - 1, 1) = 1.0 / (FDZ(KS) * CDZ(KS + 1) * FDZ(KS));
    cz(1, KS, 1) = 1.0 / (FDZ(KS) * CDZ(KS) * FDZ(KS));
    cz(2, KS, 1) = 1.0 / (FDZ(KS) * CDZ(KS) * FDZ(KS)) + 1.0 / (FDZ(KS) * CDZ(KS) * FDZ(KS)) + 1.0 / (FDZ(KS) * CDZ(KS + 1) * FDZ(KS));
    cz(3, KS, 1) = 1.0 / (FDZ(KS) * CDZ(KS) * FDZ(KS)) + 1.0 / (FDZ(KS) * CDZ(KS + 1) * FDZ(KS)) + 1.0 / (FDZ(KS) * CDZ(KS + 1) * FDZ(KS + 1));
    cz(3, KS + 1, 1) = 1.0 / (FDZ(KS) * CDZ(KS + 1) * FDZ(KS)) + 1.0 / (FDZ(KS) * CDZ(KS) * FDZ(KS)) + 1.0 / (FDZ(KS) * CDZ(KS) * FDZ(KS));
    cz(1, KE, 1) = 1.0 / (FDZ(KE - 1) * CDZ(KE) * FDZ(KE - 1));
    cz(2, KE, 1) = 1.0 / (FDZ(KE - 1) * CDZ(KE) * FDZ(KE - 1)) + 1.0 / (FDZ(KE - 1) * CDZ(KE) * FDZ(KE - 1))
                   + 1.0 / (FDZ(KE - 1) * CDZ(KE - 1) * FDZ(KE - 1));
    cz(1, KE + 1, 1) = 1.0 / (FDZ(KE - 2) * CDZ(KE - 1) * FDZ(KE - 1));
    cz(2, KE + 1, 1) = 1.0 / (FDZ(KE - 2) * CDZ(KE - 1) * FDZ(KE - 1)) + 1.0 / (FDZ(KE - 1) * CDZ(KE - 1) * FDZ(KE - 1))
                       + 1.0 / (FDZ(KE - 1) * CDZ(KE) * FDZ(KE - 1));
    cz(3, KE + 1, 1) = 1.0 / (FDZ(KE - 1) * CDZ(KE + 1) * FDZ(KE - 1)) + 1.0 / (FDZ(KE - 1) * CDZ(KE) * FDZ(KE - 1))
                       + 1.0 / (FDZ(KE - 1) * CDZ(KE) * FDZ(KE - 1));
    // z, second kind (:259-305)
    for (int k = KS + 1; k <= KE - 1; ++k) {
        cz(1, k, 2) = 1.0 / (CDZ(k + 1) * FDZ(k) * CDZ(k));
        cz(2, k, 2) = 1.0 / (CDZ(k + 1) * FDZ(k) * CDZ(k)) + 1.0 / (CDZ(k) * FDZ(k) * CDZ(k)) + 1.0 / (CDZ(k) * FDZ(k - 1) * CDZ(k));
        cz(3, k, 2) = 1.0 / (CDZ(k) * FDZ(k) * CDZ(k)) + 1.0 / (CDZ(k) * FDZ(k - 1) * CDZ(k)) + 1.0 / (CDZ(k) * FDZ(k - 1) * CDZ(k - 1));
    }
    cz(1, KS - 1, 2) = 1.0 / (CDZ(KS) * FDZ(KS) * CDZ(KS));
    cz(1, KS, 2) = 1.0 / (CDZ(KS + 1) * FDZ(KS) * CDZ(KS));
    cz(2, KS, 2) = 1.0 / (CDZ(KS + 1) * FDZ(KS) * CDZ(KS)) + 1.0 / (CDZ(KS) * FDZ(KS) * CDZ(KS)) + 1.0 / (CDZ(KS) * FDZ(KS) * CDZ(KS));
    cz(3, KS, 2) = 1.0 / (CDZ(KS) * FDZ(KS) * CDZ(KS)) + 1.0 / (CDZ(KS) * FDZ(KS) * CDZ(KS)) + 1.0 / (CDZ(KS) * FDZ(KS) * CDZ(KS + 1));
    cz(1, KE, 2) = 1.0 / (CDZ(KE - 1) * FDZ(KE - 1) * CDZ(KE));
    cz(2, KE, 2) = 1.0 / (CDZ(KE - 1) * FDZ(KE - 1) * CDZ(KE)) + 1.0 / (CDZ(KE) * FDZ(KE - 1) * CDZ(KE))
                   + 1.0 / (CDZ(KE) * FDZ(KE - 1) * CDZ(KE));
    cz(3, KE, 2) = 1.0 / (CDZ(KE) * FDZ(KE - 1) * CDZ(KE)) + 1.0 / (CDZ(KE) * FDZ(KE - 1) * CDZ(KE))
                   + 1.0 / (CDZ(KE) * FDZ(KE - 1) * CDZ(KE - 1));
    cz(1, KE + 1, 2) = 1.0 / (CDZ(KE - 2) * FDZ(KE - 2) * CDZ(KE - 1));
    cz(2, KE + 1, 2) = 1.0 / (CDZ(KE - 2) * FDZ(KE - 2) * CDZ(KE - 1)) + 1.0 / (CDZ(KE - 1) * FDZ(KE - 2) * CDZ(KE - 1))
                       + 1.0 / (CDZ(KE - 1) * FDZ(KE - 1) * CDZ(KE - 1));
    cz(3, KE + 1, 2) = 1.0 / (CDZ(KE - 1) * FDZ(KE - 2) * CDZ(KE - 1)) + 1.0 / (CDZ(KE - 1) * FDZ(KE - 1) * CDZ(KE - 1))
                       + 1.0 / (CDZ(KE - 1) * FDZ(KE - 1) * CDZ(KE));
    // x (:318-346)
    cx(1, IS - 1, 1) = 1.0 / (FDX(IS - 1) * CDX(IS - 1) * FDX(IS - 2));
    for (int i = IS; i <= IE + 1; ++i) {
        cx(1, i, 1) = 1.0 / (FDX(i) * CDX(i) * FDX(i - 1));
        cx(2, i, 1) = 1.0 / (FDX(i) * CDX(i) * FDX(i - 1)) + 1.0 / (FDX(i - 1) * CDX(i) * FDX(i - 1)) + 1.0 / (FDX(i - 1) * CDX(i - 1) * FDX(i - 1));
        cx(3, i, 1) = 1.0 / (FDX(i - 1) * CDX(i) * FDX(i - 1)) + 1.0 / (FDX(i - 1) * CDX(i - 1) * FDX(i - 1)) + 1.0 / (FDX(i - 1) * CDX(i - 1) * FDX(i - 2));
    }
    for (int i = IS - 1; i <= IE + 1; ++i) {
        cx(1, i, 2) = 1.0 / (CDX(i + 1) * FDX(i) * CDX(i));
        cx(2, i, 2) = 1.0 / (CDX(i + 1) * FDX(i) * CDX(i)) + 1.0 / (CDX(i) * FDX(i) * CDX(i)) + 1.0 / (CDX(i) * FDX(i - 1) * CDX(i));
        cx(3, i, 2) = 1.0 / (CDX(i) * FDX(i) * CDX(i)) + 1.0 / (CDX(i) * FDX(i - 1) * CDX(i)) + 1.0 / (CDX(i) * FDX(i - 1) * CDX(i - 1));
    }
    // y (:348-376)
    cy(1, JS - 1, 1) = 1.0 / (FDY(JS - 1) * CDY(JS - 1) * FDY(JS - 2));
    for (int j = JS; j <= JE + 1; ++j) {
        cy(1, j, 1) = 1.0 / (FDY(j) * CDY(j) * FDY(j - 1));
        cy(2, j, 1) = 1.0 / (FDY(j) * CDY(j) * FDY(j - 1)) + 1.0 / (FDY(j - 1) * CDY(j) * FDY(j - 1)) + 1.0 / (FDY(j - 1) * CDY(j - 1) * FDY(j - 1));
        cy(3, j, 1) = 1.0 / (FDY(j - 1) * CDY(j) * FDY(j - 1)) + 1.0 / (FDY(j - 1) * CDY(j - 1) * FDY(j - 1)) + 1.0 / (FDY(j - 1) * CDY(j - 1) * FDY(j - 2));
    }
    for (int j = JS - 1; j <= JE + 1; ++j) {
        cy(1, j, 2) = 1.0 / (CDY(j + 1) * FDY(j) * CDY(j));
        cy(2, j, 2) = 1.0 / (CDY(j + 1) * FDY(j) * CDY(j)) + 1.0 / (CDY(j) * FDY(j) * CDY(j)) + 1.0 / (CDY(j) * FDY(j - 1) * CDY(j));
        cy(3, j, 2) = 1.0 / (CDY(j) * FDY(j) * CDY(j)) + 1.0 / (CDY(j) * FDY(j - 1) * CDY(j)) + 1.0 / (CDY(j) * FDY(j - 1) * CDY(j - 1));
    }

    // fourth-order coefficients of calc_diff4 (:186-193, :253-263, :281-297, :309-317):
    // the first kind divides by CDZ/CDX/CDY, the second by FDZ/FDX/FDY
    t.CNZ4.assign(5 * (size_t)KA * 2, 0.0);
    t.CNX4.assign(5 * (size_t)IA * 2, 0.0);
    t.CNY4.assign(5 * (size_t)JA * 2, 0.0);
    auto c4 = [](std::vector<double> &v, int N, int n, int p, int s) -> double & {
        return v[(n - 1) + 5 * ((size_t)(p - 1) + (size_t)N * (s - 1))];
    };
    for (int s = 1; s <= 2; ++s) {
        for (int k = KS; k <= KE - 1; ++k) {
            const double den = s == 1 ? CDZ(k) : FDZ(k);
            c4(t.CNZ4, KA, 1, k, s) = (cz(1, k + 1, s)) / den;
            c4(t.CNZ4, KA, 2, k, s) = (cz(2, k + 1, s) + cz(1, k, s)) / den;
            c4(t.CNZ4, KA, 3, k, s) = (cz(3, k + 1, s) + cz(2, k, s)) / den;
            c4(t.CNZ4, KA, 4, k, s) = (cz(1, k, s) + cz(3, k, s)) / den;
            c4(t.CNZ4, KA, 5, k, s) = (cz(1, k - 1, s)) / den;
        }
        for (int i = IS; i <= IE; ++i) {
            const double den = s == 1 ? CDX(i) : FDX(i);
            c4(t.CNX4, IA, 1, i, s) = (cx(1, i + 1, s)) / den;
            c4(t.CNX4, IA, 2, i, s) = (cx(2, i + 1, s) + cx(1, i, s)) / den;
            c4(t.CNX4, IA, 3, i, s) = (cx(3, i + 1, s) + cx(2, i, s)) / den;
            c4(t.CNX4, IA, 4, i, s) = (cx(1, i, s) + cx(3, i, s)) / den;
            c4(t.CNX4, IA, 5, i, s) = (cx(1, i - 1, s)) / den;
        }
        for (int j = JS; j <= JE; ++j) {
            const double den = s == 1 ? CDY(j) : FDY(j);
            c4(t.CNY4, JA, 1, j, s) = (cy(1, j + 1, s)) / den;
            c4(t.CNY4, JA, 2, j, s) = (cy(2, j + 1, s) + cy(1, j, s)) / den;
            c4(t.CNY4, JA, 3, j, s) = (cy(3, j + 1, s) + cy(2, j, s)) / den;
            c4(t.CNY4, JA, 4, j, s) = (cy(1, j, s) + cy(3, j, s)) / den;
            c4(t.CNY4, JA, 5, j, s) = (cy(1, j - 1, s)) / den;
        }
    }

    // nd_coef_* (:444-463): DIFF4 = ND_COEF / (2**(4*order) * DT), coef = DIFF4 * D**(4*order)
    const int n4 = ND_ORDER * 4;
    const double DIFF4 = ND_COEF / (powi(2.0, n4) * DT);
    t.cdz.assign(KA, 0.0); t.fdz.assign(KA, 0.0);
    t.cdx.assign(IA, 0.0); t.fdx.assign(IA, 0.0);
    t.cdy.assign(JA, 0.0); t.fdy.assign(JA, 0.0);
    for (int k = KS - 1; k <= KE; ++k) t.cdz[k - 1] = DIFF4 * powi(CDZ(k), n4);
    for (int k = KS + 1; k <= KE - 1; ++k) t.fdz[k - 1] = DIFF4 * powi(FDZ(k), n4);
    for (int i = IS; i <= IE; ++i) { t.cdx[i - 1] = DIFF4 * powi(CDX(i), n4); t.fdx[i - 1] = DIFF4 * powi(FDX(i), n4); }
    for (int j = JS; j <= JE; ++j) { t.cdy[j - 1] = DIFF4 * powi(CDY(j), n4); t.fdy[j - 1] = DIFF4 * powi(FDY(j), n4); }
}

}  // namespace hevi
