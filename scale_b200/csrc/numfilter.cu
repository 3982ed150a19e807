// Numerical hyper-diffusion fluxes num_diff(KA,IA,JA,5,3) for ND_ORDER = 1
// (ATMOS_DYN_numfilter_coef, scale_atmos_dyn_common.F90:385-985, with the
// third-difference operator calc_diff3 :1600-1760 and its coefficients from
// ATMOS_DYN_filter_setup :200-330).
//
// Two kernels. k_phi evaluates the five filtered quantities (density and
// theta deviations, three velocities) once at every point into a scratch of
// five fields, so no quotient is formed twice. k_numfilter then has the lanes
// of a warp take the levels KS..KE of one interior column and write all 15
// components there, then the zero and mirrored values of the vertical halo,
// reading the quantities from the scratch. The lateral halo is filled
// afterwards by the periodic halo kernel, as COMM_vars8 does in the reference.
//
// R is the output and arithmetic type: double on the plain path, float on the
// mixed-precision path (the deviations from the base state and the quotients
// of k_phi are formed in FP64 and then stored as R).
#include "hevi_kernels.cuh"

namespace hevi {

#define CZ3(n, k, s) (R)ld(c.CNZ3 + ((n) - 1) + 3 * ((size_t)((k) - 1) + (size_t)g.KA * ((s) - 1)))
#define CX3(n, i, s) (R)ld(c.CNX3 + ((n) - 1) + 3 * ((size_t)((i) - 1) + (size_t)g.IA * ((s) - 1)))
#define CY3(n, j, s) (R)ld(c.CNY3 + ((n) - 1) + 3 * ((size_t)((j) - 1) + (size_t)g.JA * ((s) - 1)))

constexpr int PHI_THREADS = 256;

// The five filtered quantities at one point.
// q: 0 DENS-REF_dens, 1 VELZ, 2 VELX, 3 VELY, 4 RHOT/DENS-REF_pott  (:538-547, 621-626, 715-720, 799-804, 876-883)
// A velocity needs the density one point above (VELZ), east (VELX) or north
// (VELY); at the last point of the array in that direction, which no stencil
// reads, it is stored as zero. One thread per point of the (KA,IA,JA) array,
// in memory order: one fully coalesced stream with no idle lanes at the
// column ends.
template <typename R, int NM>
__global__ void __launch_bounds__(PHI_THREADS) k_phi(const Grid gt, const NdArgsT<R> a, const BatchT<NM> B)
{
    int b;
    const Grid g = block_domain(gt, B, b);
    // 32-bit index arithmetic: a field has fewer than 2^31 points (checked at setup)
    const unsigned npts = (unsigned)g.KA * g.IA * g.JA;
    const unsigned pt = (unsigned)b * PHI_THREADS + threadIdx.x;
    if (pt >= npts) return;
    const unsigned KA = g.KA, IA = g.IA;
    const unsigned r = pt / KA;
    const int k = (int)(pt - r * KA) + 1;
    const unsigned jj = r / IA;
    const int i = (int)(r - jj * IA) + 1, j = (int)jj + 1;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const size_t c = (size_t)g.cell0 + (size_t)pt;
    const double D = ld(a.DENS + c);
    a.phi[c] = R(D - ld(a.REF_dens + c));
    a.phi[c + N3] = R(k < g.KA ? 2.0 * ld(a.MOMZ + c) / (ld(a.DENS + c + 1) + D) : 0.0);
    a.phi[c + 2 * N3] = R(i < g.IA ? 2.0 * ld(a.MOMX + c) / (ld(a.DENS + c + sI) + D) : 0.0);
    a.phi[c + 3 * N3] = R(j < g.JA ? 2.0 * ld(a.MOMY + c) / (ld(a.DENS + c + sJ) + D) : 0.0);
    a.phi[c + 4 * N3] = R(ld(a.RHOT + c) / D - ld(a.REF_pott + c));
}

// the quantities read back by the stencils
template <typename R>
struct Phi {
    const Grid &g;
    const NdArgsT<R> &a;
    __device__ R operator()(int q, int k, int i, int j) const
    {
        return __ldg(a.phi + (size_t)q * n3(g) + idx3(g, k, i, j));
    }
};

// calc_diff3 z-component with KO = 0 (:1617-1655) at level k (any k in 1..KA)
template <typename R>
__device__ R dz0(const Grid &g, const NdCoef &c, const Phi<R> &phi, int q, int k, int i, int j)
{
    const int KS = g.KS, KE = g.KE;
    auto inner = [&](int m) {
        return (+CZ3(1, m + 1, 1) * phi(q, m + 2, i, j) - CZ3(2, m + 1, 1) * phi(q, m + 1, i, j)
                + CZ3(3, m + 1, 1) * phi(q, m, i, j) - CZ3(1, m, 1) * phi(q, m - 1, i, j));
    };
    auto atKS = [&]() {
        return (+CZ3(1, KS + 1, 1) * phi(q, KS + 2, i, j) - CZ3(2, KS + 1, 1) * phi(q, KS + 1, i, j)
                + CZ3(3, KS + 1, 1) * phi(q, KS, i, j) - CZ3(1, KS, 1) * phi(q, KS + 1, i, j));
    };
    auto atKEm1 = [&]() {
        return (+CZ3(1, KE, 1) * phi(q, KE - 1, i, j) - CZ3(2, KE, 1) * phi(q, KE, i, j)
                + CZ3(3, KE, 1) * phi(q, KE - 1, i, j) - CZ3(1, KE - 1, 1) * phi(q, KE - 2, i, j));
    };
    if (k >= KS + 1 && k <= KE - 2) return inner(k);
    if (k == KS) return atKS();
    if (k == KS - 1) return -atKS();
    if (k == KS - 2) return -inner(KS + 1);
    if (k == KE - 1) return atKEm1();
    if (k == KE) return -atKEm1();
    if (k == KE + 1) return -inner(KE - 2);
    return R(0.0); // KE+2
}

// calc_diff3 z-component with KO = 1 (:1657-1705)
template <typename R>
__device__ R dz1(const Grid &g, const NdCoef &c, const Phi<R> &phi, int q, int k, int i, int j)
{
    const int KS = g.KS, KE = g.KE;
    auto inner = [&](int m) {
        return (+CZ3(1, m, 2) * phi(q, m + 1, i, j) - CZ3(2, m, 2) * phi(q, m, i, j)
                + CZ3(3, m, 2) * phi(q, m - 1, i, j) - CZ3(1, m - 1, 2) * phi(q, m - 2, i, j));
    };
    auto atKSp1 = [&]() {
        return (+CZ3(1, KS + 1, 2) * phi(q, KS + 2, i, j) - CZ3(2, KS + 1, 2) * phi(q, KS + 1, i, j)
                + CZ3(3, KS + 1, 2) * phi(q, KS, i, j) - CZ3(1, KS, 2) * phi(q, KS + 1, i, j));
    };
    auto atKEm1 = [&]() {
        return (-CZ3(2, KE - 1, 2) * phi(q, KE - 1, i, j) + CZ3(3, KE - 1, 2) * phi(q, KE - 2, i, j)
                - CZ3(1, KE - 2, 2) * phi(q, KE - 3, i, j));
    };
    auto atKE = [&]() {
        return (+CZ3(1, KE, 2) * phi(q, KE - 1, i, j) + CZ3(3, KE, 2) * phi(q, KE - 1, i, j)
                - CZ3(1, KE - 1, 2) * phi(q, KE - 2, i, j));
    };
    if (k >= KS + 2 && k <= KE - 2) return inner(k);
    if (k == KS + 1) return atKSp1();
    if (k == KS) return -atKSp1();
    if (k == KS - 1) return -inner(KS + 2);
    if (k == KS - 2) return -inner(KS + 3);
    if (k == KE - 1) return atKEm1();
    if (k == KE) return atKE();
    if (k == KE + 1) return -atKE();
    return -atKEm1(); // KE+2
}

// x and y components (:1707-1760); o selects IO/JO
template <typename R>
__device__ __forceinline__ R dx(const Grid &g, const NdCoef &c, const Phi<R> &phi, int q, int o, int k, int i, int j)
{
    if (o == 0)
        return (+CX3(1, i + 1, 1) * phi(q, k, i + 2, j) - CX3(2, i + 1, 1) * phi(q, k, i + 1, j)
                + CX3(3, i + 1, 1) * phi(q, k, i, j) - CX3(1, i, 1) * phi(q, k, i - 1, j));
    return (+CX3(1, i, 2) * phi(q, k, i + 1, j) - CX3(2, i, 2) * phi(q, k, i, j)
            + CX3(3, i, 2) * phi(q, k, i - 1, j) - CX3(1, i - 1, 2) * phi(q, k, i - 2, j));
}
template <typename R>
__device__ __forceinline__ R dy(const Grid &g, const NdCoef &c, const Phi<R> &phi, int q, int o, int k, int i, int j)
{
    if (o == 0)
        return (+CY3(1, j + 1, 1) * phi(q, k, i, j + 2) - CY3(2, j + 1, 1) * phi(q, k, i, j + 1)
                + CY3(3, j + 1, 1) * phi(q, k, i, j) - CY3(1, j, 1) * phi(q, k, i, j - 1));
    return (+CY3(1, j, 2) * phi(q, k, i, j + 1) - CY3(2, j, 2) * phi(q, k, i, j)
            + CY3(3, j, 2) * phi(q, k, i, j - 1) - CY3(1, j - 1, 2) * phi(q, k, i, j - 2));
}

#ifndef HEVI_ND_MINB
#define HEVI_ND_MINB 8 // minimum resident blocks per SM asked of the register allocator
#endif

// FW: the differences come from the calc_numdiff work buffer W (ND_ORDER > 1)
// instead of being formed from phi here (ND_ORDER = 1)
//
// The lanes of a warp take the levels KS..KE of one column, so that every
// pass over 32 levels but the last is full; the halo levels (zero, except the
// mirrors at KS-1 of density and theta) are written by a short tail pass.
template <typename R, int NM, bool FW = false>
__global__ void __launch_bounds__(128, HEVI_ND_MINB)
    k_numfilter(const Grid gt, const NdCoef ct, const NdArgsT<R> a, const BatchT<NM> B, const double *W = nullptr)
{
    int b;
    const Grid g = block_domain(gt, B, b);
    const NdCoef c = NM == 1 ? ct : member_nd(ct, g);
    const Block2 p = split_block(b, (g.IMAX + 3) / 4);
    const int i = g.IS + p.x * blockDim.y + threadIdx.y;
    const int j = g.JS + p.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const int KS = g.KS, KE = g.KE;
    const Phi<R> phi{g, a};
    const double *DN = a.DENS;
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const R ncx = R(ld(c.cdx + i - 1)), nfx = R(ld(c.fdx + i - 1)), ncy = R(ld(c.cdy + j - 1)), nfy = R(ld(c.fdy + j - 1));
    const R sfc = R(c.sfc);
    // surface-factor tail of every x/y component (:581-585 and the analogous blocks)
    auto sfct = [&](int k, R v) {
        if (k == KS) return v * sfc;
        if (k == KS + 1) return v * (R(1.0) + sfc) * R(0.5);
        return v;
    };
    R *ND = a.num_diff;
    for (int k = KS + threadIdx.x; k <= KE; k += 32) {
        const size_t o = idx3(g, k, i, j);
        // the difference of quantity q in a direction: formed here from phi, or
        // read from the work buffer (the expression is then not evaluated)
#define DZ(q, expr) (FW ? R(ld(W + (size_t)(3 * (q) + 0) * N3 + o)) : (expr))
#define DX(q, expr) (FW ? R(ld(W + (size_t)(3 * (q) + 1) * N3 + o)) : (expr))
#define DY(q, expr) (FW ? R(ld(W + (size_t)(3 * (q) + 2) * N3 + o)) : (expr))
        const R ncz = R(ld(c.cdz + k - 1));
        const bool kz = k <= KE - 1;
        // one quantity at a time (the loop is kept rolled, so that the loads of
        // one quantity's three components are all that is in flight)
#pragma unroll 1
        for (int q = 0; q < 5; ++q) {
            switch (q) {
            case 0: // ---- density (:553-610) ----
                ND[o + N3 * 0] = DZ(0, dz0(g, c, phi, 0, k, i, j)) * ncz;
                ND[o + N3 * 5] = sfct(k, DX(0, dx(g, c, phi, 0, 0, k, i, j)) * ncx);
                ND[o + N3 * 10] = sfct(k, DY(0, dy(g, c, phi, 0, 0, k, i, j)) * ncy);
                break;
            case 1: { // ---- z momentum (:628-698), phi = VELZ on KS..KE-1 ----
                const bool kz1 = k >= KS + 1 && kz;
                const R nfz = kz1 ? R(ld(c.fdz + k - 1)) : R(0.0);
                ND[o + N3 * 1] = kz1 ? DZ(1, dz1(g, c, phi, 1, k, i, j)) * nfz * R(ld(DN + o)) : R(0.0);
                ND[o + N3 * 6] = kz ? sfct(k, DX(1, dx(g, c, phi, 1, 0, k, i, j)) * ncx
                                                  * R(0.25) * (R(ld(DN + o + 1 + sI)) + R(ld(DN + o + 1)) + R(ld(DN + o + sI)) + R(ld(DN + o))))
                                    : R(0.0);
                ND[o + N3 * 11] = kz ? sfct(k, DY(1, dy(g, c, phi, 1, 0, k, i, j)) * ncy
                                                   * R(0.25) * (R(ld(DN + o + 1 + sJ)) + R(ld(DN + o + 1)) + R(ld(DN + o + sJ)) + R(ld(DN + o))))
                                     : R(0.0);
                break;
            }
            case 2: // ---- x momentum (:728-790), phi = VELX ----
                ND[o + N3 * 2] = kz ? DZ(2, dz0(g, c, phi, 2, k, i, j)) * ncz
                                          * R(0.25) * (R(ld(DN + o + 1 + sI)) + R(ld(DN + o + 1)) + R(ld(DN + o + sI)) + R(ld(DN + o)))
                                    : R(0.0);
                ND[o + N3 * 7] = sfct(k, DX(2, dx(g, c, phi, 2, 1, k, i, j)) * nfx * R(ld(DN + o)));
                ND[o + N3 * 12] = sfct(k, DY(2, dy(g, c, phi, 2, 0, k, i, j)) * ncy
                                              * R(0.25) * (R(ld(DN + o + sI + sJ)) + R(ld(DN + o + sI)) + R(ld(DN + o + sJ)) + R(ld(DN + o))));
                break;
            case 3: // ---- y momentum (:812-870), phi = VELY ----
                ND[o + N3 * 3] = kz ? DZ(3, dz0(g, c, phi, 3, k, i, j)) * ncz
                                          * R(0.25) * (R(ld(DN + o + 1 + sJ)) + R(ld(DN + o + 1)) + R(ld(DN + o + sJ)) + R(ld(DN + o)))
                                    : R(0.0);
                ND[o + N3 * 8] = sfct(k, DX(3, dx(g, c, phi, 3, 0, k, i, j)) * ncx
                                             * R(0.25) * (R(ld(DN + o + sI + sJ)) + R(ld(DN + o + sJ)) + R(ld(DN + o + sI)) + R(ld(DN + o))));
                ND[o + N3 * 13] = sfct(k, DY(3, dy(g, c, phi, 3, 1, k, i, j)) * nfy * R(ld(DN + o)));
                break;
            default: { // ---- rho*theta (:885-960) ----
                const R v = DZ(4, dz0(g, c, phi, 4, k, i, j)) * ncz;
                ND[o + N3 * 4] = kz ? v * R(0.5) * (R(ld(DN + o + 1)) + R(ld(DN + o))) : v * R(ld(DN + o));
                ND[o + N3 * 9] = sfct(k, DX(4, dx(g, c, phi, 4, 0, k, i, j)) * ncx * R(0.5) * (R(ld(DN + o + sI)) + R(ld(DN + o))));
                ND[o + N3 * 14] = sfct(k, DY(4, dy(g, c, phi, 4, 0, k, i, j)) * ncy * R(0.5) * (R(ld(DN + o + sJ)) + R(ld(DN + o))));
            }
            }
        }
    }
    // halo levels 1..KS-1 and KE+1..KA: zero, except density and theta z at
    // KS-1 (the mirror -atKS of level KS)
    const int nlo = KS - 1, nh = nlo + (g.KA - KE);
    for (int h = threadIdx.x; h < nh; h += 32) {
        const int k = h < nlo ? h + 1 : KE + 1 + (h - nlo);
        const size_t o = idx3(g, k, i, j);
        for (int q = 0; q < 15; ++q) ND[o + N3 * q] = R(0.0);
        if (k == KS - 1) {
            const R ncz = R(ld(c.cdz + k - 1));
            ND[o + N3 * 0] = DZ(0, dz0(g, c, phi, 0, k, i, j)) * ncz;
            ND[o + N3 * 4] = DZ(4, dz0(g, c, phi, 4, k, i, j)) * ncz * R(R(ld(DN + idx3(g, KS, i, j))));
        }
    }
}

#undef DZ
#undef DX
#undef DY

#ifndef HEVI_FLOAT_TU // the ND_ORDER > 1 path is FP64 only
// ---- ND_ORDER > 1: calc_numdiff (scale_atmos_dyn_common.F90:1518-1573) -----------
// calc_diff3 of the five quantities (q: 0 density, 1 VELZ, 2 VELX, 3 VELY, 4
// theta) into the work buffer, at every level of the interior columns; the
// horizontal components on KS..KE-KO only, zero elsewhere (:1600-1760)
__global__ void __launch_bounds__(128) k_nd_diff3(const Grid g, const NdCoef c, const NdArgs a, double *W)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const Phi<double> phi{g, a};
    for (int k = 1 + threadIdx.x; k <= g.KA; k += 32) {
        const size_t o = idx3(g, k, i, j);
        for (int q = 0; q < 5; ++q) {
            const int KO = q == 1, IO = q == 2, JO = q == 3, KEE = g.KE - KO;
            W[(size_t)(3 * q + 0) * N3 + o] = KO ? dz1(g, c, phi, q, k, i, j) : dz0(g, c, phi, q, k, i, j);
            const bool kin = k >= g.KS && k <= KEE;
            W[(size_t)(3 * q + 1) * N3 + o] = kin ? dx(g, c, phi, q, IO, k, i, j) : 0.0;
            W[(size_t)(3 * q + 2) * N3 + o] = kin ? dy(g, c, phi, q, JO, k, i, j) : 0.0;
        }
    }
}

// calc_diff4 (:1810-1918): z on KS..KE-1 and the mirrored levels KS-1, KS-2,
// KE, KE+1 (written by the lane of the level they mirror, after a warp-wide
// pass over the levels); x and y on KS..KE-KO
__global__ void __launch_bounds__(128) k_nd_diff4(const Grid g, const NdCoef c, const double *Win, double *Wout)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g), sI = (size_t)g.KA, sJ = (size_t)g.KA * g.IA;
    const int KS = g.KS, KE = g.KE;
    const size_t c1 = idx3(g, 1, i, j);
    for (int q = 0; q < 5; ++q) {
        const int KO = q == 1, IO = q == 2, JO = q == 3, K1 = KE - KO;
        const double *CZ = c.CNZ4 + 5 * (size_t)g.KA * KO, *CX = c.CNX4 + 5 * (size_t)g.IA * IO,
                     *CY = c.CNY4 + 5 * (size_t)g.JA * JO;
        const double *iz = Win + (size_t)(3 * q) * N3, *ix = iz + N3, *iy = iz + 2 * N3;
        double *oz = Wout + (size_t)(3 * q) * N3, *ox = oz + N3, *oy = oz + 2 * N3;
        auto zval = [&](int k) {
            const size_t o = c1 + k - 1;
            const double *cz = CZ + 5 * (size_t)(k - 1);
            return (ld(cz) * ld(iz + o + 2) - ld(cz + 1) * ld(iz + o + 1) + ld(cz + 2) * ld(iz + o) - ld(cz + 3) * ld(iz + o - 1)
                    + ld(cz + 4) * ld(iz + o - 2));
        };
        for (int k = 1 + threadIdx.x; k <= g.KA; k += 32) {
            const size_t o = c1 + k - 1;
            if (k >= KS && k <= KE - 1) oz[o] = zval(k);
            else if (k == KS - 1) oz[o] = -zval(KS);
            else if (k == KS - 2) oz[o] = -zval(KS + 1);
            else if (k == KE) oz[o] = -zval(KE - 1);
            else if (k == KE + 1) oz[o] = -zval(KE - 2);
            if (k >= KS && k <= K1) {
                const double *cx = CX + 5 * (size_t)(i - 1), *cy = CY + 5 * (size_t)(j - 1);
                ox[o] = (ld(cx) * ld(ix + o + 2 * sI) - ld(cx + 1) * ld(ix + o + sI) + ld(cx + 2) * ld(ix + o)
                         - ld(cx + 3) * ld(ix + o - sI) + ld(cx + 4) * ld(ix + o - 2 * sI));
                oy[o] = (ld(cy) * ld(iy + o + 2 * sJ) - ld(cy + 1) * ld(iy + o + sJ) + ld(cy + 2) * ld(iy + o)
                         - ld(cy + 3) * ld(iy + o - sJ) + ld(cy + 4) * ld(iy + o - 2 * sJ));
            }
        }
    }
}

cudaError_t launch_numfilter_high(const Grid &g, const NdCoef &c, const NdArgs &a, double *w1, double *w2,
                                  cudaStream_t st)
{
    dim3 b(32, 4), gr((g.IMAX + 3) / 4, g.JMAX);
    const int nphi = (int)(((long)g.KA * g.IA * g.JA + PHI_THREADS - 1) / PHI_THREADS);
    const BatchT<1> one{1, {0, nphi}, {}};
    k_phi<double, 1><<<nphi, PHI_THREADS, 0, st>>>(g, a, one);
    k_nd_diff3<<<gr, b, 0, st>>>(g, c, a, w1);
    double *in = w1, *out = w2;
    for (int no = 2; no <= c.order; ++no) {
        double *f[15];
        for (int q = 0; q < 15; ++q) f[q] = in + (size_t)q * n3(g);
        periodic_halo(g, Members{}, f, 15, st); // COMM_vars8 of the work (:1557-1563)
        k_nd_diff4<<<gr, b, 0, st>>>(g, c, in, out);
        double *t = in;
        in = out;
        out = t;
    }
    const BatchT<1> oneN{1, {0, ((g.IMAX + 3) / 4) * g.JMAX}, {}};
    k_numfilter<double, 1, true><<<oneN.first[1], b, 0, st>>>(g, c, a, oneN, in);
    return cudaGetLastError();
}
#endif

template <typename R>
cudaError_t launch_numfilter(const Grid &g, const Members &mem, const NdCoef &c, const NdArgsT<R> &a, cudaStream_t st)
{
    auto nb_phi = [](const Grid &m) { return (int)(((long)m.KA * m.IA * m.JA + PHI_THREADS - 1) / PHI_THREADS); };
    auto nb_nd = [](const Grid &m) { return ((m.IMAX + 3) / 4) * m.JMAX; };
    with_batch(g, mem, nb_phi, [&](const auto &B, int nb) {
        k_phi<R, std::decay_t<decltype(B)>::NMAX><<<nb, PHI_THREADS, 0, st>>>(g, a, B);
        return cudaSuccess;
    });
    with_batch(g, mem, nb_nd, [&](const auto &B, int nb) {
        k_numfilter<R, std::decay_t<decltype(B)>::NMAX><<<nb, dim3(32, 4), 0, st>>>(g, c, a, B, nullptr);
        return cudaSuccess;
    });
    return cudaGetLastError();
}
#ifdef HEVI_FLOAT_TU
template cudaError_t launch_numfilter<float>(const Grid &, const Members &, const NdCoef &, const NdArgsT<float> &,
                                             cudaStream_t);
#else
template cudaError_t launch_numfilter<double>(const Grid &, const Members &, const NdCoef &, const NdArgsT<double> &,
                                              cudaStream_t);
#endif

}  // namespace hevi
