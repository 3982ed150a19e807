// Device bodies of the numerical filter for ND_ORDER = 1 (ATMOS_DYN_numfilter_coef,
// scale_atmos_dyn_common.F90:385-985, with the third-difference operator
// calc_diff3 :1600-1760): the filtered quantities at one point (phi_point) and
// the 15 num_diff components of one column (numfilter_column). They take their
// block and thread indices as arguments, so that the filter kernels of
// numfilter.cu and the persistent short-step kernel run the same code.
#pragma once
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
// (block x of the launch over all members, thread t of PHI_THREADS)
template <typename R, int NM>
__device__ __forceinline__ void phi_point(const Grid &gt, const NdArgsT<R> &a, const BatchT<NM> &B, int x, int t)
{
    int b;
    const Grid g = block_domain(gt, B, b, x);
    // 32-bit index arithmetic: a field has fewer than 2^31 points (checked at setup)
    const unsigned npts = (unsigned)g.KA * g.IA * g.JA;
    const unsigned pt = (unsigned)b * PHI_THREADS + t;
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
    using type = R;
    const Grid &g;
    const NdArgsT<R> &a;
    __device__ R operator()(int q, int k, int i, int j) const
    {
        return ld(a.phi + (size_t)q * n3(g) + idx3(g, k, i, j));
    }
};

// calc_diff3 z-component with KO = 0 (:1617-1655) at level k (any k in 1..KA)
// (P: an accessor phi(q, k, i, j) of the filtered quantities, P::type their type)
template <class P>
__device__ __forceinline__ typename P::type dz0(const Grid &g, const NdCoef &c, const P &phi, int q, int k, int i, int j)
{
    using R = typename P::type;
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
template <class P>
__device__ __forceinline__ typename P::type dz1(const Grid &g, const NdCoef &c, const P &phi, int q, int k, int i, int j)
{
    using R = typename P::type;
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
template <class P>
__device__ __forceinline__ typename P::type dx(const Grid &g, const NdCoef &c, const P &phi, int q, int o, int k, int i, int j)
{
    using R = typename P::type;
    if (o == 0)
        return (+CX3(1, i + 1, 1) * phi(q, k, i + 2, j) - CX3(2, i + 1, 1) * phi(q, k, i + 1, j)
                + CX3(3, i + 1, 1) * phi(q, k, i, j) - CX3(1, i, 1) * phi(q, k, i - 1, j));
    return (+CX3(1, i, 2) * phi(q, k, i + 1, j) - CX3(2, i, 2) * phi(q, k, i, j)
            + CX3(3, i, 2) * phi(q, k, i - 1, j) - CX3(1, i - 1, 2) * phi(q, k, i - 2, j));
}
template <class P>
__device__ __forceinline__ typename P::type dy(const Grid &g, const NdCoef &c, const P &phi, int q, int o, int k, int i, int j)
{
    using R = typename P::type;
    if (o == 0)
        return (+CY3(1, j + 1, 1) * phi(q, k, i, j + 2) - CY3(2, j + 1, 1) * phi(q, k, i, j + 1)
                + CY3(3, j + 1, 1) * phi(q, k, i, j) - CY3(1, j, 1) * phi(q, k, i, j - 1));
    return (+CY3(1, j, 2) * phi(q, k, i, j + 1) - CY3(2, j, 2) * phi(q, k, i, j)
            + CY3(3, j, 2) * phi(q, k, i, j - 1) - CY3(1, j - 1, 2) * phi(q, k, i, j - 2));
}

// The 15 num_diff components of cell (k,i,j) at offset o, KS <= k <= KE: phi
// and dn are accessors of the filtered quantities and of the density around
// the cell (dn(dk, di, dj) = DENS(k+dk, i+di, j+dj)); the differences come
// from phi (FW = false) or from the work buffer W. ncx..nfy: the cell's x/y
// filter factors.
template <bool FW, class P, class D>
__device__ __forceinline__ void numfilter_cell(const Grid &g, const NdCoef &c, const P &phi, const D &dn,
                                               const double *W, typename P::type *ND, size_t N3, size_t o, int k,
                                               int i, int j, typename P::type ncx, typename P::type nfx,
                                               typename P::type ncy, typename P::type nfy, typename P::type sfc)
{
    using R = typename P::type;
    const int KS = g.KS, KE = g.KE;
    // surface-factor tail of every x/y component (:581-585 and the analogous blocks)
    auto sfct = [&](int kk, R v) {
        if (kk == KS) return v * sfc;
        if (kk == KS + 1) return v * (R(1.0) + sfc) * R(0.5);
        return v;
    };
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
            ND[o + N3 * 1] = kz1 ? DZ(1, dz1(g, c, phi, 1, k, i, j)) * nfz * R(dn(0, 0, 0)) : R(0.0);
            ND[o + N3 * 6] = kz ? sfct(k, DX(1, dx(g, c, phi, 1, 0, k, i, j)) * ncx
                                              * R(0.25) * (R(dn(1, 1, 0)) + R(dn(1, 0, 0)) + R(dn(0, 1, 0)) + R(dn(0, 0, 0))))
                                : R(0.0);
            ND[o + N3 * 11] = kz ? sfct(k, DY(1, dy(g, c, phi, 1, 0, k, i, j)) * ncy
                                               * R(0.25) * (R(dn(1, 0, 1)) + R(dn(1, 0, 0)) + R(dn(0, 0, 1)) + R(dn(0, 0, 0))))
                                 : R(0.0);
            break;
        }
        case 2: // ---- x momentum (:728-790), phi = VELX ----
            ND[o + N3 * 2] = kz ? DZ(2, dz0(g, c, phi, 2, k, i, j)) * ncz
                                      * R(0.25) * (R(dn(1, 1, 0)) + R(dn(1, 0, 0)) + R(dn(0, 1, 0)) + R(dn(0, 0, 0)))
                                : R(0.0);
            ND[o + N3 * 7] = sfct(k, DX(2, dx(g, c, phi, 2, 1, k, i, j)) * nfx * R(dn(0, 0, 0)));
            ND[o + N3 * 12] = sfct(k, DY(2, dy(g, c, phi, 2, 0, k, i, j)) * ncy
                                          * R(0.25) * (R(dn(0, 1, 1)) + R(dn(0, 1, 0)) + R(dn(0, 0, 1)) + R(dn(0, 0, 0))));
            break;
        case 3: // ---- y momentum (:812-870), phi = VELY ----
            ND[o + N3 * 3] = kz ? DZ(3, dz0(g, c, phi, 3, k, i, j)) * ncz
                                      * R(0.25) * (R(dn(1, 0, 1)) + R(dn(1, 0, 0)) + R(dn(0, 0, 1)) + R(dn(0, 0, 0)))
                                : R(0.0);
            ND[o + N3 * 8] = sfct(k, DX(3, dx(g, c, phi, 3, 0, k, i, j)) * ncx
                                         * R(0.25) * (R(dn(0, 1, 1)) + R(dn(0, 0, 1)) + R(dn(0, 1, 0)) + R(dn(0, 0, 0))));
            ND[o + N3 * 13] = sfct(k, DY(3, dy(g, c, phi, 3, 1, k, i, j)) * nfy * R(dn(0, 0, 0)));
            break;
        default: { // ---- rho*theta (:885-960) ----
            const R v = DZ(4, dz0(g, c, phi, 4, k, i, j)) * ncz;
            ND[o + N3 * 4] = kz ? v * R(0.5) * (R(dn(1, 0, 0)) + R(dn(0, 0, 0))) : v * R(dn(0, 0, 0));
            ND[o + N3 * 9] = sfct(k, DX(4, dx(g, c, phi, 4, 0, k, i, j)) * ncx * R(0.5) * (R(dn(0, 1, 0)) + R(dn(0, 0, 0))));
            ND[o + N3 * 14] = sfct(k, DY(4, dy(g, c, phi, 4, 0, k, i, j)) * ncy * R(0.5) * (R(dn(0, 0, 1)) + R(dn(0, 0, 0))));
        }
        }
    }
#undef DZ
#undef DX
#undef DY
}

// density around cell o of a global array
struct DensG {
    const double *p;
    long sI, sJ;
    __device__ double operator()(int dk, int di, int dj) const { return ld(p + dk + di * sI + dj * sJ); }
};

// The vertical halo levels 1..KS-1 and KE+1..KA of column (i,j), one lane per
// level: zero, except density and theta z at KS-1 (the mirror -atKS of level KS)
template <bool FW, class P>
__device__ __forceinline__ void numfilter_halo_levels(const Grid &g, const NdCoef &c, const P &phi, const double *W,
                                                      typename P::type *ND, size_t N3, const double *DN, int i, int j,
                                                      int lane)
{
    using R = typename P::type;
    const int KS = g.KS, KE = g.KE;
    const int nlo = KS - 1, nh = nlo + (g.KA - KE);
    for (int h = lane; h < nh; h += 32) {
        const int k = h < nlo ? h + 1 : KE + 1 + (h - nlo);
        const size_t o = idx3(g, k, i, j);
        for (int q = 0; q < 15; ++q) ND[o + N3 * q] = R(0.0);
        if (k == KS - 1) {
            const R ncz = R(ld(c.cdz + k - 1));
            const R d0 = FW ? R(ld(W + (size_t)0 * N3 + o)) : dz0(g, c, phi, 0, k, i, j);
            const R d4 = FW ? R(ld(W + (size_t)12 * N3 + o)) : dz0(g, c, phi, 4, k, i, j);
            ND[o + N3 * 0] = d0 * ncz;
            ND[o + N3 * 4] = d4 * ncz * R(R(ld(DN + idx3(g, KS, i, j))));
        }
    }
}

// FW: the differences come from the calc_numdiff work buffer W (ND_ORDER > 1)
// instead of being formed from phi here (ND_ORDER = 1)
//
// The lanes of a warp take the levels KS..KE of one column, so that every
// pass over 32 levels but the last is full; the halo levels (zero, except the
// mirrors at KS-1 of density and theta) are written by a short tail pass.
// A block of the launch is ND_WARPS warps over consecutive columns of one row:
// block x of the launch over all members, warp wy of the block, lane lane.
constexpr int ND_WARPS = 4;
template <typename R, int NM, bool FW>
__device__ __forceinline__ void numfilter_column(const Grid &gt, const NdCoef &ct, const NdArgsT<R> &a,
                                                 const BatchT<NM> &B, const double *W, int x, int wy, int lane)
{
    int b;
    const Grid g = block_domain(gt, B, b, x);
    const NdCoef c = NM == 1 ? ct : member_nd(ct, g);
    const Block2 p = split_block(b, (g.IMAX + ND_WARPS - 1) / ND_WARPS);
    const int i = g.IS + p.x * ND_WARPS + wy;
    const int j = g.JS + p.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g);
    const int KS = g.KS, KE = g.KE;
    const Phi<R> phi{g, a};
    const double *DN = a.DENS;
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const R ncx = R(ld(c.cdx + i - 1)), nfx = R(ld(c.fdx + i - 1)), ncy = R(ld(c.cdy + j - 1)), nfy = R(ld(c.fdy + j - 1));
    const R sfc = R(c.sfc);
    R *ND = a.num_diff;
    for (int k = KS + lane; k <= KE; k += 32) {
        const size_t o = idx3(g, k, i, j);
        numfilter_cell<FW>(g, c, phi, DensG{DN + o, sI, sJ}, W, ND, N3, o, k, i, j, ncx, nfx, ncy, nfy, sfc);
    }
    numfilter_halo_levels<FW>(g, c, phi, W, ND, N3, DN, i, j, lane);
}

}  // namespace hevi
