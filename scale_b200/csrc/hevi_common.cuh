// Shared device definitions for the B200 HEVI short-step kernels.
//
// Layout: every 3-D field is the reference's Fortran array (KA,IA,JA), k fastest,
// halo width 2 in every direction (scale_atmos_grid_cartesC_index.F90:256-265).
// Kernels use the reference's 1-based (k,i,j) indices so each expression can be
// checked against the Fortran line it restates.
//
// Arithmetic: FP64, compiled with --fmad=false, and each expression keeps the
// Fortran evaluation order, so the plain path reproduces the reference's
// IEEE-754 results operation by operation. Flat terrain is assumed by the
// fused kernels (GSQRT = 1, J13G = J23G = 0, MAPF = 1; classified by the host
// before any launch): the metric factors then multiply or divide by exactly 1
// and the J13/J23 flux terms are exact zeros, so dropping them leaves every
// non-zero value unchanged. Other metrics go to the general-metric stage
// (terrain_stage in hevi_stage.cu), which keeps every metric term.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace hevi {

// flux schemes (ATMOS_DYN_FVM_FLUX_TYPE names)
// (ATMOS_DYN_FVM_FLUX_TYPE / _TRACER_TYPE names: UD3, CD4, UD3KOREN1993, CD2)
enum Scheme : int { UD3 = 1, CD4 = 2, KOREN = 3, CD2 = 4, UD5 = 5, CD6 = 6 };
// the 6-point schemes, which read three points on each side (IHALO = JHALO = 3)
__host__ __device__ constexpr bool wide_scheme(int s) { return s == UD5 || s == CD6; }

struct Grid {
    int KA, IA, JA;
    int KS, KE, IS, IE, JS, JE;
    int KMAX, IMAX, JMAX;
    int IHALO, JHALO;
    int IEH, JEH;
    // device 1-D tables, 0-based storage of the 1-based reference arrays
    const double *CDZ, *FDZ, *RCDZ, *RFDZ;  // (KA), FDZ/RFDZ (KA-1)
    const double *F2H1, *F2H2;              // face weights CDZ(k)/(CDZ(k)+CDZ(k+1)), CDZ(k+1)/(...)
    const double *FDX, *RCDX, *RFDX;        // (IA)
    const double *FDY, *RCDY, *RFDY;        // (JA)
    // Ensemble pooling (all zero offsets for a single domain): the domain's
    // (KA,IA,JA) fields start at point cell0 of pooled arrays whose components
    // (num_diff(...,15), mflx_hi(...,3), ...) lie `stride` points apart; its
    // (IA,JA) fields start at c2 and its 1-D vectors at z0/x0/y0 of pooled
    // tables that hold each member's KA/IA/JA values back to back.
    int cell0, c2, z0, x0, y0;
    size_t stride;
};

__host__ __device__ __forceinline__ size_t idx3(const Grid &g, int k, int i, int j)
{
    return (size_t)g.cell0 + (size_t)(k - 1) + (size_t)g.KA * ((size_t)(i - 1) + (size_t)g.IA * (size_t)(j - 1));
}
// distance between the components of a multi-field array
__host__ __device__ __forceinline__ size_t n3(const Grid &g) { return g.stride; }

// ---- ensembles: members of different sizes advanced by the same launches ----
// Every kernel flattens its per-domain grid of blocks to one dimension and
// concatenates the members' block ranges; a block finds its member by a
// binary search over the range starts (kernel parameters, so the search reads
// the constant bank). NM = 1 compiles the single-domain form without it.
#ifndef HEVI_MAX_MEMBERS
#define HEVI_MAX_MEMBERS 64
#endif
struct MemberGeom {
    int KMAX, IMAX, JMAX;
    int z0, x0, y0;  // offsets of the member's 1-D vectors in the pooled tables
    int cell0, c2;   // offsets of its 3-D and 2-D fields in the pooled arrays
};
template <int NM>
struct BatchT {
    static constexpr int NMAX = NM;
    int n;             // members in this launch
    int first[NM + 1]; // first block of each member; first[n] = all blocks
    MemberGeom m[NM];
};

// the member's Grid: sizes, offsets and table pointers of member M (vertical
// halo 2; the lateral halo IHALO = JHALO of the pooled grid t, common to all members)
__host__ __device__ __forceinline__ Grid member_grid(const Grid &t, const MemberGeom &M)
{
    Grid g = t;
    const int H = t.IHALO;
    g.KMAX = M.KMAX; g.IMAX = M.IMAX; g.JMAX = M.JMAX;
    g.KA = M.KMAX + 4; g.IA = M.IMAX + 2 * H; g.JA = M.JMAX + 2 * H;
    g.KS = 3; g.KE = M.KMAX + 2; g.IS = H + 1; g.IE = M.IMAX + H; g.JS = H + 1; g.JE = M.JMAX + H;
    g.IHALO = H; g.JHALO = H; g.IEH = g.IE; g.JEH = g.JE;
    g.cell0 = M.cell0; g.c2 = M.c2; g.z0 = M.z0; g.x0 = M.x0; g.y0 = M.y0;
    g.CDZ = t.CDZ + M.z0; g.FDZ = t.FDZ + M.z0; g.RCDZ = t.RCDZ + M.z0; g.RFDZ = t.RFDZ + M.z0;
    g.F2H1 = t.F2H1 + M.z0; g.F2H2 = t.F2H2 + M.z0;
    g.FDX = t.FDX + M.x0; g.RCDX = t.RCDX + M.x0; g.RFDX = t.RFDX + M.x0;
    g.FDY = t.FDY + M.y0; g.RCDY = t.RCDY + M.y0; g.RFDY = t.RFDY + M.y0;
    return g;
}

// The domain of block x of a launch over all members, and its block index b
// within that domain.
template <int NM>
__device__ __forceinline__ Grid block_domain(const Grid &t, const BatchT<NM> &B, int &b, int x)
{
    if constexpr (NM == 1) {
        // a single domain has zero offsets; stating them lets them fold away
        b = x;
        Grid g = t;
        g.cell0 = 0; g.c2 = 0; g.z0 = 0; g.x0 = 0; g.y0 = 0;
        return g;
    } else {
        int lo = 0;
#pragma unroll
        for (int step = NM / 2; step > 0; step >>= 1)
            if (lo + step < B.n && B.first[lo + step] <= x) lo += step;
        b = x - B.first[lo];
        return member_grid(t, B.m[lo]);
    }
}
// this block's domain (block blockIdx.x of the launch)
template <int NM>
__device__ __forceinline__ Grid block_domain(const Grid &t, const BatchT<NM> &B, int &b)
{
    return block_domain(t, B, b, (int)blockIdx.x);
}

constexpr double GRAV = 9.80665;      // scale_const.F90:46
constexpr double EPS = 2.220446049250313080847263336181640625e-16; // epsilon(0.0_RP)

// SIGN(a,b) of Fortran = |a| with the sign bit of b
template <typename R>
__device__ __forceinline__ R fsign(R a, R b) { return copysign(fabs(a), b); }
__device__ __forceinline__ double fmax2(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double fmin2(double a, double b) { return a < b ? a : b; }

// value of a scalar of any arithmetic type of the kernels, for comparisons
template <typename R>
__device__ __forceinline__ double vof(const R &x) { return (double)x; }
template <typename R>
__device__ __forceinline__ R rmax(R a, R b) { return vof(a) > vof(b) ? a : b; }
template <typename R>
__device__ __forceinline__ R rmin(R a, R b) { return vof(a) < vof(b) ? a : b; }

// ---- UD3KOREN1993 (scale_atmos_dyn_fvm_flux_ud3Koren1993.F90) ----
// the Koren (1993) limiter phi (:1690-1710)
template <typename R>
__device__ __forceinline__ R koren_phi(R v1, R v2, R v3)
{
    const R eps = R(EPS);
    const R zerosw1 = eps - fsign(eps, fabs(v1 - v2) - eps);
    const R zerosw2 = eps - fsign(eps, fabs(v2 - v3) - eps);
    const R r2 = R(2.0) * (v1 - v2 + zerosw1 * zerosw2) / (v2 - v3 + zerosw2);
    return rmax(R(0.0), rmin(r2, rmin((R(1.0) + r2) / R(3.0), R(2.0))));
}

// ---- face interpolation of the flux schemes ----------------------------------
// UD3: scale_atmos_dyn_fvm_flux_ud3.F90:87-89,124-125 ; CD4: ..._cd4.F90:87-88,123-124;
// CD2: ..._cd2.F90 (F2*(v0+vp1) at every face); UD3KOREN1993: the limited
// upwind value of ..._ud3Koren1993.F90 (:200-206 interior, :236-241 above KS,
// :243-249 below KE). The face lies between v0 and vp1. R is the arithmetic
// type (double on the plain path; float for the flux arithmetic of the
// mixed-precision path; dual numbers and jets in the differentiated step).
template <int S, typename R>
__device__ __forceinline__ R ip4(R vel, R vm1, R v0, R vp1, R vp2)
{
    if constexpr (S == UD3) {
        const R F31 = R(-1.0 / 12.0), F32 = R(7.0 / 12.0), F33 = R(3.0 / 12.0);
        return (F31 * (vp2 + vm1) + F32 * (vp1 + v0)) - (F31 * (vp2 - vm1) + F33 * (vp1 - v0)) * fsign(R(1.0), vel);
    } else if constexpr (S == CD4) {
        const R F41 = R(7.0 / 12.0), F42 = R(-1.0 / 12.0);
        return F41 * (vp1 + v0) + F42 * (vp2 + vm1);
    } else if constexpr (S == CD2) {
        return R(0.5) * (vp1 + v0);
    } else {
        return (v0 + R(0.5) * koren_phi(vp1, v0, vm1) * (v0 - vm1)) * (R(0.5) + fsign(R(0.5), vel))
               + (vp1 + R(0.5) * koren_phi(v0, vp1, vp2) * (vp1 - vp2)) * (R(0.5) - fsign(R(0.5), vel));
    }
}
// value at the KS face from val(KS), val(KS+1), val(KS+2) (ud3.F90:142-145, cd4.F90:141;
// UD5 and CD6 use the UD3 and the F2 form, ud5.F90:162-165, cd6.F90:156)
template <int S, typename R>
__device__ __forceinline__ R ipL(R vel, R v0, R v1, R v2)
{
    if constexpr (S == UD3 || S == UD5)
        return R(0.5) * (v1 + v0) * (R(0.5) + fsign(R(0.5), vel))
               + (R(2.0) * v0 + R(5.0) * v1 - v2) / R(6.0) * (R(0.5) - fsign(R(0.5), vel));
    else if constexpr (S == KOREN)
        return v0 * (R(0.5) + fsign(R(0.5), vel))
               + (v1 + R(0.5) * koren_phi(v0, v1, v2) * (v1 - v2)) * (R(0.5) - fsign(R(0.5), vel));
    else
        return R(0.5) * (v1 + v0);
}
// value at the KE-1 face from val(KE), val(KE-1), val(KE-2) (ud3.F90:146-149, cd4.F90:142;
// ud5.F90:166-169, cd6.F90:157)
template <int S, typename R>
__device__ __forceinline__ R ipH(R vel, R vE, R vE1, R vE2)
{
    if constexpr (S == UD3 || S == UD5)
        return (R(2.0) * vE + R(5.0) * vE1 - vE2) / R(6.0) * (R(0.5) + fsign(R(0.5), vel))
               + R(0.5) * (vE + vE1) * (R(0.5) - fsign(R(0.5), vel));
    else if constexpr (S == KOREN)
        return (vE1 + R(0.5) * koren_phi(vE2, vE1, vE) * (vE1 - vE)) * (R(0.5) + fsign(R(0.5), vel))
               + vE * (R(0.5) - fsign(R(0.5), vel));
    else
        return R(0.5) * (vE + vE1);
}

// ---- 6-point schemes: UD5 (scale_atmos_dyn_fvm_flux_ud5.F90) and CD6 (..._cd6.F90),
// from the same generator template as UD3/CD4. Interior face value from two
// more points on each side (ud5.F90:92-96,133-138; cd6.F90:89-91,130-132); for
// the 4-point schemes ip6 is ip4 of the inner four points, whose callers then
// never read the outer two (they are compile-time dead).
template <int S, typename R>
__device__ __forceinline__ R ip6(R vel, R vm2, R vm1, R v0, R vp1, R vp2, R vp3)
{
    if constexpr (S == UD5) {
        const R F51 = R(1.0 / 60.0), F52 = R(-8.0 / 60.0), F53 = R(37.0 / 60.0), F54 = R(-5.0 / 60.0),
                F55 = R(10.0 / 60.0);
        return (F51 * (vp3 + vm2) + F52 * (vp2 + vm1) + F53 * (vp1 + v0))
               - (F51 * (vp3 - vm2) + F54 * (vp2 - vm1) + F55 * (vp1 - v0)) * fsign(R(1.0), vel);
    } else if constexpr (S == CD6) {
        const R F61 = R(37.0 / 60.0), F62 = R(-8.0 / 60.0), F63 = R(1.0 / 60.0);
        return F61 * (vp1 + v0) + F62 * (vp2 + vm1) + F63 * (vp3 + vm2);
    } else {
        return ip4<S>(vel, vm1, v0, vp1, vp2);
    }
}
// the KS+1 face of the 6-point schemes from val(KS..KS+4) (ud5.F90:171-177, cd6.F90:159-160)
template <int S, typename R>
__device__ __forceinline__ R ipL2(R vel, R v0, R v1, R v2, R v3, R v4)
{
    if constexpr (S == UD5)
        return (R(2.0) * v2 + R(5.0) * v1 - v0) / R(6.0) * (R(0.5) + fsign(R(0.5), vel))
               + (R(-3.0) * v0 + R(27.0) * v1 + R(47.0) * v2 - R(13.0) * v3 + R(2.0) * v4) / R(60.0)
                     * (R(0.5) - fsign(R(0.5), vel));
    else
        return R(7.0 / 12.0) * (v2 + v1) + R(-1.0 / 12.0) * (v3 + v0);
}
// the KE-2 face of the 6-point schemes from val(KE), ..., val(KE-4) (ud5.F90:179-185, cd6.F90:161-162)
template <int S, typename R>
__device__ __forceinline__ R ipH2(R vel, R vE, R vE1, R vE2, R vE3, R vE4)
{
    if constexpr (S == UD5)
        return (R(-3.0) * vE + R(27.0) * vE1 + R(47.0) * vE2 - R(13.0) * vE3 + R(2.0) * vE4) / R(60.0)
                   * (R(0.5) + fsign(R(0.5), vel))
               + (R(2.0) * vE2 + R(5.0) * vE1 - vE) / R(6.0) * (R(0.5) - fsign(R(0.5), vel));
    else
        return R(7.0 / 12.0) * (vE1 + vE2) + R(-1.0 / 12.0) * (vE + vE3);
}

// Face value at w-level m (between levels m and m+1) of a column; v(l) returns
// the value at level l. The near-wall forms: ipL at KS, ipH at KE-1, and for
// the 6-point schemes ipL2 at KS+1 and ipH2 at KE-2 (the interior loops are
// KS+1..KE-2 in ud3.F90/cd4.F90 and KS+2..KE-3 in ud5.F90/cd6.F90). Only the
// levels the chosen form needs are read.
template <int S, typename R, typename V>
__device__ __forceinline__ R zface(R vel, int m, int KS, int KE, const V &v)
{
    if (m == KS) return ipL<S>(vel, v(KS), v(KS + 1), v(KS + 2));
    if (m == KE - 1) return ipH<S>(vel, v(KE), v(KE - 1), v(KE - 2));
    if constexpr (wide_scheme(S)) {
        if (m == KS + 1) return ipL2<S>(vel, v(KS), v(KS + 1), v(KS + 2), v(KS + 3), v(KS + 4));
        if (m == KE - 2) return ipH2<S>(vel, v(KE), v(KE - 1), v(KE - 2), v(KE - 3), v(KE - 4));
        return ip6<S>(vel, v(m - 2), v(m - 1), v(m), v(m + 1), v(m + 2), v(m + 3));
    } else {
        return ip4<S>(vel, v(m - 1), v(m), v(m + 1), v(m + 2));
    }
}

// read-only load through the non-coherent cache
#if HEVI_COHERENT_LOADS
// ordinary global loads: the persistent short step reads fields that earlier
// phases of the same launch wrote (after a grid barrier), which the read-only
// path may not serve
template <typename T>
__device__ __forceinline__ T ld(const T *p) { return *p; }
#else
template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }
#endif

// device status word bits, read by the host after each call
enum StatusBits : unsigned {
    ST_NONFINITE = 1u << 0,   // a prognostic output is NaN/Inf
    ST_TMA_TIMEOUT = 1u << 1, // a bulk tensor copy did not complete within its wait limit
    ST_BARRIER_TIMEOUT = 1u << 2, // a grid barrier of the persistent short step did not complete within its wait limit
};

}  // namespace hevi
