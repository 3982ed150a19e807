// One HEVI short-step stage (ATMOS_DYN_Tstep_short_fvm_hevi,
// scalelib/src/atmos-rm/dynamics/scale_atmos_dyn_tstep_short_fvm_hevi.F90:128-1089)
// as one kernel, k_hevi_stage.
//
// A CTA owns a tile of TX x TY columns over all levels. A column is KA
// contiguous doubles, so each warp works on one column with its lanes along k
// (256-byte coalesced accesses); horizontal neighbours are other columns, read
// through L1/L2, or from shared memory when they lie in the tile. Per-level values of the vertical implicit
// problem live in shared memory ([quantity][column][level], odd pitch):
//   1. POTT = RHOT/DENS; x/y mass fluxes and the mass source Sr; A(k)      (k-parallel)
//   2. PT (theta at w-faces), vertical and x/y theta fluxes, St             (k-parallel)
//   3. x/y w-momentum fluxes, Sw and the right-hand side C(k) (:698-722)    (k-parallel)
//   4. warp 0: Thomas solve, one lane per column (solve_direct :1092-1127);
//      the other warps meanwhile update rho*u and rho*v (hevi_momx :814-928,
//      hevi_momy :934-1048), which do not depend on the solve
//   5. back-update of rho, rho*w, rho*theta and the vertical fluxes (:728-790)
// Every value keeps the reference's operation order, so the stage is
// bit-identical to the sequential formulation.
//
// The kernel is a template on R, the type of the flux arithmetic and of the
// flux-like arrays (num_diff, tendencies, DDIV, mflx_hi/tflx_hi, their RK sums,
// the column-solve sources). R = double is the plain path above. R = float is
// the mixed-precision path: fluxes and divergences in FP32, while the state,
// the pressure and density deviations from the base state, the right-hand
// side and the Thomas solve stay FP64. Every FP64 operand is converted with
// R(...) at its use, which is the identity for R = double.
//
// k_hevi_stage takes flat terrain (see hevi_common.cuh); the general-metric
// stage at the end of this file takes any GSQRT/J13G/J23G/MAPF. Line numbers below refer to the
// reference HEVI file unless a flux file is named.
#include "hevi_stage_body.cuh"

namespace hevi {

template <int S, typename R, int TX, int NM>
__global__ void __launch_bounds__(32 * HEVI_COL_TC, HEVI_COL_MINB)
    k_hevi_stage(const Grid gt, const StageArgsT<R> a, const BatchT<NM> B)
{
    hevi_stage_block<S, R, TX, NM>(gt, a, B, (int)blockIdx.x);
}
#ifndef HEVI_FLOAT_TU // the FP64-only kernels live in the FP64 translation unit
// =============================================================================
// the HEVE stage (ATMOS_DYN_Tstep_short_fvm_heve, scale_atmos_dyn_tstep_short_fvm_heve.F90:109-1518,
// without the momentum/theta FCT branches): every tendency is explicit, so each
// warp updates one column, lanes along k, with no column solve. The rho*u and
// rho*v updates are the HEVI ones (the two modules write them alike up to the
// divergence-damping term); the vertical mass flux is the explicit
// J33G * MOMZ + num_diff (:460-479), and the theta flux, the pressure gradient
// and the buoyancy of rho*w follow :622-688 and :1328-1371. Line numbers refer
// to the HEVE file. FP64, flat terrain as in the HEVI kernel.
// =============================================================================
constexpr int HEVE_WARPS = 4; // columns (warps) per CTA
#ifndef HEVE_MINB
#define HEVE_MINB 8 // resident CTAs per SM the register allocator must allow (32 warps)
#endif

template <int S, int NM>
__global__ void __launch_bounds__(32 * HEVE_WARPS, HEVE_MINB)
    k_heve_stage(const Grid gt, const StageArgsT<double> a, const BatchT<NM> B)
{
    using R = double;
    __shared__ double spott[HEVE_WARPS][MAXKA]; // POTT of each warp's column
    int b;
    const Grid g = block_domain(gt, B, b);
    const Block2 p = split_block(b, (g.IMAX + HEVE_WARPS - 1) / HEVE_WARPS);
    const int lane = threadIdx.x, w = threadIdx.y;
    const int i = g.IS + p.x * HEVE_WARPS + w, j = g.JS + p.y;
    if (i > g.IE) return; // warp-uniform; the kernel has no block-wide barrier
    const size_t N3 = n3(g);
    const int sI = g.KA, sJ = g.KA * g.IA;
    const int KS = g.KS, KE = g.KE;
    const int col = (int)idx3(g, 1, i, j);
    const Nd<R> nd(a, N3);
    const double dt = a.dtrk, J33G = a.J33G;
    const bool use_div = a.divdmp_coef != 0.0;
    const R ddc = use_div ? R(a.divdmp_coef / dt) : R(0.0);
    const R rcdx = ld(g.RCDX + i - 1), rcdy = ld(g.RCDY + j - 1);
    constexpr bool W6 = wide_scheme(S);
    const unsigned FULL = 0xffffffffu;
    double *P = spott[w];

    // potential temperature of the column, :375-382
    for (int L = KS + lane; L <= KE; L += 32) P[L - 1] = ld(a.RHOT + col + L - 1) / ld(a.DENS + col + L - 1);
    __syncwarp();
    auto pott = [&](int l) { return P[l - 1]; };
    // the explicit vertical mass flux at w-level m (zero at KS-1 and KE), :460-479 (flat terrain)
    auto mflx_z = [&](int m) -> R {
        if (m < KS || m > KE - 1) return R(0.0);
        return J33G * ld(a.MOMZ + col + m - 1) + ld(nd.DZ() + col + m - 1);
    };
    // theta flux at w-level m, fluxZ_XYZ (ud3.F90:157-247)
    auto tflx_z = [&](int m) -> R {
        if (m < KS || m > KE - 1) return R(0.0);
        const R vel = mflx_z(m);
        return vel * zface<S>(vel, m, KS, KE, pott) + ld(nd.TZ() + col + m - 1);
    };
    // w-momentum flux at level m (between w-levels m-1 and m... as fluxZ_XYW writes flux(m)), zero outside KS..KE-2
    auto qz_w = [&](int m) -> R {
        if (m < KS || m > KE - 2) return R(0.0);
        const R Mk = ld(a.MOMZ + col + m - 1), Mk1 = ld(a.MOMZ + col + m);
        const R vel = (R(0.5) * (Mk + Mk1)) / R(ld(a.DENS + col + m));
        const R q = zface<S>(vel, m, KS, KE, [&](int l) { return R(ld(a.MOMZ + col + l - 1)); });
        return R(J33G) * vel * q + ld(nd.WZ() + col + m);
    };
    auto dpres = [&](int c) { return ld(a.DPRES0 + c) + ld(a.RT2P + c) * (ld(a.RHOT + c) - ld(a.REF_rhot + c)); };
    // POTT of a horizontal neighbour column
    auto pott_at = [&](int c) { return ld(a.RHOT + c) / ld(a.DENS + c); };

    for (int L0 = KS; L0 <= KE; L0 += 32) {
        const int L = L0 + lane;
        const bool valid = L <= KE;
        const int c = col + L - 1;
        // z fluxes through the face above each level; the face below is the previous lane's
        const R mz = valid ? mflx_z(L) : R(0.0), tz = valid ? tflx_z(L) : R(0.0), qz = valid ? qz_w(L) : R(0.0);
        R mzm = __shfl_up_sync(FULL, mz, 1), tzm = __shfl_up_sync(FULL, tz, 1), qzm = __shfl_up_sync(FULL, qz, 1);
        if (lane == 0) { mzm = mflx_z(L - 1); tzm = tflx_z(L - 1); qzm = qz_w(L - 1); }
        if (valid) {
            const R rcdz = ld(g.RCDZ + L - 1);
            // ---- density, :460-532 ----
            const MassFlux<R> m = mass_flux(a, nd, c, sI, sJ);
            {
                const R advcv = -(mz - mzm) * rcdz;
                const R advch = -(m.Xe - m.Xw) * rcdx - (m.Yn - m.Ys) * rcdy;
                put_state(a, N3, 0, a.DENS_RK, a.DENS0, c, ld(a.DENS0 + c) + dt * ((advcv + advch) + ld(a.DENS_t + c)), true);
            }
            put_flux(a, N3, 0, c, mz, true);
            put_flux(a, N3, 1, c, m.Xe, true);
            put_flux(a, N3, 2, c, m.Yn, true);
            if (i == g.IS) put_flux(a, N3, 1, c - sI, m.Xw, false);
            if (j == g.JS) put_flux(a, N3, 2, c - sJ, m.Ys, false);
            // ---- rho*theta, :1328-1371 ----
            {
                const R P00 = P[L - 1];
                auto px = [&](int d) { return d == 0 ? P00 : pott_at(c + d * sI); };
                auto py = [&](int d) { return d == 0 ? P00 : pott_at(c + d * sJ); };
                const R Pm3 = W6 ? px(-3) : R(0.0), Pp3 = W6 ? px(3) : R(0.0);
                const R Qm3 = W6 ? py(-3) : R(0.0), Qp3 = W6 ? py(3) : R(0.0);
                const R Pm2 = px(-2), Pm1 = px(-1), Pp1 = px(1), Pp2 = px(2);
                const R Qm2 = py(-2), Qm1 = py(-1), Qp1 = py(1), Qp2 = py(2);
                const R tXe = m.Xe * ip6<S>(m.Xe, Pm2, Pm1, P00, Pp1, Pp2, Pp3) + ld(nd.TX() + c);
                const R tXw = m.Xw * ip6<S>(m.Xw, Pm3, Pm2, Pm1, P00, Pp1, Pp2) + ld(nd.TX() + c - sI);
                const R tYn = m.Yn * ip6<S>(m.Yn, Qm2, Qm1, P00, Qp1, Qp2, Qp3) + ld(nd.TY() + c);
                const R tYs = m.Ys * ip6<S>(m.Ys, Qm3, Qm2, Qm1, P00, Qp1, Qp2) + ld(nd.TY() + c - sJ);
                const R advcv = -(tz - tzm) * rcdz;
                const R advch = -(tXe - tXw) * rcdx - (tYn - tYs) * rcdy;
                put_state(a, N3, 4, a.RHOT_RK, a.RHOT0, c, ld(a.RHOT0 + c) + dt * ((advcv + advch) + ld(a.RHOT_t + c)), true);
                put_flux(a, N3, 3, c, tz, true);
                put_flux(a, N3, 4, c, tXe, true);
                put_flux(a, N3, 5, c, tYn, true);
                if (i == g.IS) put_flux(a, N3, 4, c - sI, tXw, false);
                if (j == g.JS) put_flux(a, N3, 5, c - sJ, tYs, false);
            }
            // ---- rho*w, :586-688 ----
            if (L <= KE - 1) {
                const R advcv = -(qz - qzm) * R(ld(g.RFDZ + L - 1));
                const R advch = adv_w_h<S>(g, a, nd, c, L, sI, sJ, rcdx, rcdy);
                const R pgf = J33G * (dpres(c + 1) - dpres(c)) * ld(g.RFDZ + L - 1);
                const R buoy = GRAV * (ld(g.F2H1 + L - 1) * (ld(a.DENS + c + 1) - ld(a.REF_dens + c + 1))
                                       + ld(g.F2H2 + L - 1) * (ld(a.DENS + c) - ld(a.REF_dens + c)));
                const R wdamp = -ld(a.wdamp + g.z0 + L - 1) * ld(a.MOMZ0 + c);
                const R div = use_div ? ddc * R(ld(g.FDZ + L - 1)) * (ld(a.DDIV + c + 1) - ld(a.DDIV + c)) : R(0.0);
                const double val = ld(a.MOMZ0 + c) + dt * ((((advcv + advch) - pgf) - buoy) + wdamp + div + ld(a.MOMZ_t + c));
                put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, val, true);
            } else {
                put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, 0.0, false);
            }
        }
        // ---- rho*u and rho*v, :819-1170 (all 32 lanes take part: the updates shuffle) ----
        update_mom<S, 0, R, true>(g, a, nd, N3, L, i, j, valid);
        update_mom<S, 1, R, true>(g, a, nd, N3, L, i, j, valid);
    }
    if (lane == 0) {
        // MOMZ_RK(KS-1) and the zero fluxes through the surface
        put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, col + KS - 2, 0.0, false);
        put_flux(a, N3, 0, col + KS - 2, R(0.0), false);
        put_flux(a, N3, 3, col + KS - 2, R(0.0), false);
    }
}

template <int S, int NM>
static cudaError_t launch_heve_one(const Grid &g, const StageArgsT<double> &a, const BatchT<NM> &B, int nblocks,
                                   cudaStream_t st)
{
    k_heve_stage<S, NM><<<nblocks, dim3(32, HEVE_WARPS), 0, st>>>(g, a, B);
    return cudaGetLastError();
}

cudaError_t launch_heve_stage(const Grid &g, const Members &mem, const StageArgsT<double> &a, int scheme,
                              cudaStream_t st)
{
    int maxKA = g.KA;
    for (int q = 0; q < mem.n; ++q) maxKA = mem.m[q].KMAX + 4 > maxKA ? mem.m[q].KMAX + 4 : maxKA;
    if (maxKA > MAXKA) return cudaErrorInvalidValue;
    auto nblocks = [](const Grid &m) { return ((m.IMAX + HEVE_WARPS - 1) / HEVE_WARPS) * m.JMAX; };
    return with_batch(g, mem, nblocks, [&](const auto &B, int nb) -> cudaError_t {
        constexpr int NM = std::decay_t<decltype(B)>::NMAX;
        switch (scheme) {
        case UD3: return launch_heve_one<UD3, NM>(g, a, B, nb, st);
        case CD4: return launch_heve_one<CD4, NM>(g, a, B, nb, st);
        case KOREN: return launch_heve_one<KOREN, NM>(g, a, B, nb, st);
        case CD2: return launch_heve_one<CD2, NM>(g, a, B, nb, st);
        case UD5: return launch_heve_one<UD5, NM>(g, a, B, nb, st);
        case CD6: return launch_heve_one<CD6, NM>(g, a, B, nb, st);
        default: return cudaErrorInvalidValue;
        }
    });
}
#endif // HEVI_FLOAT_TU

#undef AT
#undef AR

// ---- host launcher ----------------------------------------------------------
// Opens the dynamic shared memory of a kernel instantiation to the per-CTA
// maximum, once per device (keeps later launches free of non-stream calls,
// e.g. inside a graph capture).
template <class K>
static cudaError_t allow_smem(K kern)
{
    static std::pair<const void *, int> done[64];
    static int ndone = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    for (int q = 0; q < ndone; ++q)
        if (done[q].first == (const void *)kern && done[q].second == dev) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e == cudaSuccess && ndone < 64) done[ndone++] = {(const void *)kern, dev};
    return e;
}

template <int S, typename R, int TX, int NM>
static cudaError_t launch_one(const Grid &g, StageArgsT<R> a, const BatchT<NM> &B, int nblocks, size_t smem,
                              int raster, cudaStream_t st)
{
    auto kern = k_hevi_stage<S, R, TX, NM>;
    cudaError_t e = allow_smem(kern);
    if (e != cudaSuccess) return e;
    a.raster = raster > 0 ? raster : STAGE_RASTER_DEFAULT;
    kern<<<nblocks, dim3(32, HEVI_COL_TC), smem, st>>>(g, a, B);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_hevi_stage(const Grid &g, const Members &mem, const StageArgsT<R> &a, int scheme,
                              StageShape shape, cudaStream_t st, int *launches, bool *tiled)
{
    if (launches) *launches = 1;
    if (tiled) *tiled = false;
    if (shape.tile_x == 0) {
        const cudaError_t e = launch_hevi_stage_tiled(g, mem, a, scheme, shape.raster, st);
        if (e != cudaErrorNotSupported) {
            if (tiled) *tiled = true;
            return e;
        }
    }
    int maxKA = g.KA;
    for (int q = 0; q < mem.n; ++q) maxKA = mem.m[q].KMAX + 4 > maxKA ? mem.m[q].KMAX + 4 : maxKA;
    if (maxKA > MAXKA) return cudaErrorInvalidValue;
    const size_t smem = (size_t)COL_ARRAYS * HEVI_COL_TC * col_pitch(maxKA) * sizeof(double);
    const int tx = shape.tile_x > 0 ? shape.tile_x : STAGE_TILE_X_DEFAULT;
    auto go = [&](auto tile, const auto &B, int nb) -> cudaError_t {
        constexpr int TX = decltype(tile)::value, NM = std::decay_t<decltype(B)>::NMAX;
        switch (scheme) {
        case UD3: return launch_one<UD3, R, TX, NM>(g, a, B, nb, smem, shape.raster, st);
        case CD4: return launch_one<CD4, R, TX, NM>(g, a, B, nb, smem, shape.raster, st);
        case KOREN: return launch_one<KOREN, R, TX, NM>(g, a, B, nb, smem, shape.raster, st);
        case CD2: return launch_one<CD2, R, TX, NM>(g, a, B, nb, smem, shape.raster, st);
        case UD5: return launch_one<UD5, R, TX, NM>(g, a, B, nb, smem, shape.raster, st);
        case CD6: return launch_one<CD6, R, TX, NM>(g, a, B, nb, smem, shape.raster, st);
        default: return cudaErrorInvalidValue;
        }
    };
    auto dispatch = [&](auto tile) {
        constexpr int TX = decltype(tile)::value, TY = HEVI_COL_TC / TX;
        auto nblocks = [](const Grid &m) { return ((m.IMAX + TX - 1) / TX) * ((m.JMAX + TY - 1) / TY); };
        return with_batch(g, mem, nblocks, [&](const auto &B, int nb) { return go(tile, B, nb); });
    };
    switch (tx) {
    case 16: return dispatch(std::integral_constant<int, 16>{});
    case 8: return dispatch(std::integral_constant<int, 8>{});
    case 4: return dispatch(std::integral_constant<int, 4>{});
    default: return cudaErrorInvalidValue;
    }
}
#ifdef HEVI_FLOAT_TU
template cudaError_t launch_hevi_stage<float>(const Grid &, const Members &, const StageArgsT<float> &, int,
                                              StageShape, cudaStream_t, int *, bool *);
#else
template cudaError_t launch_hevi_stage<double>(const Grid &, const Members &, const StageArgsT<double> &, int,
                                               StageShape, cudaStream_t, int *, bool *);

// =============================================================================
// The HEVI stage with terrain-following metrics (GSQRT, J13G, J23G) and map
// factors (MAPF): ATMOS_DYN_Tstep_short_fvm_hevi (:128-1089) with every metric
// term, each loop nest of the reference one launch over its own (i,j) range,
// lanes along k, the intermediate fields in device work arrays. The flux
// routines are those of scale_atmos_dyn_fvm_flux_ud3.F90 (and the other
// scheme files), restated with their metric arguments. The outputs go through
// put_state/put_flux, so the RK4/RK3 folds of the fused kernel apply unchanged.
// FP64, one domain.
// =============================================================================
// at least 10 CTAs per SM (51 registers): the loop nests are bound by load
// latency, and unbounded they took 29-90 registers (5 CTAs per SM for the
// largest); 512x512x128 CD4 terrain short step 81.1 -> 75.4 ms (8 CTAs 77.4,
// 12 CTAs 78.9)
#ifndef HEVI_GCOLS_MINB
#define HEVI_GCOLS_MINB 10
#endif
template <class F>
__global__ void __launch_bounds__(128, HEVI_GCOLS_MINB) k_gcols(int i0, int ni, int j0, int ncol, F f)
{
    const int col = blockIdx.x * 4 + threadIdx.y;
    if (col >= ncol) return;
    f(i0 + col % ni, j0 + col / ni, (int)threadIdx.x);
}
// f(i, j, lane) for every column of i0..i1 x j0..j1, one warp per column
template <class F>
static void gcols(int i0, int i1, int j0, int j1, cudaStream_t st, F f)
{
    const int ni = i1 - i0 + 1, ncol = ni * (j1 - j0 + 1);
    if (ni <= 0 || ncol <= 0) return;
    k_gcols<<<(ncol + 3) / 4, dim3(32, 4), 0, st>>>(i0, ni, j0, ncol, f);
}

// solve_direct (tstep_short_fvm_hevi.F90:1092-1127) of the general-metric
// stage: a warp per column stages F1, F2, F3 and C of its column in shared
// memory (coalesced), lane 0 runs the recurrence there, the lanes store the
// solution back. Shared memory: 4 columns x 6 arrays x KA doubles per block.
__global__ void __launch_bounds__(128) k_terrain_solve(const Grid g, const TerrainWork W)
{
    extern __shared__ double sh[];
    const int KA = g.KA, KS = g.KS, KE = g.KE, ni = g.IMAX, ncol = g.IMAX * g.JMAX;
    const int w = threadIdx.y, lane = threadIdx.x;
    const int col = blockIdx.x * 4 + w;
    if (col >= ncol) return; // warp-uniform
    const int i = g.IS + col % ni, j = g.JS + col / ni;
    // level k at index k-1
    double *F1 = sh + (size_t)w * 6 * KA, *F2 = F1 + KA, *F3 = F2 + KA, *C = F3 + KA, *e = C + KA, *f = e + KA;
    const size_t c1 = idx3(g, 1, i, j);
    for (int k = KS + lane; k <= KE - 1; k += 32) {
        F1[k - 1] = W.F1[c1 + k - 1];
        F2[k - 1] = W.F2[c1 + k - 1];
        F3[k - 1] = W.F3[c1 + k - 1];
        C[k - 1] = W.C[c1 + k - 1];
    }
    __syncwarp();
    if (lane == 0) {
        double rdenom = 1.0 / F2[KS - 1];
        e[KS - 1] = -F1[KS - 1] * rdenom;
        f[KS - 1] = C[KS - 1] * rdenom;
        for (int k = KS + 1; k <= KE - 2; ++k) {
            rdenom = 1.0 / (F2[k - 1] + F3[k - 1] * e[k - 2]);
            e[k - 1] = -F1[k - 1] * rdenom;
            f[k - 1] = (C[k - 1] - F3[k - 1] * f[k - 2]) * rdenom;
        }
        C[KE - 2] = (C[KE - 2] - F3[KE - 2] * f[KE - 3]) / (F2[KE - 2] + F3[KE - 2] * e[KE - 3]);
        for (int k = KE - 2; k >= KS; --k) C[k - 1] = e[k - 1] * C[k] + f[k - 1];
    }
    __syncwarp();
    for (int k = KS + lane; k <= KE - 1; k += 32) W.C[c1 + k - 1] = C[k - 1];
}

static void terrain_solve(const Grid &g, const TerrainWork &W, cudaStream_t st)
{
    const int ncol = g.IMAX * g.JMAX;
    const size_t smem = (size_t)4 * 6 * g.KA * sizeof(double);
    // above 48 KB (KA > 256) the opt-in size is needed; a failure shows in the
    // launch error the caller returns
    (void)allow_smem(k_terrain_solve);
    k_terrain_solve<<<(ncol + 3) / 4, dim3(32, 4), smem, st>>>(g, W);
}

// a field that no kernel of the stage writes: elements through the read-only
// cache (so loads shared by several expressions are formed once), pointer
// arithmetic as for the plain pointer
struct RoField {
    const double *p;
    __device__ double operator[](size_t q) const { return __ldg(p + q); }
    __device__ const double *operator+(size_t q) const { return p + q; }
};

// face value between p[0] and p[s] along a horizontal direction of stride s
template <int S>
__device__ __forceinline__ double hface(double vel, const double *p, long s)
{
    if constexpr (wide_scheme(S)) return ip6<S>(vel, p[-2 * s], p[-s], p[0], p[s], p[2 * s], p[3 * s]);
    else return ip4<S>(vel, p[-s], p[0], p[s], p[2 * s]);
}

// staggering ids (scale_atmos_grid_cartesC_index.F90:90-101), variable ids and directions
enum : int { I_XYZ = 1, I_XYW, I_UYW, I_XVW, I_UYZ, I_XVZ, I_UVZ };
enum : int { I_XY = 1, I_UY, I_XV, I_UV };
enum : int { V_DENS = 1, V_MOMZ, V_MOMX, V_MOMY, V_RHOT };
enum : int { DZIR = 1, DXIR, DYIR };

template <int S>
static void terrain_stage(const Grid &g, const StageArgsT<double> &a, const Metrics &M, const TerrainWork &W,
                          cudaStream_t st)
{
    const int KS = g.KS, KE = g.KE, IS = g.IS, IE = g.IE, JS = g.JS, JE = g.JE;
    const int IEH = g.IEH < IE ? g.IEH : IE, JEH = g.JEH < JE ? g.JEH : JE;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const double dt = a.dtrk, J33G = a.J33G;
    const bool use_div = a.divdmp_coef != 0.0;
#define X3(k, i, j) idx3(g, k, i, j)
#define GSs(idx) (M.GSQRT + (size_t)((idx) - 1) * N3)
#define J13s(idx) (M.J13G + (size_t)((idx) - 1) * N3)
#define J23s(idx) (M.J23G + (size_t)((idx) - 1) * N3)
#define GS(k, i, j, idx) ld(GSs(idx) + X3(k, i, j))
#define J13(k, i, j, idx) ld(J13s(idx) + X3(k, i, j))
#define J23(k, i, j, idx) ld(J23s(idx) + X3(k, i, j))
#define MAPFv(i, j, aa, bb) \
    ld(M.MAPF + ((size_t)((i) - 1) + (size_t)g.IA * ((size_t)((j) - 1) + (size_t)g.JA * ((size_t)((aa) - 1) + 2 * (size_t)((bb) - 1)))))
#define NDp(v, dir) (a.num_diff + N3 * (size_t)(((v) - 1) + 5 * ((dir) - 1)))
#define CDZv(k) ld(g.CDZ + (k) - 1)
    // F2H(k,p) of a GSQRT slice Gs (ud3.F90:75, tstep_short_fvm_hevi.F90:62)
#define F2Hg(Gs, k, p) (CDZv((k) + (p) - 1) * ld((Gs) + X3((k) + (p) - 1, i, j)) \
                        / (CDZv(k) * ld((Gs) + X3(k, i, j)) + CDZv((k) + 1) * ld((Gs) + X3((k) + 1, i, j))))
    const RoField DN{a.DENS}, MZ{a.MOMZ}, MX{a.MOMX}, MY{a.MOMY}; // the stage input, read-only here

    // ---- hevi_pres :343-361 ----
    gcols(IS, IE + 1, JS, JE + 1, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            W.DPRES[c] = a.DPRES0[c] + a.RT2P[c] * (a.RHOT[c] - a.REF_rhot[c]);
        }
        if (lane == 0) {
            W.DPRES[X3(KS - 1, i, j)] = a.DPRES0[X3(KS - 1, i, j)] - DN[X3(KS, i, j)] * (M.PHI[X3(KS - 1, i, j)] - M.PHI[X3(KS + 1, i, j)]);
            W.DPRES[X3(KE + 1, i, j)] = a.DPRES0[X3(KE + 1, i, j)] - DN[X3(KE, i, j)] * (M.PHI[X3(KE + 1, i, j)] - M.PHI[X3(KE - 1, i, j)]);
        }
    });
    // ---- hevi_mflx_z :365-397 (the halo column IS-1 is an output too) ----
    gcols(IS - 1, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const bool in = i >= IS;
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double v = J13(k, i, j, I_XYW) * 0.25 / MAPFv(i, j, 2, I_XY)
                                 * (MX[X3(k + 1, i, j)] + MX[X3(k + 1, i - 1, j)] + MX[c] + MX[X3(k, i - 1, j)])
                             + J23(k, i, j, I_XYW) * 0.25 / MAPFv(i, j, 1, I_XY)
                                 * (MY[X3(k + 1, i, j)] + MY[X3(k + 1, i, j - 1)] + MY[c] + MY[X3(k, i, j - 1)])
                             + GS(k, i, j, I_XYW) / (MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY)) * NDp(V_DENS, DZIR)[c];
            W.mZ[c] = v;
            if (!in) put_flux(a, N3, 0, c, v, false);
        }
        if (lane == 0) {
            W.mZ[X3(KS - 1, i, j)] = 0.0;
            W.mZ[X3(KE, i, j)] = 0.0;
            if (!in) {
                put_flux(a, N3, 0, X3(KS - 1, i, j), 0.0, false);
                put_flux(a, N3, 0, X3(KE, i, j), 0.0, false);
            }
        }
    });
    // ---- hevi_mflx_x :399-421, hevi_mflx_y :423-438 ----
    gcols(IS - 1, IEH, JS, JE, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double v = GS(k, i, j, I_UYZ) / MAPFv(i, j, 2, I_UY) * (MX[c] + NDp(V_DENS, DXIR)[c]);
            W.mX[c] = v;
            put_flux(a, N3, 1, c, v, i >= IS);
        }
    });
    gcols(IS, IE, JS - 1, JEH, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double v = GS(k, i, j, I_XVZ) / MAPFv(i, j, 1, I_XV) * (MY[c] + NDp(V_DENS, DYIR)[c]);
            W.mY[c] = v;
            put_flux(a, N3, 2, c, v, j >= JS);
        }
    });
    // ---- hevi_sr :443-479 ----
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double advcv = -(W.mZ[c] - W.mZ[c - 1]) * ld(g.RCDZ + k - 1);
            const double advch = -((W.mX[c] - W.mX[c - sI]) * ld(g.RCDX + i - 1) + (W.mY[c] - W.mY[c - sJ]) * ld(g.RCDY + j - 1));
            W.Sr[c] = (advcv + advch) * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY) / GS(k, i, j, I_XYZ) + a.DENS_t[c];
        }
    });
    // ---- momentum (z) fluxes :485-525 ----
    // fluxZ_XYW (ud3.F90:358-452): flux(k-1) for k = KS+1..KE-1
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XYZ), *nd = NDp(V_MOMZ, DZIR), *col = MZ + X3(1, i, j);
        for (int k = KS + 1 + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MZ[c - 1] + MZ[c])) / DN[c];
            W.qZ[c - 1] = J33G * vel * zface<S>(vel, k - 1, KS, KE, [&](int l) { return col[l - 1]; }) + Gs[c] * nd[c];
        }
        if (lane == 0) {
            W.qZ[X3(KS - 1, i, j)] = 0.0;
            W.qZ[X3(KE - 1, i, j)] = 0.0;
            W.qZ[X3(KE, i, j)] = 0.0;
        }
    });
    // fluxJ13_XYW (ud3.F90:457-523) and fluxJ23_XYW (:527-593)
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        constexpr bool wide = wide_scheme(S);
        const int kend = wide ? KE - 2 : KE - 1;
        const double *J1 = J13s(I_XYZ), *J2 = J23s(I_XYZ);
        const double m2 = MAPFv(i, j, 2, I_XY), m1 = MAPFv(i, j, 1, I_XY);
        auto V = [&](int k) { return MZ[X3(k, i, j)]; };
        auto face = [&](double vel, int k) {
            if constexpr (wide) return ip6<S>(vel, V(k - 3), V(k - 2), V(k - 1), V(k), V(k + 1), V(k + 2));
            else return ip4<S>(vel, V(k - 2), V(k - 1), V(k), V(k + 1));
        };
        for (int k = KS + 2 + lane; k <= kend; k += 32) {
            const size_t c = X3(k, i, j);
            double vel = (0.5 * (MX[c] + MX[c - sI])) / DN[c];
            vel = vel * J1[c];
            W.qJ13[c - 1] = vel / m2 * face(vel, k);
            double vel2 = (0.5 * (MY[c] + MY[c - sJ])) / DN[c];
            vel2 = vel2 * J2[c];
            W.qJ23[c - 1] = vel2 / m1 * face(vel2, k);
        }
        if (lane == 0) {
            W.qJ13[X3(KS - 1, i, j)] = 0.0;
            W.qJ23[X3(KS - 1, i, j)] = 0.0;
            const size_t c0 = X3(KS, i, j), c1 = X3(KS + 1, i, j);
            double vel = ((0.5 * (MX[c1] + MX[c1 - sI])) / DN[c1] + (0.5 * (MX[c0] + MX[c0 - sI])) / DN[c0]) * 0.5;
            vel = vel * J1[c1];
            W.qJ13[c0] = vel / m2 * ipL<S>(vel, V(KS), V(KS + 1), V(KS + 2));
            double vel2 = ((0.5 * (MY[c1] + MY[c1 - sJ])) / DN[c1] + (0.5 * (MY[c0] + MY[c0 - sJ])) / DN[c0]) * 0.5;
            vel2 = vel2 * J2[c1];
            W.qJ23[c0] = vel2 / m1 * ipL<S>(vel2, V(KS), V(KS + 1), V(KS + 2));
            if constexpr (wide) {
                const size_t ce = X3(KE - 1, i, j);
                double ve = (0.5 * (MX[ce] + MX[ce - sI])) / DN[ce];
                ve = ve * J1[ce];
                W.qJ13[X3(KE - 2, i, j)] = ve / m2 * ipH<S>(ve, V(KE - 1), V(KE - 2), V(KE - 3));
                double ve2 = (0.5 * (MY[ce] + MY[ce - sJ])) / DN[ce];
                ve2 = ve2 * J2[ce];
                W.qJ23[X3(KE - 2, i, j)] = ve2 / m1 * ipH<S>(ve2, V(KE - 1), V(KE - 2), V(KE - 3));
            }
            W.qJ13[X3(KE - 1, i, j)] = 0.0;
            W.qJ23[X3(KE - 1, i, j)] = 0.0;
        }
    });
    // fluxX_XYW (ud3.F90:598-671)
    gcols(IS - 1, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_UYW), *nd = NDp(V_MOMZ, DXIR);
        const double mp = MAPFv(i, j, 2, I_UY);
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (F2Hg(Gs, k, 1) * MX[c + 1] + F2Hg(Gs, k, 2) * MX[c])
                               / (F2Hg(Gs, k, 1) * 0.5 * (DN[c + 1] + DN[c + 1 + sI]) + F2Hg(Gs, k, 2) * 0.5 * (DN[c] + DN[c + sI]));
            W.qX[c] = Gs[c] / mp * vel * hface<S>(vel, MZ + c, sI) + Gs[c] * nd[c];
        }
        if (lane == 0) W.qX[X3(KE, i, j)] = 0.0;
    });
    // fluxY_XYW (ud3.F90:675-748)
    gcols(IS, IE, JS - 1, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XVW), *nd = NDp(V_MOMZ, DYIR);
        const double mp = MAPFv(i, j, 1, I_XV);
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (F2Hg(Gs, k, 1) * MY[c + 1] + F2Hg(Gs, k, 2) * MY[c])
                               / (F2Hg(Gs, k, 1) * 0.5 * (DN[c + 1] + DN[c + 1 + sJ]) + F2Hg(Gs, k, 2) * 0.5 * (DN[c] + DN[c + sJ]));
            W.qY[c] = Gs[c] / mp * vel * hface<S>(vel, MZ + c, sJ) + Gs[c] * nd[c];
        }
        if (lane == 0) W.qY[X3(KE, i, j)] = 0.0;
    });
    // ---- hevi_sw :528-578 ----
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double advcv = -(W.qZ[c] - W.qZ[c - 1] + W.qJ13[c] - W.qJ13[c - 1] + W.qJ23[c] - W.qJ23[c - 1]) * ld(g.RFDZ + k - 1);
            const double advch = -((W.qX[c] - W.qX[c - sI]) * ld(g.RCDX + i - 1) + (W.qY[c] - W.qY[c - sJ]) * ld(g.RCDY + j - 1))
                                 * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY);
            const double wdmp = -ld(a.wdamp + g.z0 + k - 1) * a.MOMZ0[c];
            const double div = use_div ? a.divdmp_coef / dt * (a.DDIV[c + 1] - a.DDIV[c]) * ld(g.FDZ + k - 1) : 0.0;
            W.Sw[c] = (advcv + advch) / GS(k, i, j, I_XYW) + wdmp + div + a.MOMZ_t[c];
        }
    });
    // ---- POTT :586-598, over the halo too ----
    gcols(IS - g.IHALO, IE + g.IHALO, JS - g.JHALO, JE + g.JHALO, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            W.POTT[c] = a.RHOT[c] / DN[c];
        }
    });
    // ---- theta fluxes :603-622: fluxZ_XYZ (ud3.F90:157-247) ----
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XYW), *nd = NDp(V_RHOT, DZIR), *col = W.POTT + X3(1, i, j);
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = W.mZ[c];
            W.tZ[c] = vel * zface<S>(vel, k, KS, KE, [&](int l) { return col[l - 1]; }) + Gs[c] * nd[c];
        }
        if (lane == 0) {
            W.tZ[X3(KS - 1, i, j)] = 0.0;
            W.tZ[X3(KE, i, j)] = 0.0;
        }
    });
    // fluxX_XYZ (:251-300), fluxY_XYZ (:304-353)
    gcols(IS - 1, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_UYZ), *nd = NDp(V_RHOT, DXIR);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = W.mX[c];
            const double v = vel * hface<S>(vel, W.POTT + c, sI) + Gs[c] * nd[c];
            W.tX[c] = v;
            put_flux(a, N3, 4, c, v, i >= IS);
        }
    });
    gcols(IS, IE, JS - 1, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XVZ), *nd = NDp(V_RHOT, DYIR);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = W.mY[c];
            const double v = vel * hface<S>(vel, W.POTT + c, sJ) + Gs[c] * nd[c];
            W.tY[c] = v;
            put_flux(a, N3, 5, c, v, j >= JS);
        }
    });
    // ---- hevi_st :625-661 ----
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double advcv = -(W.tZ[c] - W.tZ[c - 1]) * ld(g.RCDZ + k - 1);
            const double advch = -((W.tX[c] - W.tX[c - sI]) * ld(g.RCDX + i - 1) + (W.tY[c] - W.tY[c - sJ]) * ld(g.RCDY + j - 1));
            W.St[c] = (advcv + advch) * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY) / GS(k, i, j, I_XYZ) + a.RHOT_t[c];
        }
    });
    // ---- hevi_solver :665-809: the coefficients and right-hand side of each
    // column (one warp per column, lanes along k), the solve, the back-update ----
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *GW = GSs(I_XYW), *GZ = GSs(I_XYZ);
        const double *col_mz = MZ + X3(1, i, j), *col_pt = W.POTT + X3(1, i, j);
        const size_t c1 = X3(1, i, j);
        double *A = W.A + c1 - 1, *PT = W.PT + c1 - 1, *F1 = W.F1 + c1 - 1, *F2 = W.F2 + c1 - 1, *F3 = W.F3 + c1 - 1;
        double *C = W.C + c1 - 1; // 1-based level index
        for (int k = KS + lane; k <= KE; k += 32) {
            if (k <= KE - 1) PT[k] = zface<S>(col_mz[k - 1], k, KS, KE, [&](int l) { return col_pt[l - 1]; }); // valueW_Z
            A[k] = dt * dt * J33G * ld(g.RCDZ + k - 1) * a.RT2P[c1 + k - 1] * J33G / GZ[c1 + k - 1];
        }
        __syncwarp();
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const double B = GRAV * (dt * dt) * J33G / (CDZv(k + 1) + CDZv(k));
            const double rfdz = ld(g.RFDZ + k - 1), gw = GW[c1 + k - 1];
            if (k <= KE - 2) F1[k] = -(PT[k + 1] * rfdz * A[k + 1] + B) / gw;
            F2[k] = 1.0 + (PT[k] * rfdz * (A[k + 1] + A[k])) / gw;
            if (k >= KS + 1) F3[k] = -(PT[k - 1] * rfdz * A[k] - B) / gw;
            const size_t c = c1 + k - 1;
            const double pg = -(W.DPRES[c + 1] + a.RT2P[c + 1] * dt * W.St[c + 1] - W.DPRES[c] - a.RT2P[c] * dt * W.St[c])
                                  * rfdz * J33G / gw
                              - GRAV * (F2Hg(GZ, k, 1) * (DN[c + 1] - a.REF_dens[c + 1] + W.Sr[c + 1] * dt)
                                        + F2Hg(GZ, k, 2) * (DN[c] - a.REF_dens[c] + W.Sr[c] * dt));
            C[k] = MZ[c] + dt * (pg + W.Sw[c]);
        }
    });
    // solve_direct (:1092-1127), one warp per column with the column in shared memory
    terrain_solve(g, W, st);
    // back-update of the column (:728-790)
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *GZ = GSs(I_XYZ);
        const size_t c1 = X3(1, i, j);
        const double *PT = W.PT + c1 - 1, *C = W.C + c1 - 1;
        const double mm = MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = c1 + k - 1;
            const double rcdz = ld(g.RCDZ + k - 1), gz = GZ[c];
            double adr, adt;
            if (k == KS) {
                adr = -C[KS] * J33G * rcdz / gz;
                adt = -C[KS] * PT[KS] * J33G * rcdz / gz;
            } else if (k == KE) {
                adr = C[KE - 1] * J33G * rcdz / gz;
                adt = C[KE - 1] * PT[KE - 1] * J33G * rcdz / gz;
            } else {
                adr = -(C[k] - C[k - 1]) * J33G * rcdz / gz;
                adt = -(C[k] * PT[k] - C[k - 1] * PT[k - 1]) * J33G * rcdz / gz;
            }
            put_state(a, N3, 0, a.DENS_RK, a.DENS0, c, a.DENS0[c] + dt * (adr + W.Sr[c]), true);
            put_state(a, N3, 4, a.RHOT_RK, a.RHOT0, c, a.RHOT0[c] + dt * (adt + W.St[c]), true);
            if (k <= KE - 1) {
                put_flux(a, N3, 0, c, W.mZ[c] + J33G * C[k] / mm, true);
                put_flux(a, N3, 3, c, W.tZ[c] + J33G * C[k] * PT[k] / mm, true);
                put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, a.MOMZ0[c] + (C[k] - MZ[c]), true);
            } else {
                put_flux(a, N3, 0, c, 0.0, true);
                put_flux(a, N3, 3, c, 0.0, true);
                put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, 0.0, false);
            }
        }
        if (lane == 0) {
            put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c1 + KS - 2, 0.0, false);
            put_flux(a, N3, 0, c1 + KS - 2, 0.0, false);
            put_flux(a, N3, 3, c1 + KS - 2, 0.0, false);
        }
    });

    // ---- hevi_momx :814-928 ----
#define DEN_UYZ(Gs, k) (F2Hg(Gs, k, 1) * 0.5 * (DN[X3((k) + 1, i, j)] + DN[X3((k) + 1, i + 1, j)]) \
                        + F2Hg(Gs, k, 2) * 0.5 * (DN[X3(k, i, j)] + DN[X3(k, i + 1, j)]))
#define DEN_XVZ(Gs, k) (F2Hg(Gs, k, 1) * 0.5 * (DN[X3((k) + 1, i, j)] + DN[X3((k) + 1, i, j + 1)]) \
                        + F2Hg(Gs, k, 2) * 0.5 * (DN[X3(k, i, j)] + DN[X3(k, i, j + 1)]))
#define AVG4_UV(m, k) (0.25 * ((m)[X3(k, i, j)] + (m)[X3(k, i + 1, j)] + (m)[X3(k, i, j - 1)] + (m)[X3(k, i + 1, j - 1)]))
#define AVG4_XV(m, k) (0.25 * ((m)[X3(k, i, j)] + (m)[X3(k, i - 1, j)] + (m)[X3(k, i, j + 1)] + (m)[X3(k, i - 1, j + 1)]))
    // fluxZ_UYZ (ud3.F90:753-859), fluxJ13_UYZ (:863-954), fluxJ23_UYZ (:958-1049)
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gw = GSs(I_UYW), *Gz = GSs(I_UYZ), *J1 = J13s(I_UYW), *J2 = J23s(I_UYW), *nd = NDp(V_MOMX, DZIR);
        const double *col = MX + X3(1, i, j);
        auto V = [&](int l) { return col[l - 1]; };
        const double m2 = MAPFv(i, j, 2, I_UY), m1 = MAPFv(i, j, 1, I_UY);
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MZ[c] + MZ[c + sI])) / DEN_UYZ(Gw, k);
            W.qZ[c] = J33G * vel * zface<S>(vel, k, KS, KE, V) + Gw[c] * nd[c];
            double v1 = (F2Hg(Gz, k, 1) * MX[c + 1] + F2Hg(Gz, k, 2) * MX[c]) / DEN_UYZ(Gz, k);
            v1 = v1 * J1[c];
            W.qJ13[c] = v1 / m2 * zface<S>(v1, k, KS, KE, V);
            double v2 = (F2Hg(Gz, k, 1) * AVG4_UV(MY, k + 1) + F2Hg(Gz, k, 2) * AVG4_UV(MY, k)) / DEN_UYZ(Gz, k);
            v2 = v2 * J2[c];
            W.qJ23[c] = v2 / m1 * zface<S>(v2, k, KS, KE, V);
        }
        if (lane == 0) {
            W.qZ[X3(KS - 1, i, j)] = 0.0; W.qZ[X3(KE, i, j)] = 0.0;
            W.qJ13[X3(KS - 1, i, j)] = 0.0; W.qJ13[X3(KE, i, j)] = 0.0;
            W.qJ23[X3(KS - 1, i, j)] = 0.0; W.qJ23[X3(KE, i, j)] = 0.0;
        }
    });
    // fluxX_UYZ (ud3.F90:1053-1109): flux(k,i-1) for i = IS..IE+1
    gcols(IS, IE + 1, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XYZ), *nd = NDp(V_MOMX, DXIR);
        const double mp = MAPFv(i, j, 2, I_XY);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MX[c] + MX[c - sI])) / (DN[c]);
            W.qX[c - sI] = Gs[c] / mp * vel * hface<S>(vel, MX + c - sI, sI) + Gs[c] * nd[c];
        }
    });
    // fluxY_UYZ (:1113-1167)
    gcols(IS, IE, JS - 1, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_UVZ), *nd = NDp(V_MOMX, DYIR);
        const double mp = MAPFv(i, j, 1, I_UV);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MY[c] + MY[c + sI])) / (0.25 * (DN[c] + DN[c + sI] + DN[c + sJ] + DN[c + sI + sJ]));
            W.qY[c] = Gs[c] / mp * vel * hface<S>(vel, MX + c, sJ) + Gs[c] * nd[c];
        }
    });
    gcols(IS, IEH, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *GZ = GSs(I_XYZ), *GUZ = GSs(I_UYZ);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double *DP = W.DPRES;
            const double advcv = -(W.qZ[c] - W.qZ[c - 1] + W.qJ13[c] - W.qJ13[c - 1] + W.qJ23[c] - W.qJ23[c - 1]) * ld(g.RCDZ + k - 1);
            const double advch = -((W.qX[c] - W.qX[c - sI]) * ld(g.RFDX + i - 1) + (W.qY[c] - W.qY[c - sJ]) * ld(g.RCDY + j - 1))
                                 * MAPFv(i, j, 1, I_UY) * MAPFv(i, j, 2, I_UY);
            const double *Gu = GUZ;
            const double pg = ((GZ[c + sI] * DP[c + sI] - GZ[c] * DP[c]) * ld(g.RFDX + i - 1)
                               + (J13(k, i, j, I_UYW)
                                      * 0.5 * (F2Hg(Gu, k, 1) * (DP[c + 1 + sI] + DP[c + 1]) + F2Hg(Gu, k, 2) * (DP[c + sI] + DP[c]))
                                  - J13(k - 1, i, j, I_UYW)
                                      * 0.5 * (F2Hg(Gu, k, 1) * (DP[c + sI] + DP[c]) + F2Hg(Gu, k, 2) * (DP[c - 1 + sI] + DP[c - 1])))
                                     * ld(g.RCDZ + k - 1))
                              * MAPFv(i, j, 1, I_UY);
            const double sumy = MY[c] + MY[c - sJ] + MY[c + sI] + MY[c + sI - sJ];
            const double cf = 0.125 * (a.CORIOLI[g.c2 + (size_t)i + (size_t)g.IA * (j - 1)] + a.CORIOLI[g.c2 + (size_t)(i - 1) + (size_t)g.IA * (j - 1)])
                                  * (MY[c + sI] + MY[c] + MY[c + sI - sJ] + MY[c - sJ])
                              + 0.25 * MAPFv(i, j, 1, I_UY) * MAPFv(i, j, 2, I_UY) * sumy
                                  * (sumy * 0.25 * (1.0 / MAPFv(i + 1, j, 2, I_XY) - 1.0 / MAPFv(i, j, 2, I_XY)) * ld(g.RFDX + i - 1)
                                     - MX[c] * (1.0 / MAPFv(i, j, 1, I_UV) - 1.0 / MAPFv(i, j - 1, 1, I_UV)) * ld(g.RCDY + j - 1))
                                  * 2.0 / (DN[c + sI] + DN[c]);
            const double div = use_div ? a.divdmp_coef / dt * (a.DDIV[c + sI] / MAPFv(i + 1, j, 2, I_XY) - a.DDIV[c] / MAPFv(i, j, 1, I_XY))
                                             * MAPFv(i, j, 1, I_UY) * MAPFv(i, j, 2, I_UY) * ld(g.FDX + i - 1)
                                       : 0.0;
            put_state(a, N3, 2, a.MOMX_RK, a.MOMX0, c,
                      a.MOMX0[c] + dt * ((advcv + advch - pg) / GUZ[c] + cf + div + a.MOMX_t[c]), true);
        }
    });

    // ---- hevi_momy :934-1048 ----
    // fluxZ_XVZ (ud3.F90:1173-1279), fluxJ13_XVZ (:1283-1374), fluxJ23_XVZ (:1378-1469)
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gw = GSs(I_XVW), *Gz = GSs(I_XVZ), *J1 = J13s(I_XVW), *J2 = J23s(I_XVW), *nd = NDp(V_MOMY, DZIR);
        const double *col = MY + X3(1, i, j);
        auto V = [&](int l) { return col[l - 1]; };
        const double m2 = MAPFv(i, j, 2, I_XV), m1 = MAPFv(i, j, 1, I_XV);
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MZ[c] + MZ[c + sJ])) / DEN_XVZ(Gw, k);
            W.qZ[c] = J33G * vel * zface<S>(vel, k, KS, KE, V) + Gw[c] * nd[c];
            double v1 = (F2Hg(Gz, k, 1) * AVG4_XV(MX, k + 1) + F2Hg(Gz, k, 2) * AVG4_XV(MX, k)) / DEN_XVZ(Gz, k);
            v1 = v1 * J1[c];
            W.qJ13[c] = v1 / m2 * zface<S>(v1, k, KS, KE, V);
            double v2 = (F2Hg(Gz, k, 1) * MY[c + 1] + F2Hg(Gz, k, 2) * MY[c]) / DEN_XVZ(Gz, k);
            v2 = v2 * J2[c];
            W.qJ23[c] = v2 / m1 * zface<S>(v2, k, KS, KE, V);
        }
        if (lane == 0) {
            W.qZ[X3(KS - 1, i, j)] = 0.0; W.qZ[X3(KE, i, j)] = 0.0;
            W.qJ13[X3(KS - 1, i, j)] = 0.0; W.qJ13[X3(KE, i, j)] = 0.0;
            W.qJ23[X3(KS - 1, i, j)] = 0.0; W.qJ23[X3(KE, i, j)] = 0.0;
        }
    });
    // fluxX_XVZ (:1473-1527)
    gcols(IS - 1, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_UVZ), *nd = NDp(V_MOMY, DXIR);
        const double mp = MAPFv(i, j, 2, I_UV);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MX[c] + MX[c + sJ])) / (0.25 * (DN[c] + DN[c + sI] + DN[c + sJ] + DN[c + sI + sJ]));
            W.qX[c] = Gs[c] / mp * vel * hface<S>(vel, MY + c, sI) + Gs[c] * nd[c];
        }
    });
    // fluxY_XVZ (:1531-1587): flux(k,i,j-1) for j = JS..JE+1
    gcols(IS, IE, JS, JE + 1, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XYZ), *nd = NDp(V_MOMY, DYIR);
        const double mp = MAPFv(i, j, 1, I_XY);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MY[c] + MY[c - sJ])) / (DN[c]);
            W.qY[c - sJ] = Gs[c] / mp * vel * hface<S>(vel, MY + c - sJ, sJ) + Gs[c] * nd[c];
        }
    });
    gcols(IS, IE, JS, JEH, st, [=] __device__(int i, int j, int lane) {
        const double *GZ = GSs(I_XYZ), *GVZ = GSs(I_XVZ);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double *DP = W.DPRES;
            const double advcv = -(W.qZ[c] - W.qZ[c - 1] + W.qJ13[c] - W.qJ13[c - 1] + W.qJ23[c] - W.qJ23[c - 1]) * ld(g.RCDZ + k - 1);
            const double advch = -((W.qX[c] - W.qX[c - sI]) * ld(g.RCDX + i - 1) + (W.qY[c] - W.qY[c - sJ]) * ld(g.RFDY + j - 1))
                                 * MAPFv(i, j, 1, I_XV) * MAPFv(i, j, 2, I_XV);
            const double *Gv = GVZ;
            const double pg = ((GZ[c + sJ] * DP[c + sJ] - GZ[c] * DP[c]) * ld(g.RFDY + j - 1)
                               + (J23(k, i, j, I_XVW)
                                      * 0.5 * (F2Hg(Gv, k, 1) * (DP[c + 1 + sJ] + DP[c + 1]) + F2Hg(Gv, k, 2) * (DP[c + sJ] + DP[c]))
                                  - J23(k - 1, i, j, I_XVW)
                                      * 0.5 * (F2Hg(Gv, k - 1, 1) * (DP[c + sJ] + DP[c]) + F2Hg(Gv, k - 1, 2) * (DP[c - 1 + sJ] + DP[c - 1])))
                                     * ld(g.RCDZ + k - 1))
                              * MAPFv(i, j, 2, I_XV);
            const double sumx = MX[c] + MX[c - sI] + MX[c + sJ] + MX[c - sI + sJ];
            const double cf = -0.125 * (a.CORIOLI[g.c2 + (size_t)(i - 1) + (size_t)g.IA * j] + a.CORIOLI[g.c2 + (size_t)(i - 1) + (size_t)g.IA * (j - 1)])
                                  * (MX[c + sJ] + MX[c] + MX[c - sI + sJ] + MX[c - sI])
                              - 0.25 * MAPFv(i, j, 1, I_XV) * MAPFv(i, j, 2, I_XV) * sumx
                                  * (MY[c] * (1.0 / MAPFv(i, j, 2, I_UV) - 1.0 / MAPFv(i - 1, j, 2, I_UV)) * ld(g.RCDX + i - 1)
                                     - 0.25 * (MX[c] + MX[c - sI] + MX[c + sJ] + MX[c - sI + sJ])
                                           * (1.0 / MAPFv(i, j + 1, 1, I_XY) - 1.0 / MAPFv(i, j, 1, I_XY)) * ld(g.RFDY + j - 1))
                                  * 2.0 / (DN[c + sJ] + DN[c]);
            const double div = use_div ? a.divdmp_coef / dt * (a.DDIV[c + sJ] / MAPFv(i, j + 1, 1, I_XY) - a.DDIV[c] / MAPFv(i, j, 1, I_XY))
                                             * MAPFv(i, j, 1, I_XV) * MAPFv(i, j, 2, I_XV) * ld(g.FDY + j - 1)
                                       : 0.0;
            put_state(a, N3, 3, a.MOMY_RK, a.MOMY0, c,
                      a.MOMY0[c] + dt * ((advcv + advch - pg) / GVZ[c] + cf + div + a.MOMY_t[c]), true);
        }
    });
#undef X3
#undef GSs
#undef J13s
#undef J23s
#undef GS
#undef J13
#undef J23
#undef MAPFv
#undef NDp
#undef CDZv
#undef F2Hg
#undef DEN_UYZ
#undef DEN_XVZ
#undef AVG4_UV
#undef AVG4_XV
}

// The HEVE stage with terrain-following metrics (ATMOS_DYN_Tstep_short_fvm_heve,
// scale_atmos_dyn_tstep_short_fvm_heve.F90:109-1518 without the momentum/theta
// FCT branches), in the same form as terrain_stage: one launch per loop nest,
// the flux routines with their metric arguments, outputs through put_state/put_flux.
template <int S>
static void terrain_heve_stage(const Grid &g, const StageArgsT<double> &a, const Metrics &M, const TerrainWork &W,
                               cudaStream_t st)
{
    const int KS = g.KS, KE = g.KE, IS = g.IS, IE = g.IE, JS = g.JS, JE = g.JE;
    const int IEH = g.IEH < IE ? g.IEH : IE, JEH = g.JEH < JE ? g.JEH : JE;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const double dt = a.dtrk, J33G = a.J33G;
    const bool use_div = a.divdmp_coef != 0.0;
#define X3(k, i, j) idx3(g, k, i, j)
#define GSs(idx) (M.GSQRT + (size_t)((idx) - 1) * N3)
#define J13s(idx) (M.J13G + (size_t)((idx) - 1) * N3)
#define J23s(idx) (M.J23G + (size_t)((idx) - 1) * N3)
#define GS(k, i, j, idx) ld(GSs(idx) + X3(k, i, j))
#define J13(k, i, j, idx) ld(J13s(idx) + X3(k, i, j))
#define J23(k, i, j, idx) ld(J23s(idx) + X3(k, i, j))
#define MAPFv(i, j, aa, bb) \
    ld(M.MAPF + ((size_t)((i) - 1) + (size_t)g.IA * ((size_t)((j) - 1) + (size_t)g.JA * ((size_t)((aa) - 1) + 2 * (size_t)((bb) - 1)))))
#define NDp(v, dir) (a.num_diff + N3 * (size_t)(((v) - 1) + 5 * ((dir) - 1)))
#define CDZv(k) ld(g.CDZ + (k) - 1)
#define F2Hg(Gs, k, p) (CDZv((k) + (p) - 1) * ld((Gs) + X3((k) + (p) - 1, i, j)) \
                        / (CDZv(k) * ld((Gs) + X3(k, i, j)) + CDZv((k) + 1) * ld((Gs) + X3((k) + 1, i, j))))
#define DEN_UYZ(Gs, k) (F2Hg(Gs, k, 1) * 0.5 * (DN[X3((k) + 1, i, j)] + DN[X3((k) + 1, i + 1, j)]) \
                        + F2Hg(Gs, k, 2) * 0.5 * (DN[X3(k, i, j)] + DN[X3(k, i + 1, j)]))
#define DEN_XVZ(Gs, k) (F2Hg(Gs, k, 1) * 0.5 * (DN[X3((k) + 1, i, j)] + DN[X3((k) + 1, i, j + 1)]) \
                        + F2Hg(Gs, k, 2) * 0.5 * (DN[X3(k, i, j)] + DN[X3(k, i, j + 1)]))
#define AVG4_UV(m, k) (0.25 * ((m)[X3(k, i, j)] + (m)[X3(k, i + 1, j)] + (m)[X3(k, i, j - 1)] + (m)[X3(k, i + 1, j - 1)]))
#define AVG4_XV(m, k) (0.25 * ((m)[X3(k, i, j)] + (m)[X3(k, i - 1, j)] + (m)[X3(k, i, j + 1)] + (m)[X3(k, i - 1, j + 1)]))
    const RoField DN{a.DENS}, MZ{a.MOMZ}, MX{a.MOMX}, MY{a.MOMY}; // the stage input, read-only here

    // ---- pressure :360-373, potential temperature :375-382 ----
    gcols(IS - 2, IE + 2, JS - 2, JE + 2, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            W.DPRES[c] = a.DPRES0[c] + a.RT2P[c] * (a.RHOT[c] - a.REF_rhot[c]);
        }
        if (lane == 0) {
            W.DPRES[X3(KS - 1, i, j)] = a.DPRES0[X3(KS - 1, i, j)] - DN[X3(KS, i, j)] * (M.PHI[X3(KS - 1, i, j)] - M.PHI[X3(KS + 1, i, j)]);
            W.DPRES[X3(KE + 1, i, j)] = a.DPRES0[X3(KE + 1, i, j)] - DN[X3(KE, i, j)] * (M.PHI[X3(KE + 1, i, j)] - M.PHI[X3(KE - 1, i, j)]);
        }
    });
    gcols(IS - g.IHALO, IE + g.IHALO, JS - g.JHALO, JE + g.JHALO, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            W.POTT[c] = a.RHOT[c] / DN[c];
        }
    });
    // ---- mass fluxes :460-510 ----
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double m1 = MAPFv(i, j, 1, I_XY), m2 = MAPFv(i, j, 2, I_XY);
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double v = J33G * MZ[c] / (m1 * m2)
                             + J13(k, i, j, I_XYW) * 0.25 * (MX[c + 1] + MX[c + 1 - sI] + MX[c] + MX[c - sI]) / m2
                             + J23(k, i, j, I_XYW) * 0.25 * (MY[c + 1] + MY[c + 1 - sJ] + MY[c] + MY[c - sJ]) / m1
                             + GS(k, i, j, I_XYW) * NDp(V_DENS, DZIR)[c] / (m1 * m2);
            W.mZ[c] = v;
            put_flux(a, N3, 0, c, v, true);
        }
        if (lane == 0) {
            W.mZ[X3(KS - 1, i, j)] = 0.0;
            W.mZ[X3(KE, i, j)] = 0.0;
            put_flux(a, N3, 0, X3(KS - 1, i, j), 0.0, false);
            put_flux(a, N3, 0, X3(KE, i, j), 0.0, true);
        }
    });
    gcols(IS - 1, IEH, JS, JE, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double v = GS(k, i, j, I_UYZ) / MAPFv(i, j, 2, I_UY) * (MX[c] + NDp(V_DENS, DXIR)[c]);
            W.mX[c] = v;
            put_flux(a, N3, 1, c, v, i >= IS);
        }
    });
    gcols(IS, IE, JS - 1, JEH, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double v = GS(k, i, j, I_XVZ) / MAPFv(i, j, 1, I_XV) * (MY[c] + NDp(V_DENS, DYIR)[c]);
            W.mY[c] = v;
            put_flux(a, N3, 2, c, v, j >= JS);
        }
    });
    // ---- density :512-532 ----
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double advcv = -(W.mZ[c] - W.mZ[c - 1]) * ld(g.RCDZ + k - 1);
            const double advch = -(W.mX[c] - W.mX[c - sI]) * ld(g.RCDX + i - 1) - (W.mY[c] - W.mY[c - sJ]) * ld(g.RCDY + j - 1);
            put_state(a, N3, 0, a.DENS_RK, a.DENS0, c,
                      a.DENS0[c] + dt * ((advcv + advch) * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY) / GS(k, i, j, I_XYZ) + a.DENS_t[c]),
                      true);
        }
    });
    // ---- momentum (z): fluxes :586-620 (the HEVI routines) ----
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XYZ), *nd = NDp(V_MOMZ, DZIR), *col = MZ + X3(1, i, j);
        for (int k = KS + 1 + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MZ[c - 1] + MZ[c])) / DN[c];
            W.qZ[c - 1] = J33G * vel * zface<S>(vel, k - 1, KS, KE, [&](int l) { return col[l - 1]; }) + Gs[c] * nd[c];
        }
        if (lane == 0) {
            W.qZ[X3(KS - 1, i, j)] = 0.0;
            W.qZ[X3(KE - 1, i, j)] = 0.0;
            W.qZ[X3(KE, i, j)] = 0.0;
        }
    });
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        constexpr bool wide = wide_scheme(S);
        const int kend = wide ? KE - 2 : KE - 1;
        const double *J1 = J13s(I_XYZ), *J2 = J23s(I_XYZ);
        const double m2 = MAPFv(i, j, 2, I_XY), m1 = MAPFv(i, j, 1, I_XY);
        auto V = [&](int k) { return MZ[X3(k, i, j)]; };
        auto face = [&](double vel, int k) {
            if constexpr (wide) return ip6<S>(vel, V(k - 3), V(k - 2), V(k - 1), V(k), V(k + 1), V(k + 2));
            else return ip4<S>(vel, V(k - 2), V(k - 1), V(k), V(k + 1));
        };
        for (int k = KS + 2 + lane; k <= kend; k += 32) {
            const size_t c = X3(k, i, j);
            double vel = (0.5 * (MX[c] + MX[c - sI])) / DN[c];
            vel = vel * J1[c];
            W.qJ13[c - 1] = vel / m2 * face(vel, k);
            double vel2 = (0.5 * (MY[c] + MY[c - sJ])) / DN[c];
            vel2 = vel2 * J2[c];
            W.qJ23[c - 1] = vel2 / m1 * face(vel2, k);
        }
        if (lane == 0) {
            W.qJ13[X3(KS - 1, i, j)] = 0.0;
            W.qJ23[X3(KS - 1, i, j)] = 0.0;
            const size_t c0 = X3(KS, i, j), c1 = X3(KS + 1, i, j);
            double vel = ((0.5 * (MX[c1] + MX[c1 - sI])) / DN[c1] + (0.5 * (MX[c0] + MX[c0 - sI])) / DN[c0]) * 0.5;
            vel = vel * J1[c1];
            W.qJ13[c0] = vel / m2 * ipL<S>(vel, V(KS), V(KS + 1), V(KS + 2));
            double vel2 = ((0.5 * (MY[c1] + MY[c1 - sJ])) / DN[c1] + (0.5 * (MY[c0] + MY[c0 - sJ])) / DN[c0]) * 0.5;
            vel2 = vel2 * J2[c1];
            W.qJ23[c0] = vel2 / m1 * ipL<S>(vel2, V(KS), V(KS + 1), V(KS + 2));
            if constexpr (wide) {
                const size_t ce = X3(KE - 1, i, j);
                double ve = (0.5 * (MX[ce] + MX[ce - sI])) / DN[ce];
                ve = ve * J1[ce];
                W.qJ13[X3(KE - 2, i, j)] = ve / m2 * ipH<S>(ve, V(KE - 1), V(KE - 2), V(KE - 3));
                double ve2 = (0.5 * (MY[ce] + MY[ce - sJ])) / DN[ce];
                ve2 = ve2 * J2[ce];
                W.qJ23[X3(KE - 2, i, j)] = ve2 / m1 * ipH<S>(ve2, V(KE - 1), V(KE - 2), V(KE - 3));
            }
            W.qJ13[X3(KE - 1, i, j)] = 0.0;
            W.qJ23[X3(KE - 1, i, j)] = 0.0;
        }
    });
    gcols(IS - 1, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_UYW), *nd = NDp(V_MOMZ, DXIR);
        const double mp = MAPFv(i, j, 2, I_UY);
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (F2Hg(Gs, k, 1) * MX[c + 1] + F2Hg(Gs, k, 2) * MX[c])
                               / (F2Hg(Gs, k, 1) * 0.5 * (DN[c + 1] + DN[c + 1 + sI]) + F2Hg(Gs, k, 2) * 0.5 * (DN[c] + DN[c + sI]));
            W.qX[c] = Gs[c] / mp * vel * hface<S>(vel, MZ + c, sI) + Gs[c] * nd[c];
        }
        if (lane == 0) W.qX[X3(KE, i, j)] = 0.0;
    });
    gcols(IS, IE, JS - 1, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XVW), *nd = NDp(V_MOMZ, DYIR);
        const double mp = MAPFv(i, j, 1, I_XV);
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (F2Hg(Gs, k, 1) * MY[c + 1] + F2Hg(Gs, k, 2) * MY[c])
                               / (F2Hg(Gs, k, 1) * 0.5 * (DN[c + 1] + DN[c + 1 + sJ]) + F2Hg(Gs, k, 2) * 0.5 * (DN[c] + DN[c + sJ]));
            W.qY[c] = Gs[c] / mp * vel * hface<S>(vel, MZ + c, sJ) + Gs[c] * nd[c];
        }
        if (lane == 0) W.qY[X3(KE, i, j)] = 0.0;
    });
    // pressure gradient :622-631, buoyancy :633-644, update :646-688
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *GZ = GSs(I_XYZ);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            if (k == KE) { put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, 0.0, false); continue; }
            const double pgf = J33G * (W.DPRES[c + 1] - W.DPRES[c]) * ld(g.RFDZ + k - 1);
            const double buoy = GRAV * GS(k, i, j, I_XYW)
                                * (F2Hg(GZ, k, 1) * (DN[c + 1] - a.REF_dens[c + 1]) + F2Hg(GZ, k, 2) * (DN[c] - a.REF_dens[c]));
            const double advcv = -(W.qZ[c] - W.qZ[c - 1] + W.qJ13[c] - W.qJ13[c - 1] + W.qJ23[c] - W.qJ23[c - 1]) * ld(g.RFDZ + k - 1);
            const double advch = -((W.qX[c] - W.qX[c - sI]) * ld(g.RCDX + i - 1) + (W.qY[c] - W.qY[c - sJ]) * ld(g.RCDY + j - 1))
                                 * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY);
            const double wdamp = -ld(a.wdamp + g.z0 + k - 1) * a.MOMZ0[c];
            const double div = use_div ? a.divdmp_coef / dt * ld(g.FDZ + k - 1) * (a.DDIV[c + 1] - a.DDIV[c]) : 0.0;
            put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c,
                      a.MOMZ0[c] + dt * ((advcv + advch - pgf - buoy) / GS(k, i, j, I_XYW) + wdamp + div + a.MOMZ_t[c]), true);
        }
        if (lane == 0) put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, X3(KS - 1, i, j), 0.0, false);
    });

    // ---- momentum (x): fluxes :829-860, pressure gradient, Coriolis, update :862-922 ----
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gw = GSs(I_UYW), *Gz = GSs(I_UYZ), *J1 = J13s(I_UYW), *J2 = J23s(I_UYW), *nd = NDp(V_MOMX, DZIR);
        const double *col = MX + X3(1, i, j);
        auto V = [&](int l) { return col[l - 1]; };
        const double m2 = MAPFv(i, j, 2, I_UY), m1 = MAPFv(i, j, 1, I_UY);
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MZ[c] + MZ[c + sI])) / DEN_UYZ(Gw, k);
            W.qZ[c] = J33G * vel * zface<S>(vel, k, KS, KE, V) + Gw[c] * nd[c];
            double v1 = (F2Hg(Gz, k, 1) * MX[c + 1] + F2Hg(Gz, k, 2) * MX[c]) / DEN_UYZ(Gz, k);
            v1 = v1 * J1[c];
            W.qJ13[c] = v1 / m2 * zface<S>(v1, k, KS, KE, V);
            double v2 = (F2Hg(Gz, k, 1) * AVG4_UV(MY, k + 1) + F2Hg(Gz, k, 2) * AVG4_UV(MY, k)) / DEN_UYZ(Gz, k);
            v2 = v2 * J2[c];
            W.qJ23[c] = v2 / m1 * zface<S>(v2, k, KS, KE, V);
        }
        if (lane == 0) {
            W.qZ[X3(KS - 1, i, j)] = 0.0; W.qZ[X3(KE, i, j)] = 0.0;
            W.qJ13[X3(KS - 1, i, j)] = 0.0; W.qJ13[X3(KE, i, j)] = 0.0;
            W.qJ23[X3(KS - 1, i, j)] = 0.0; W.qJ23[X3(KE, i, j)] = 0.0;
        }
    });
    gcols(IS, IE + 1, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XYZ), *nd = NDp(V_MOMX, DXIR);
        const double mp = MAPFv(i, j, 2, I_XY);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MX[c] + MX[c - sI])) / (DN[c]);
            W.qX[c - sI] = Gs[c] / mp * vel * hface<S>(vel, MX + c - sI, sI) + Gs[c] * nd[c];
        }
    });
    gcols(IS, IE, JS - 1, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_UVZ), *nd = NDp(V_MOMX, DYIR);
        const double mp = MAPFv(i, j, 1, I_UV);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MY[c] + MY[c + sI])) / (0.25 * (DN[c] + DN[c + sI] + DN[c + sJ] + DN[c + sI + sJ]));
            W.qY[c] = Gs[c] / mp * vel * hface<S>(vel, MX + c, sJ) + Gs[c] * nd[c];
        }
    });
    gcols(IS, IEH, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *GZ = GSs(I_XYZ), *Gu = GSs(I_UYZ);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double *DP = W.DPRES;
            const double pgf = ((GZ[c + sI] * DP[c + sI] - GZ[c] * DP[c]) * ld(g.RFDX + i - 1)
                                + (J13(k, i, j, I_UYW)
                                       * 0.5 * (F2Hg(Gu, k, 1) * (DP[c + 1 + sI] + DP[c + 1]) + F2Hg(Gu, k, 2) * (DP[c + sI] + DP[c]))
                                   - J13(k - 1, i, j, I_UYW)
                                       * 0.5 * (F2Hg(Gu, k, 1) * (DP[c + sI] + DP[c]) + F2Hg(Gu, k, 2) * (DP[c - 1 + sI] + DP[c - 1])))
                                      * ld(g.RCDZ + k - 1))
                               * MAPFv(i, j, 1, I_UY);
            const double sumy = MY[c] + MY[c - sJ] + MY[c + sI] + MY[c + sI - sJ];
            const double cor = 0.125 * (a.CORIOLI[g.c2 + (size_t)i + (size_t)g.IA * (j - 1)] + a.CORIOLI[g.c2 + (size_t)(i - 1) + (size_t)g.IA * (j - 1)])
                                   * (MY[c + sI] + MY[c] + MY[c + sI - sJ] + MY[c - sJ])
                               + 0.25 * MAPFv(i, j, 1, I_UY) * MAPFv(i, j, 2, I_UY) * sumy
                                   * (sumy * 0.25 * (1.0 / MAPFv(i + 1, j, 2, I_XY) - 1.0 / MAPFv(i, j, 2, I_XY)) * ld(g.RFDX + i - 1)
                                      - MX[c] * (1.0 / MAPFv(i, j, 1, I_UV) - 1.0 / MAPFv(i, j - 1, 1, I_UV)) * ld(g.RCDY + j - 1))
                                   * 2.0 / (DN[c + sI] + DN[c]);
            const double advcv = -(W.qZ[c] - W.qZ[c - 1] + W.qJ13[c] - W.qJ13[c - 1] + W.qJ23[c] - W.qJ23[c - 1]) * ld(g.RCDZ + k - 1);
            const double advch = -((W.qX[c] - W.qX[c - sI]) * ld(g.RFDX + i - 1) + (W.qY[c] - W.qY[c - sJ]) * ld(g.RCDY + j - 1))
                                 * MAPFv(i, j, 1, I_UY) * MAPFv(i, j, 2, I_UY);
            const double div = use_div ? a.divdmp_coef / dt * ld(g.FDX + i - 1) * (a.DDIV[c + sI] - a.DDIV[c]) : 0.0;
            put_state(a, N3, 2, a.MOMX_RK, a.MOMX0, c,
                      a.MOMX0[c] + dt * ((advcv + advch - pgf) / Gu[c] + cor + div + a.MOMX_t[c]), true);
        }
    });

    // ---- momentum (y): fluxes :1076-1107, pressure gradient, Coriolis, update :1109-1170 ----
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gw = GSs(I_XVW), *Gz = GSs(I_XVZ), *J1 = J13s(I_XVW), *J2 = J23s(I_XVW), *nd = NDp(V_MOMY, DZIR);
        const double *col = MY + X3(1, i, j);
        auto V = [&](int l) { return col[l - 1]; };
        const double m2 = MAPFv(i, j, 2, I_XV), m1 = MAPFv(i, j, 1, I_XV);
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MZ[c] + MZ[c + sJ])) / DEN_XVZ(Gw, k);
            W.qZ[c] = J33G * vel * zface<S>(vel, k, KS, KE, V) + Gw[c] * nd[c];
            double v1 = (F2Hg(Gz, k, 1) * AVG4_XV(MX, k + 1) + F2Hg(Gz, k, 2) * AVG4_XV(MX, k)) / DEN_XVZ(Gz, k);
            v1 = v1 * J1[c];
            W.qJ13[c] = v1 / m2 * zface<S>(v1, k, KS, KE, V);
            double v2 = (F2Hg(Gz, k, 1) * MY[c + 1] + F2Hg(Gz, k, 2) * MY[c]) / DEN_XVZ(Gz, k);
            v2 = v2 * J2[c];
            W.qJ23[c] = v2 / m1 * zface<S>(v2, k, KS, KE, V);
        }
        if (lane == 0) {
            W.qZ[X3(KS - 1, i, j)] = 0.0; W.qZ[X3(KE, i, j)] = 0.0;
            W.qJ13[X3(KS - 1, i, j)] = 0.0; W.qJ13[X3(KE, i, j)] = 0.0;
            W.qJ23[X3(KS - 1, i, j)] = 0.0; W.qJ23[X3(KE, i, j)] = 0.0;
        }
    });
    gcols(IS - 1, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_UVZ), *nd = NDp(V_MOMY, DXIR);
        const double mp = MAPFv(i, j, 2, I_UV);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MX[c] + MX[c + sJ])) / (0.25 * (DN[c] + DN[c + sI] + DN[c + sJ] + DN[c + sI + sJ]));
            W.qX[c] = Gs[c] / mp * vel * hface<S>(vel, MY + c, sI) + Gs[c] * nd[c];
        }
    });
    gcols(IS, IE, JS, JE + 1, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XYZ), *nd = NDp(V_MOMY, DYIR);
        const double mp = MAPFv(i, j, 1, I_XY);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = (0.5 * (MY[c] + MY[c - sJ])) / (DN[c]);
            W.qY[c - sJ] = Gs[c] / mp * vel * hface<S>(vel, MY + c - sJ, sJ) + Gs[c] * nd[c];
        }
    });
    gcols(IS, IE, JS, JEH, st, [=] __device__(int i, int j, int lane) {
        const double *GZ = GSs(I_XYZ), *Gv = GSs(I_XVZ);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double *DP = W.DPRES;
            const double pgf = ((GZ[c + sJ] * DP[c + sJ] - GZ[c] * DP[c]) * ld(g.RFDY + j - 1)
                                + (J23(k, i, j, I_XVW)
                                       * 0.5 * (F2Hg(Gv, k, 1) * (DP[c + 1 + sJ] + DP[c + 1]) + F2Hg(Gv, k, 2) * (DP[c + sJ] + DP[c]))
                                   - J23(k - 1, i, j, I_XVW)
                                       * 0.5 * (F2Hg(Gv, k - 1, 1) * (DP[c + sJ] + DP[c]) + F2Hg(Gv, k - 1, 2) * (DP[c - 1 + sJ] + DP[c - 1])))
                                      * ld(g.RCDZ + k - 1))
                               * MAPFv(i, j, 2, I_XV);
            const double sumx = MX[c] + MX[c - sI] + MX[c + sJ] + MX[c - sI + sJ];
            const double cor = -0.125 * (a.CORIOLI[g.c2 + (size_t)(i - 1) + (size_t)g.IA * j] + a.CORIOLI[g.c2 + (size_t)(i - 1) + (size_t)g.IA * (j - 1)])
                                   * (MX[c + sJ] + MX[c] + MX[c - sI + sJ] + MX[c - sI])
                               - 0.25 * MAPFv(i, j, 1, I_XV) * MAPFv(i, j, 2, I_XV) * sumx
                                   * (MY[c] * (1.0 / MAPFv(i, j, 2, I_UV) - 1.0 / MAPFv(i - 1, j, 2, I_UV)) * ld(g.RCDX + i - 1)
                                      - 0.25 * (MX[c] + MX[c - sI] + MX[c + sJ] + MX[c - sI + sJ])
                                            * (1.0 / MAPFv(i, j + 1, 1, I_XY) - 1.0 / MAPFv(i, j, 1, I_XY)) * ld(g.RFDY + j - 1))
                                   * 2.0 / (DN[c] + DN[c + sJ]);
            const double advcv = -(W.qZ[c] - W.qZ[c - 1] + W.qJ13[c] - W.qJ13[c - 1] + W.qJ23[c] - W.qJ23[c - 1]) * ld(g.RCDZ + k - 1);
            const double advch = -((W.qX[c] - W.qX[c - sI]) * ld(g.RCDX + i - 1) + (W.qY[c] - W.qY[c - sJ]) * ld(g.RFDY + j - 1))
                                 * MAPFv(i, j, 1, I_XV) * MAPFv(i, j, 2, I_XV);
            const double div = use_div ? a.divdmp_coef / dt * ld(g.FDY + j - 1) * (a.DDIV[c + sJ] - a.DDIV[c]) : 0.0;
            put_state(a, N3, 3, a.MOMY_RK, a.MOMY0, c,
                      a.MOMY0[c] + dt * ((advcv + advch - pgf) / Gv[c] + cor + div + a.MOMY_t[c]), true);
        }
    });

    // ---- rho*theta: fluxes :1328-1348 (mass fluxes as they are), update :1350-1371 ----
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XYW), *nd = NDp(V_RHOT, DZIR), *col = W.POTT + X3(1, i, j);
        for (int k = KS + lane; k <= KE - 1; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = W.mZ[c];
            const double v = vel * zface<S>(vel, k, KS, KE, [&](int l) { return col[l - 1]; }) + Gs[c] * nd[c];
            W.tZ[c] = v;
            put_flux(a, N3, 3, c, v, true);
        }
        if (lane == 0) {
            W.tZ[X3(KS - 1, i, j)] = 0.0;
            W.tZ[X3(KE, i, j)] = 0.0;
            put_flux(a, N3, 3, X3(KS - 1, i, j), 0.0, false);
            put_flux(a, N3, 3, X3(KE, i, j), 0.0, true);
        }
    });
    gcols(IS - 1, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_UYZ), *nd = NDp(V_RHOT, DXIR);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = W.mX[c];
            const double v = vel * hface<S>(vel, W.POTT + c, sI) + Gs[c] * nd[c];
            W.tX[c] = v;
            put_flux(a, N3, 4, c, v, i >= IS);
        }
    });
    gcols(IS, IE, JS - 1, JE, st, [=] __device__(int i, int j, int lane) {
        const double *Gs = GSs(I_XVZ), *nd = NDp(V_RHOT, DYIR);
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double vel = W.mY[c];
            const double v = vel * hface<S>(vel, W.POTT + c, sJ) + Gs[c] * nd[c];
            W.tY[c] = v;
            put_flux(a, N3, 5, c, v, j >= JS);
        }
    });
    gcols(IS, IE, JS, JE, st, [=] __device__(int i, int j, int lane) {
        for (int k = KS + lane; k <= KE; k += 32) {
            const size_t c = X3(k, i, j);
            const double advcv = -(W.tZ[c] - W.tZ[c - 1]) * ld(g.RCDZ + k - 1);
            const double advch = -(W.tX[c] - W.tX[c - sI]) * ld(g.RCDX + i - 1) - (W.tY[c] - W.tY[c - sJ]) * ld(g.RCDY + j - 1);
            put_state(a, N3, 4, a.RHOT_RK, a.RHOT0, c,
                      a.RHOT0[c] + dt * ((advcv + advch) * MAPFv(i, j, 1, I_XY) * MAPFv(i, j, 2, I_XY) / GS(k, i, j, I_XYZ) + a.RHOT_t[c]),
                      true);
        }
    });
#undef X3
#undef GSs
#undef J13s
#undef J23s
#undef GS
#undef J13
#undef J23
#undef MAPFv
#undef NDp
#undef CDZv
#undef F2Hg
#undef DEN_UYZ
#undef DEN_XVZ
#undef AVG4_UV
#undef AVG4_XV
}

cudaError_t launch_terrain_stage(const Grid &g, const StageArgsT<double> &a, const Metrics &M, const TerrainWork &W,
                                 int scheme, cudaStream_t st)
{
    switch (scheme) {
    case UD3: terrain_stage<UD3>(g, a, M, W, st); break;
    case CD4: terrain_stage<CD4>(g, a, M, W, st); break;
    case KOREN: terrain_stage<KOREN>(g, a, M, W, st); break;
    case CD2: terrain_stage<CD2>(g, a, M, W, st); break;
    case UD5: terrain_stage<UD5>(g, a, M, W, st); break;
    case CD6: terrain_stage<CD6>(g, a, M, W, st); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_terrain_heve_stage(const Grid &g, const StageArgsT<double> &a, const Metrics &M,
                                      const TerrainWork &W, int scheme, cudaStream_t st)
{
    switch (scheme) {
    case UD3: terrain_heve_stage<UD3>(g, a, M, W, st); break;
    case CD4: terrain_heve_stage<CD4>(g, a, M, W, st); break;
    case KOREN: terrain_heve_stage<KOREN>(g, a, M, W, st); break;
    case CD2: terrain_heve_stage<CD2>(g, a, M, W, st); break;
    case UD5: terrain_heve_stage<UD5>(g, a, M, W, st); break;
    case CD6: terrain_heve_stage<CD6>(g, a, M, W, st); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

#endif // HEVI_FLOAT_TU

}  // namespace hevi
