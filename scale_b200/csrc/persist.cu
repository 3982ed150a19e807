// One short step of every ensemble member as ONE persistent cooperative
// launch: the numerical filter (ATMOS_DYN_numfilter_coef, ND_ORDER = 1), the
// four RK4 HEVI stages (scale_atmos_dyn_tinteg_short_rk4.F90:199-666 with
// ATMOS_DYN_Tstep_short_fvm_hevi), the vertical boundary values and the halo
// fills of the large step's loop (scale_atmos_dyn_tstep_large_fvm_heve.F90:
// 847-944), on flat terrain without divergence damping.
//
// The grid is as many CTAs as the SMs hold at once (a cooperative launch
// guarantees they are all resident). Each phase is the same device body the
// separate kernels run (phi_point, numfilter_column, halo_column,
// hevi_stage_block, vbc_column), applied to the blocks of that phase's launch
// over all members, whose block maps are kernel parameters: a CTA takes the
// blocks x = blockIdx.x, blockIdx.x + gridDim.x, ... of a fill or of phi in
// sub-blocks of 4 or 8 warps, the filter's blocks four at a time and the stage
// tiles one at a time from counters (columns of different heights cost
// different times). Between phases a grid barrier: CTA
// arrivals counted on a device word with a release, polled with an acquire,
// and bounded in time; a barrier that does not complete within the wait limit
// sets ST_BARRIER_TIMEOUT in the status word and the CTA returns (so does
// every other CTA at that barrier), which the host reports as an error.
//
// This translation unit reads every field with ordinary coherent loads
// (HEVI_COHERENT_LOADS): the filter output, the RK stage buffers and their
// halos are written and read again within the launch, which the read-only
// cache path does not allow. The arithmetic is the separate kernels', so a
// member advanced here is bit-identical to the same member advanced by them.
#define HEVI_COHERENT_LOADS 1
#include "hevi_stage_body.cuh"
#include "numfilter_body.cuh"
#include "fill_body.cuh"

namespace hevi {
namespace persist {

constexpr int WARPS = HEVI_COL_TC; // warps per CTA (the stage tile's)
constexpr int NM = HEVI_MAX_MEMBERS;

template <typename R>
struct Args {
    BatchT<NM> bphi, bnd, bhalo, bstage, bvbc; // the block maps of the phases
    NdCoef ndc;
    NdArgsT<R> nd;
    StageArgsT<R> st[4];
    double *rk[3][5];  // the outputs of stages 1-3, halo-filled after each
    double *X[5];      // the state: stage 4 writes it, then its vertical and lateral halo
    unsigned *bar;     // [0] arrival counter, [1 + s] tiles taken in stage s, [5] filter blocks taken; zero at launch
    unsigned *status;
    long long wait;    // clock cycles a barrier waits at most
    unsigned extra;    // arrivals a barrier waits for beyond the grid's own (0)
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// The n-th grid barrier: every CTA's writes before it are visible to every
// CTA after it. False when it did not complete within the wait limit.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned target, unsigned *status, long long wait, int *s_ok)
{
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        const long long t0 = clock64();
        int ok = 1;
        while (ld_acquire(bar) < target) {
            if (clock64() - t0 > wait) {
                ok = 0;
                atomicOr(status, ST_BARRIER_TIMEOUT);
                break;
            }
            __nanosleep(128);
        }
        __threadfence();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// the blocks [0, nvb) of a phase whose bodies take VW warps: this CTA's share
template <int VW, class F>
__device__ __forceinline__ void for_blocks(int nvb, F f)
{
    constexpr int PER = WARPS / VW;
    static_assert(PER * VW == WARPS, "a sub-block must divide the CTA");
    const int sub = threadIdx.y / VW, wy = threadIdx.y % VW;
    for (int base = blockIdx.x * PER; base < nvb; base += gridDim.x * PER) {
        const int x = base + sub;
        if (x < nvb) f(x, wy, (int)threadIdx.x);
    }
}

// the same, taking WARPS / VW blocks at a time from the counter *next (zero at
// launch), so that blocks of different cost even out across the CTAs; s_x is
// a shared word of the CTA
template <int VW, class F>
__device__ __forceinline__ void take_blocks(unsigned *next, int nvb, int *s_x, F f)
{
    constexpr int PER = WARPS / VW;
    static_assert(PER * VW == WARPS, "a sub-block must divide the CTA");
    const int sub = threadIdx.y / VW, wy = threadIdx.y % VW;
    for (;;) {
        if (threadIdx.x == 0 && threadIdx.y == 0) *s_x = (int)atomicAdd(next, (unsigned)PER);
        __syncthreads();
        const int base = *s_x; // block-uniform
        __syncthreads();       // every thread has read it before the next take
        if (base >= nvb) break;
        const int x = base + sub;
        if (x < nvb) f(x, wy, (int)threadIdx.x);
    }
}

template <int S, typename R, int TX>
__global__ void __launch_bounds__(32 * WARPS, HEVI_COL_MINB) k_short_step(const Grid gt, const __grid_constant__ Args<R> a)
{
    __shared__ int s_ok, s_x;
    const Args<R> &P = a;
    const size_t N3 = n3(gt);
    unsigned nbar = 0;
    auto barrier = [&]() {
        ++nbar;
        return grid_barrier(a.bar, nbar * gridDim.x + a.extra, a.status, a.wait, &s_ok);
    };
    // lateral halo of nf fields of type T
    auto halo = [&](auto *const *f, int nf) {
        const int nb = P.bhalo.first[P.bhalo.n];
        for_blocks<FILL_WARPS>(nb * nf, [&](int x, int wy, int lane) {
            const int q = x / nb;
            halo_column(gt, f[q], P.bhalo, x - q * nb, wy, lane);
        });
    };

    // ---- numerical filter: the filtered quantities, then num_diff, then its halo ----
    for_blocks<PHI_THREADS / 32>(P.bphi.first[P.bphi.n],
                                 [&](int x, int wy, int lane) { phi_point(gt, a.nd, P.bphi, x, wy * 32 + lane); });
    if (!barrier()) return;
    take_blocks<ND_WARPS>(a.bar + 5, P.bnd.first[P.bnd.n], &s_x, [&](int x, int wy, int lane) {
        numfilter_column<R, NM, false>(gt, a.ndc, a.nd, P.bnd, nullptr, x, wy, lane);
    });
    if (!barrier()) return;
    {
        R *f[15];
        for (int q = 0; q < 15; ++q) f[q] = a.nd.num_diff + (size_t)q * N3;
        halo(f, 15);
    }
    if (!barrier()) return;

    // ---- the RK4 stages; the outputs of stages 1-3 get their halo ----
    // A CTA takes the next tile of the stage from a counter, so that tiles of
    // members of different heights even out across the CTAs.
    for (int s = 0; s < 4; ++s) {
        const int nst = P.bstage.first[P.bstage.n];
        for (;;) {
            if (threadIdx.x == 0 && threadIdx.y == 0) s_x = (int)atomicAdd(a.bar + 1 + s, 1u);
            __syncthreads();
            const int x = s_x; // block-uniform
            if (x >= nst) break;
            hevi_stage_block<S, R, TX, NM>(gt, a.st[s], P.bstage, x);
            __syncthreads(); // s_x and the tile's shared arrays are free for the next tile
        }
        if (!barrier()) return;
        if (s < 3) {
            halo(a.rk[s], 5);
            if (!barrier()) return;
        }
    }

    // ---- vertical boundary values, then the lateral halo of the state ----
    for_blocks<FILL_WARPS>(P.bvbc.first[P.bvbc.n], [&](int x, int wy, int lane) {
        vbc_column(gt, a.X[0], a.X[1], a.X[2], a.X[3], a.X[4], P.bvbc, x, wy, lane);
    });
    if (!barrier()) return;
    halo(a.X, 5);
}

// ---- host side ---------------------------------------------------------------
template <class NB>
static void fill_batch(BatchT<NM> &B, const Grid &g, const Members &mem, NB nblocks_of)
{
    B = BatchT<NM>{};
    B.n = mem.n > 0 ? mem.n : 1;
    long long total = 0;
    for (int q = 0; q < B.n; ++q) {
        B.first[q] = (int)total;
        if (mem.n > 0) B.m[q] = mem.m[q];
        else {
            // one domain: its own geometry at zero offsets
            MemberGeom &m = B.m[q];
            m.KMAX = g.KMAX; m.IMAX = g.IMAX; m.JMAX = g.JMAX;
            m.z0 = m.x0 = m.y0 = m.cell0 = m.c2 = 0;
        }
        total += nblocks_of(member_grid(g, B.m[q]));
    }
    for (int q = B.n; q <= NM; ++q) B.first[q] = (int)total;
}

template <int S, typename R, int TX>
static cudaError_t launch_s(const Grid &g, const Members &mem, const PersistStepT<R> &p, int maxKA, cudaStream_t st,
                            int *grid)
{
    auto kern = k_short_step<S, R, TX>;
    const size_t smem = (size_t)COL_ARRAYS * HEVI_COL_TC * col_pitch(maxKA) * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0, per = 0, khz = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 32 * WARPS, smem)) != cudaSuccess) return e;
    if (per < 1) return cudaErrorInvalidConfiguration;
    Args<R> a{}; // about 12 KB of kernel parameters
    constexpr int TY = HEVI_COL_TC / TX;
    fill_batch(a.bphi, g, mem, [](const Grid &m) { return (int)(((long)m.KA * m.IA * m.JA + PHI_THREADS - 1) / PHI_THREADS); });
    fill_batch(a.bnd, g, mem, [](const Grid &m) { return ((m.IMAX + ND_WARPS - 1) / ND_WARPS) * m.JMAX; });
    fill_batch(a.bhalo, g, mem, [](const Grid &m) { return halo_blocks(m); });
    fill_batch(a.bstage, g, mem, [](const Grid &m) { return ((m.IMAX + TX - 1) / TX) * ((m.JMAX + TY - 1) / TY); });
    fill_batch(a.bvbc, g, mem, [](const Grid &m) { return vbc_blocks(m); });
    a.ndc = p.ndc;
    a.nd = p.nd;
    for (int s = 0; s < 4; ++s) {
        a.st[s] = p.st[s];
        a.st[s].raster = p.raster > 0 ? p.raster : STAGE_RASTER_DEFAULT;
    }
    for (int s = 0; s < 3; ++s)
        for (int v = 0; v < 5; ++v) a.rk[s][v] = p.rk[s][v];
    for (int v = 0; v < 5; ++v) a.X[v] = p.X[v];
    a.bar = p.bar;
    a.status = p.status;
    a.wait = (long long)(p.wait_s * 1e3 * (double)khz);
    a.extra = p.extra;
    if ((e = cudaMemsetAsync(p.bar, 0, PERSIST_WORDS * sizeof(unsigned), st)) != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nsm * per);
    cfg.blockDim = dim3(32, WARPS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (grid) *grid = nsm * per;
    return cudaLaunchKernelEx(&cfg, kern, g, a);
}

}  // namespace persist


template <typename R>
cudaError_t launch_short_step_persistent(const Grid &g, const Members &mem, const PersistStepT<R> &p, int scheme,
                                         cudaStream_t st, int *grid)
{
    int maxKA = g.KA;
    for (int q = 0; q < mem.n; ++q) maxKA = mem.m[q].KMAX + 4 > maxKA ? mem.m[q].KMAX + 4 : maxKA;
    if (maxKA > MAXKA) return cudaErrorInvalidValue;
    constexpr int TX = STAGE_TILE_X_DEFAULT;
    switch (scheme) {
    case UD3: return persist::launch_s<UD3, R, TX>(g, mem, p, maxKA, st, grid);
    case CD4: return persist::launch_s<CD4, R, TX>(g, mem, p, maxKA, st, grid);
    case KOREN: return persist::launch_s<KOREN, R, TX>(g, mem, p, maxKA, st, grid);
    case CD2: return persist::launch_s<CD2, R, TX>(g, mem, p, maxKA, st, grid);
    case UD5: return persist::launch_s<UD5, R, TX>(g, mem, p, maxKA, st, grid);
    case CD6: return persist::launch_s<CD6, R, TX>(g, mem, p, maxKA, st, grid);
    default: return cudaErrorInvalidValue;
    }
}
#ifdef HEVI_FLOAT_TU
template cudaError_t launch_short_step_persistent<float>(const Grid &, const Members &, const PersistStepT<float> &,
                                                         int, cudaStream_t, int *);
#else
template cudaError_t launch_short_step_persistent<double>(const Grid &, const Members &, const PersistStepT<double> &,
                                                          int, cudaStream_t, int *);
#endif

}  // namespace hevi
