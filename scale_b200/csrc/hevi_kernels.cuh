// Argument blocks and host launchers of every device kernel of the library.
#pragma once
#include <type_traits>
#include <utility>
#include "hevi_stage.cuh"

namespace hevi {

// ---- ensemble members on the host ----
// A lateral halo fill that the launchers below call between their own kernels
// in place of the periodic fill: fn(ctx, fields, n, elem_bytes) fills n
// (KA,IA,JA) fields of elem_bytes-sized values and returns 0, or a nonzero
// status that makes the launcher return cudaErrorUnknown. Used for the
// exchange of a decomposed domain; null: the periodic fill on the device.
struct HaloFill {
    int (*fn)(void *ctx, void *const *fields, int n, int elem_bytes);
    void *ctx;
};

// The members that share the pooled arrays of one library state; a single
// domain is one member with zero offsets (or no list at all). The launchers
// below run every member in the same launch. A view: the caller owns the array.
struct Members {
    const MemberGeom *m = nullptr;
    int n = 0;
};

// Calls launch(B, nblocks) with the block map of the members for a kernel
// whose per-domain block count is nblocks_of(member Grid): the single-domain
// form BatchT<1> for one member, BatchT<HEVI_MAX_MEMBERS> otherwise.
template <class NB, class L>
cudaError_t with_batch(const Grid &g, const Members &mem, NB nblocks_of, L launch)
{
    if (mem.n <= 1) {
        BatchT<1> B{};
        B.n = 1;
        B.first[0] = 0;
        B.first[1] = nblocks_of(g);
        if (mem.n == 1) B.m[0] = mem.m[0];
        return B.first[1] > 0 ? launch(B, B.first[1]) : cudaSuccess;
    }
    if (mem.n > HEVI_MAX_MEMBERS) return cudaErrorInvalidValue;
    BatchT<HEVI_MAX_MEMBERS> B{};
    B.n = mem.n;
    long long total = 0;
    for (int q = 0; q < B.n; ++q) {
        B.first[q] = (int)total;
        B.m[q] = mem.m[q];
        total += nblocks_of(member_grid(g, mem.m[q]));
    }
    if (total >= (1LL << 31)) return cudaErrorInvalidValue;
    for (int q = B.n; q <= HEVI_MAX_MEMBERS; ++q) B.first[q] = (int)total;
    return launch(B, (int)total);
}

// per-member block index b -> (bx, by) of a kernel whose per-domain grid is gx wide
struct Block2 { int x, y; };
__device__ __forceinline__ Block2 split_block(int b, int gx) { return {b % gx, b / gx}; }

// ---- the HEVI stage with terrain-following metrics (hevi_stage.cu) ----
// GSQRT, J13G, J23G (KA,IA,JA,7), MAPF (IA,JA,2,4), PHI (KA,IA,JA): device arrays
struct Metrics {
    const double *GSQRT, *J13G, *J23G, *MAPF, *PHI;
};
// work arrays of one field each (KA,IA,JA), device memory
struct TerrainWork {
    double *POTT, *DPRES, *qZ, *qX, *qY, *qJ13, *qJ23, *Sr, *Sw, *St;
    double *mZ, *mX, *mY, *tZ, *tX, *tY;
    double *A, *PT, *F1, *F2, *F3, *C, *e, *f;
};
constexpr int TERRAIN_WORK_FIELDS = 24;
constexpr int TERRAIN_STAGE_LAUNCHES = 26; // kernels of one general-metric stage
constexpr int TERRAIN_HEVE_LAUNCHES = 23;  // kernels of one general-metric HEVE stage
cudaError_t launch_terrain_heve_stage(const Grid &g, const StageArgsT<double> &a, const Metrics &M,
                                      const TerrainWork &W, int scheme, cudaStream_t st);
cudaError_t launch_terrain_stage(const Grid &g, const StageArgsT<double> &a, const Metrics &M, const TerrainWork &W,
                                 int scheme, cudaStream_t st);

// ---- numerical filter (numfilter.cu) ----
// coefficient tables built on the host (grid_coef.cpp), 0-based storage of
// CNZ3(3,KA,2), CNX3(3,IA,2), CNY3(3,JA,2) and the nd_coef_* vectors
struct NdCoef {
    const double *CNZ3, *CNX3, *CNY3;
    const double *cdz, *fdz, *cdx, *fdx, *cdy, *fdy; // DIFF4 * D**(4*order) (nd_coef_cdz, ...)
    double sfc;                                      // ND_SFC_FACT
    const double *CNZ4, *CNX4, *CNY4;                // calc_diff4 coefficients (5,KA,2) ...
    int order;                                       // ND_ORDER
};
template <typename R>
struct NdArgsT {
    R *num_diff;
    const double *DENS, *MOMZ, *MOMX, *MOMY, *RHOT, *REF_dens, *REF_pott;
    R *phi; // 5*N3 scratch: the five filtered quantities at every point
};
using NdArgs = NdArgsT<double>;
// status: the library's status word, which also lets one domain use the tiled
// form (launch_numfilter_tiled); null keeps the column form k_numfilter
template <typename R>
cudaError_t launch_numfilter(const Grid &g, const Members &mem, const NdCoef &c, const NdArgsT<R> &a, cudaStream_t st,
                             unsigned *status = nullptr);
// num_diff from the phi scratch by the tiled kernel (hevi_tma.cu) after k_phi has
// filled it; cudaErrorNotSupported where the tiled form does not apply
template <typename R>
cudaError_t launch_numfilter_tiled(const Grid &g, const Members &mem, const NdCoef &c, const NdArgsT<R> &a,
                                   unsigned *status, cudaStream_t st);
// ND_ORDER > 1 (FP64, one domain): the differences of the five quantities go
// through work buffers w1/w2 (15 fields each; component 3*q + dir, dir 0 z,
// 1 x, 2 y) and ND_ORDER-1 applications of calc_diff4 with the periodic halo
// before each; num_diff is then formed from the last one
cudaError_t launch_numfilter_high(const Grid &g, const NdCoef &c, const NdArgs &a, double *w1, double *w2,
                                  cudaStream_t st, const HaloFill *fill = nullptr);
// the member's coefficient tables in the pooled ones (per member: CN*3 hold
// 6 values per level or point, the nd_coef_* vectors one)
__host__ __device__ __forceinline__ NdCoef member_nd(const NdCoef &c, const Grid &g)
{
    NdCoef m = c;
    m.CNZ3 += 6 * (size_t)g.z0; m.CNX3 += 6 * (size_t)g.x0; m.CNY3 += 6 * (size_t)g.y0;
    m.cdz += g.z0; m.fdz += g.z0; m.cdx += g.x0; m.fdx += g.x0; m.cdy += g.y0; m.fdy += g.y0;
    m.CNZ4 += 10 * (size_t)g.z0; m.CNX4 += 10 * (size_t)g.x0; m.CNY4 += 10 * (size_t)g.y0;
    return m;
}

// ---- tracer advection (tracer.cu) ----
// R: the type of the flux and limiter arithmetic and of the flux-like arrays
// (mass fluxes, num_diff, the tendency, the limiter scratch): double on the
// plain path, float on the mixed-precision path. The tracer itself (the stage
// values and QTRC0), the densities and the update stay FP64.
template <typename R>
struct TracerArgsT {
    double *QTRCo;
    const double *QTRC;   // stage input (high-order flux values)
    const double *QTRC0;  // value at the start of the large step (phi_in of the limiter)
    const R *RHOQ_t;
    const double *DENS0, *DENS;
    int dens_mode;        // density of the stage: 0 DENS, 1 DENS0+(DENS-DENS0)/3, 2 DENS0+(DENS-DENS0)*0.5
    const R *mflx;        // (KA,IA,JA,3)
    const R *ndq;         // (KA,IA,JA,3) or null for ND_COEF_Q = 0
    double dtl;
    R *phi_lo, *anti, *rjp, *rjm; // limiter scratch (anti is 3 fields)
    int along_stream;
    // terrain-following metrics, null on flat terrain: GSQRT (KA,IA,JA,7) and
    // the MAPF slice (IA,JA,2) of the mass points (FP64 path only)
    const double *GS, *MAPF;
    // device status word: with it, a limited stage runs the fused form
    // (k_fct_limit, R+/R- halo, k_fct_update) where QTRC0 admits a tensor map
    // and records a staging timeout there; null keeps the three-kernel form
    unsigned *status;
};
using TracerArgs = TracerArgsT<double>;
// one stage; *nk (when given) receives the number of kernels it launched
template <typename R>
cudaError_t launch_tracer_stage(const Grid &g, const TracerArgsT<R> &a, int scheme, bool fct, cudaStream_t st,
                                const HaloFill *fill = nullptr, int *nk = nullptr);
// ATMOS_DYN_divergence with every metric term (misc.cu)
void divergence_terrain(const Grid &g, double *DDIV, const double *MOMZ, const double *MOMX, const double *MOMY,
                        const Metrics &M, double J33G, cudaStream_t st);

// ---- HEVI stage (hevi_stage.cu) ----
// Form and launch shape of the stage. tile_x = 0: the tiled stage (hevi_tma.cu:
// 4 x 4 column tiles staged by bulk tensor copies) where it applies, else the
// fused kernel with its default tile;
// tile_x = 16, 8 or 4: the fused kernel k_hevi_stage with a tile of tile_x x
// (16/tile_x) columns. raster: rows of tiles per raster group; 0 selects the default.
struct StageShape {
    int tile_x = 0, raster = 0;
};
constexpr int STAGE_TILE_XS[3] = {16, 8, 4};
constexpr int STAGE_TILE_X_DEFAULT = 16;
constexpr int STAGE_RASTER_DEFAULT = 16;
// *launches (optional) receives the number of kernels launched, *tiled
// (optional) whether the tiled form ran
template <typename R>
cudaError_t launch_hevi_stage(const Grid &g, const Members &mem, const StageArgsT<R> &a, int scheme, StageShape shape,
                              cudaStream_t st, int *launches = nullptr, bool *tiled = nullptr);
// the tiled stage alone; cudaErrorNotSupported where it does not apply (an
// ensemble, odd KA, a field off a 16-byte boundary, no tiled column scratch)
template <typename R>
cudaError_t launch_hevi_stage_tiled(const Grid &g, const Members &mem, const StageArgsT<R> &a, int scheme, int raster,
                                    cudaStream_t st);
// one HEVE stage (FP64), same arguments; the RK4 combine modes apply as for HEVI
cudaError_t launch_heve_stage(const Grid &g, const Members &mem, const StageArgsT<double> &a, int scheme,
                              cudaStream_t st);

// ---- utilities (misc.cu) ----
template <typename T>
void periodic_halo(const Grid &g, const Members &mem, T *const *fields, int nf, cudaStream_t st);
void divergence(const Grid &g, double *DDIV, const double *MOMZ, const double *MOMX, const double *MOMY,
                const double *RCDZ, const double *RCDX, const double *RCDY, double J33G, cudaStream_t st);
void vertical_bc(const Grid &g, const Members &mem, double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT,
                 cudaStream_t st);
struct PrepArgs {
    double *RT2P, *DPRES0, *REF_rhot;
    const double *RHOT, *QTRC, *REF_pres;
    int QA;
    double AQ_R[8], AQ_CV[8], AQ_CP[8], AQ_MASS[8];
};
void large_prep(const Grid &g, const PrepArgs &a, cudaStream_t st);
void count_not_equal(const double *p, size_t n, double want, unsigned long long *count, cudaStream_t st);
void domain_sum(const Grid &g, const double *var, const double *CDX, const double *CDY, const double *CDZ,
                double *part, double *out, cudaStream_t st);
// FP64 totals of ENGT, ENGP, ENGK, ENGI (dry air) into out[0..3]; part: 4*IMAX*JMAX
void energy_sum(const Grid &g, const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY,
                const double *RHOT, const double *CZ, const double *CDX, const double *CDY, const double *CDZ,
                double *part, double *out, cudaStream_t st);
void mflx_accumulate(const Grid &g, double *av, const double *mflx, cudaStream_t st);
void mflx_average(const Grid &g, double *mflx, const double *av, int nstep, cudaStream_t st);

// message returned by scale_hevi_last_error() (capi.cu)
void set_last_error(const char *msg);

// ---- the persistent short step (persist.cu) ----
// One short step of every member as one cooperative launch: the numerical
// filter (ND_ORDER = 1), the four RK4 HEVI stages with the halo of stages 1-3,
// the vertical boundary values and the halo of the state. Flat terrain, no
// divergence damping, the fused stage's default tile width.
template <typename R>
struct PersistStepT {
    NdCoef ndc;
    NdArgsT<R> nd;
    StageArgsT<R> st[4];
    double *rk[3][5];  // outputs of stages 1-3 (the inputs of stages 2-4)
    double *X[5];      // the state, written by stage 4
    unsigned *bar;     // PERSIST_WORDS device words: the grid barriers' arrival count, then per-phase work counters
    unsigned *status;
    int raster;        // rows of tiles per raster group of the stage phases
    double wait_s;     // time limit of each grid barrier
    unsigned extra;    // arrivals each barrier waits for beyond the grid's own (0; a test of the limit sets 1)
};
constexpr int PERSIST_WORDS = 64;
template <typename R>
cudaError_t launch_short_step_persistent(const Grid &g, const Members &mem, const PersistStepT<R> &p, int scheme,
                                         cudaStream_t st, int *grid);

}  // namespace hevi
