// The HEVI stage (ATMOS_DYN_Tstep_short_fvm_hevi,
// scalelib/src/atmos-rm/dynamics/scale_atmos_dyn_tstep_short_fvm_hevi.F90:128-1089)
// as one kernel, k_hevi_tiled, that stages its tiles in shared memory with the
// tensor memory accelerator (TMA). Line numbers refer to that file unless a
// flux file is named.
//
// A CTA owns a 4 x 4 tile of columns, one warp per column with its lanes along
// k. It marches up the columns in chunks of 32 levels. For each chunk one
// thread issues cp.async.bulk.tensor copies of the five state fields (DENS,
// MOMZ, MOMX, MOMY, RHOT) over the tile, its lateral halo (2 points; 3 for the
// 6-point schemes) and the levels from 4 below to 2-3 above the chunk into
// shared memory, completing on an mbarrier; the tensor maps cover this GPU's
// own memory and the copies have no cluster multicast. Every stencil then
// reads shared memory at compile-time offsets. Per chunk:
//   a. the pressure deviation DPRES (hevi_pres :343-361) of the tile and of its
//      +x/+y neighbour columns; RHOT -> POTT in place (:586-600)
//   b. x/y mass fluxes (:399-438), Sr (:443-479), PT and the vertical theta
//      flux (valueW_Z, fluxZ_XYZ), the x/y theta fluxes and St (:603-661)
//   c. one level lower: Sw (:528-578) and the right-hand side C (:698-722)
//   d. rho*u and rho*v (hevi_momx :814-928, hevi_momy :934-1048)
// The z flux through the face below a level is the previous lane's flux
// above it, by a warp shuffle; lane 0 takes the previous chunk's lane 31's.
// Chunks clear of the near-wall face forms run without level dispatch.
// The fluxes and momenta leave through the RK folds of put_flux/put_state;
// Sr, St, tZ, PT and C go to the column scratch. After the march the staged
// box holds the tile's column arrays: C, PT and A(k) come back from the
// scratch (L2-resident), warp 0 runs the Thomas solve (solve_direct
// :1092-1127) one lane per column, and the warps back-update rho, rho*w,
// rho*theta and the vertical fluxes (:728-790). While one CTA of an SM solves,
// the other keeps the SM's issue slots busy with its march.
//
// Every value keeps the operation order of the fused kernel k_hevi_stage
// (hevi_stage.cu) and of the reference, so the two forms give identical bits.
// Flat terrain, one domain, even KA (the tensor maps need 16-byte strides);
// the launcher returns cudaErrorNotSupported otherwise and the fused kernel runs.
#include "hevi_epilogue.cuh"
#include "hevi_kernels.cuh"
#include "numfilter_body.cuh"
#include "tma_util.cuh"

namespace hevi {
namespace tma {

constexpr int TX = 4, TY = 4, NCOL = TX * TY; // tile columns; one warp each
constexpr int KC = 32;                        // levels per chunk (one per lane)
constexpr int KLO = 4;                        // box levels below the chunk's first level
template <int S> __host__ __device__ constexpr int reach() { return wide_scheme(S) ? 3 : 2; }
// box levels: L0-4 .. L0+33 (4-point schemes) or L0-4 .. L0+35 (6-point), L0
// the chunk's first level; 38 and 40 keep the inner box a multiple of 16 bytes
template <int S> __host__ __device__ constexpr int box_k() { return wide_scheme(S) ? 40 : 38; }
template <int S> __host__ __device__ constexpr int box_w() { return TX + 2 * reach<S>(); }
template <int S> __host__ __device__ constexpr int box_h() { return TY + 2 * reach<S>(); }
template <int S> __host__ __device__ constexpr int plane() { return box_k<S>() * box_w<S>() * box_h<S>(); }
constexpr int NF = 5;                         // staged fields
enum StagedField : int { F_DN = 0, F_MZ = 1, F_MX = 2, F_MY = 3, F_RT = 4 };
constexpr int NDP = 33;                       // DPRES levels per column: L0-1 .. L0+31
constexpr int DP_COLS = (TX + 1) * (TY + 1);  // tile columns and their +x/+y neighbours
constexpr int NLT = 6;                        // level tables per chunk: RCDZ, RFDZ, F2H1, F2H2, FDZ, wdamp

template <int S> constexpr size_t smem_bytes()
{
    return (size_t)NF * plane<S>() * sizeof(double) + (size_t)(DP_COLS + NCOL + NLT) * NDP * sizeof(double) + 16;
}

struct StateMaps {
    CUtensorMap m[NF]; // DENS, MOMZ, MOMX, MOMY, RHOT as (KA, IA, JA) FP64 tensors
};

// =============================================================================
// k_hevi_explicit
// =============================================================================
// the face value at w-level m in a chunk that lies clear of the near-wall
// forms: zface<S> without its level dispatch
template <int S, typename R, typename V>
__device__ __forceinline__ R zface_in(R vel, int m, const V &v)
{
    if constexpr (wide_scheme(S)) return ip6<S>(vel, v(m - 2), v(m - 1), v(m), v(m + 1), v(m + 2), v(m + 3));
    else return ip4<S>(vel, v(m - 1), v(m), v(m + 1), v(m + 2));
}

template <int S, typename R, int NM>
__global__ void __launch_bounds__(32 * NCOL, 2)
    k_hevi_explicit(const Grid gt, const StageArgsT<R> a, const BatchT<NM> B, const __grid_constant__ StateMaps maps)
{
    constexpr int H = reach<S>(), BW = box_w<S>(), BK = box_k<S>(), PL = plane<S>();
    constexpr int KX = BK, KY = BW * BK; // shared-memory strides of one column step in i and in j
    constexpr bool W6 = wide_scheme(S);
    extern __shared__ __align__(1024) double sm[];
    double *stg = sm;                    // NF staged fields, [j][i][k] each
    double *sdp = sm + NF * PL;          // DPRES, [DP_COLS][NDP]
    double *srp = sdp + DP_COLS * NDP;   // RT2P of the tile's own columns, [NCOL][NDP]
    double *slt = srp + NCOL * NDP;      // the chunk's level tables, [NLT][NDP]
    uint64_t *bar = reinterpret_cast<uint64_t *>(slt + NLT * NDP);
    __shared__ int s_ok;

    int b;
    const Grid g = block_domain(gt, B, b);
    const int lane = threadIdx.x, w = threadIdx.y, tid = w * 32 + lane;
    const int tx = w % TX, ty = w / TX;
    int ti, tj;
    {
        // raster: consecutive CTAs walk down a.raster rows of tiles, then step in i
        const int nti = (g.IMAX + TX - 1) / TX, ntj = (g.JMAX + TY - 1) / TY, RJ = a.raster;
        const int grp = b / (nti * RJ), rem = b - grp * (nti * RJ);
        const int rows = min(RJ, ntj - grp * RJ);
        tj = grp * RJ + rem % rows;
        ti = rem / rows;
    }
    const int i0 = g.IS + ti * TX, j0 = g.JS + tj * TY;
    const int i = i0 + tx, j = j0 + ty;
    const bool col_ok = i <= g.IE && j <= g.JE;
    const size_t N3 = n3(g);
    const int sI = g.KA, sJ = g.KA * g.IA;
    const int KS = g.KS, KE = g.KE;
    const int col = (int)idx3(g, 1, i, j); // offset of level 1 of this warp's column
    const Nd<R> nd(a, N3);
    const double dt = a.dtrk, J33G = a.J33G;
    const bool use_div = a.divdmp_coef != 0.0;
    const R ddc = use_div ? R(a.divdmp_coef / dt) : R(0.0);
    const R rcdx = col_ok ? R(ld(g.RCDX + i - 1)) : R(0.0), rcdy = col_ok ? R(ld(g.RCDY + j - 1)) : R(0.0);
    const R h = R(0.5), qr = R(0.25), J33R = R(J33G);
    const unsigned FULL = 0xffffffffu;
    const int NC = (g.KMAX + KC - 1) / KC;
    R *const sSr = a.colscr, *const sSt = a.colscr + N3, *const stZ = a.colscr + 2 * N3, *const sPT = a.colscr + 3 * N3;

    auto issue = [&](int ch) {
        // box origin (0-based): level L0-4 = 32*ch - 2 (even, so its byte offset is a
        // multiple of 16), column i0-H, row j0-H
        const int x = KC * ch + (KS - 1) - KLO, y = i0 - H - 1, z = j0 - H - 1;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(bar, (unsigned)(NF * PL * sizeof(double)));
        for (int f = 0; f < NF; ++f) tma_load_3d(stg + f * PL, &maps.m[f], x, y, z, bar);
    };
    if (tid == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        issue(0);
    }
    __syncthreads();

    // this warp's column in the staged box, at the lane's level of the chunk
    const int cbox = ((ty + H) * BW + (tx + H)) * BK + KLO + lane;
    const double *sDN = stg + F_DN * PL + cbox, *sMZ = stg + F_MZ * PL + cbox;
    const double *sMX = stg + F_MX * PL + cbox, *sMY = stg + F_MY * PL + cbox;
    double *sPO = stg + F_RT * PL + cbox; // RHOT, then POTT
    // Values of the previous chunk's lane 31 that lane 0 of the next chunk
    // needs: the fluxes through the face below its level (mass, theta, w, u, v)
    // and Sr, St one level down. Zero below KS, where every one of them is zero.
    R Sr_prev = R(0.0), St_prev = R(0.0);
    R cy_mZ = R(0.0), cy_tZ = R(0.0), cy_qw = R(0.0), cy_qu = R(0.0), cy_qv = R(0.0);
    double cy_rd = 0.0; // REF_dens one level down
    // broadcast of lane 31's value (the carry into the next chunk)
    auto from31 = [&](R v) { return __shfl_sync(FULL, v, 31); };

    for (int ch = 0; ch < NC; ++ch) {
        const int L0 = KS + KC * ch, L = L0 + lane;
        // ---- the chunk's copies: thread 0 waits (bounded), the block learns the outcome ----
        if (tid == 0) {
            const bool ok = mbar_wait(bar, ch & 1);
            // on a timeout, wait once more (bounded) for the copies still in flight
            // into this block's shared memory before the block leaves
            if (!ok) (void)mbar_wait(bar, ch & 1);
            s_ok = ok ? 1 : 0;
        }
        __syncthreads();
        if (!s_ok) {
            if (tid == 0) atomicOr(a.status, ST_TMA_TIMEOUT);
            return; // block-uniform
        }
        (void)mbar_try(bar, ch & 1); // completed phase: makes the copied data visible to this thread

        // ---- a. the chunk's level tables (levels L0-1..L0+31, clamped to KE), DPRES
        // of the tile and its +x/+y neighbours (:355) ----
        if (w == NCOL - 1) {
            for (int lv = lane; lv < NDP; lv += 32) {
                const int Lq = min(L0 - 1 + lv, KE);
                slt[0 * NDP + lv] = ld(g.RCDZ + Lq - 1);
                slt[1 * NDP + lv] = ld(g.RFDZ + Lq - 1);
                slt[2 * NDP + lv] = ld(g.F2H1 + Lq - 1);
                slt[3 * NDP + lv] = ld(g.F2H2 + Lq - 1);
                slt[4 * NDP + lv] = ld(g.FDZ + Lq - 1);
                slt[5 * NDP + lv] = ld(a.wdamp + g.z0 + Lq - 1);
            }
        }
        for (int q = w; q < DP_COLS; q += NCOL) {
            const int qx = q % (TX + 1), qy = q / (TX + 1);
            const int ii = i0 + qx, jj = j0 + qy;
            if (ii > g.IE + 1 || jj > g.JE + 1) continue;
            const int cq = (int)idx3(g, 1, ii, jj);
            const double *rt = stg + F_RT * PL + ((qy + H) * BW + (qx + H)) * BK + KLO - 1;
            for (int lv = lane; lv < NDP; lv += 32) {
                const int Lq = L0 - 1 + lv;
                if (Lq > KE) break;
                const int cc = cq + Lq - 1;
                const double rt2p = ld(a.RT2P + cc);
                sdp[q * NDP + lv] = ld(a.DPRES0 + cc) + rt2p * (rt[lv] - ld(a.REF_rhot + cc));
                if (qx < TX && qy < TY) srp[(qy * TX + qx) * NDP + lv] = rt2p;
            }
        }
        __syncthreads();
        // RHOT -> POTT = RHOT/DENS (:586-600): the tile's own columns over the whole
        // box height (the vertical stencils), the x/y arms of the halo at the chunk's
        // levels (the horizontal theta fluxes)
        for (int lv = lane; lv < BK; lv += 32) {
            double *p = sPO - lane - KLO + lv; // box level lv of this warp's column
            p[0] = (double)(R(p[0]) / R(p[(F_DN - F_RT) * PL]));
        }
        for (int q = w; q < 2 * H * (TX + TY); q += NCOL) {
            int bx, by;
            if (q < 2 * H * TY) {
                const int s = q % (2 * H);
                by = q / (2 * H) + H;
                bx = s < H ? s : s + TX;
            } else {
                const int q2 = q - 2 * H * TY, s = q2 % (2 * H);
                bx = q2 / (2 * H) + H;
                by = s < H ? s : s + TY;
            }
            double *p = stg + F_RT * PL + (by * BW + bx) * BK + KLO + lane;
            p[0] = (double)(R(p[0]) / R(p[(F_DN - F_RT) * PL]));
        }
        __syncthreads();

        // Chunks clear of the near-wall face forms (every face of the chunk, from
        // the one below L0-1 to the one above L0+31, in the interior range, and
        // every level of the chunk at or below KE) run without level dispatch or
        // range checks: EDGE = false.
        const bool interior = L0 - 1 >= KS + (W6 ? 2 : 1) && L0 + 31 <= KE - (W6 ? 3 : 2);
        // the level tables at this lane's level L (slot lane+1) and at k = L-1 (slot lane)
        const double *lt = slt + lane;
#define rcdz_L lt[0 * NDP + 1]
#define rfdz_k lt[1 * NDP]
#define f1_L lt[2 * NDP + 1]
#define f1_k lt[2 * NDP]
#define f2_L lt[3 * NDP + 1]
#define f2_k lt[3 * NDP]
#define fdz_k lt[4 * NDP]
#define wd_k lt[5 * NDP]
        auto chunk = [&](auto edge) {
            constexpr bool EDGE = decltype(edge)::value;
            auto zf = [&](R vel, int m, const auto &v) -> R {
                if constexpr (EDGE) return zface<S>(vel, m, KS, KE, v);
                else return zface_in<S>(vel, m, v);
            };
            // ---- b. level L: mass and theta fluxes, Sr, St, PT, tZ ----
            const bool vb = col_ok && (!EDGE || L <= KE);
            const int c = col + L - 1;
            R Sr = R(0.0), St = R(0.0);
            {
                // the vertical mass flux through the face above L (hevi_mflx_z :383-391);
                // the face below is the previous lane's (lane 0: the previous chunk's lane 31)
                const R mZ = (vb && (!EDGE || L <= KE - 1)) ? ld(nd.DZ() + c) : R(0.0);
                R mZm1 = __shfl_up_sync(FULL, mZ, 1);
                if (lane == 0) mZm1 = cy_mZ;
                cy_mZ = from31(mZ);
                auto P = [&](int l) { return R(sPO[l - L]); };
                R PT = R(0.0), tZ = R(0.0);
                if (vb && (!EDGE || L <= KE - 1)) {
                    // PT: valueW_Z (ud3.F90:98-153); tZ: fluxZ_XYZ (ud3.F90:157-247)
                    PT = zf(R(sMZ[0]), L, P);
                    tZ = mZ * zf(mZ, L, P) + lds(nd.TZ() + c);
                }
                R tZm = __shfl_up_sync(FULL, tZ, 1);
                if (lane == 0) tZm = cy_tZ;
                cy_tZ = from31(tZ);
                if (vb) {
                    const R Xe = R(sMX[0]) + ld(nd.DX() + c), Xw = R(sMX[-KX]) + ld(nd.DX() + c - sI);
                    const R Yn = R(sMY[0]) + ld(nd.DY() + c), Ys = R(sMY[-KY]) + ld(nd.DY() + c - sJ);
                    const R adv_r = -((Xe - Xw) * rcdx + (Yn - Ys) * rcdy);
                    put_flux(a, N3, 1, c, Xe, true);
                    put_flux(a, N3, 2, c, Yn, true);
                    if (i == g.IS) put_flux(a, N3, 1, c - sI, Xw, false);
                    if (j == g.JS) put_flux(a, N3, 2, c - sJ, Ys, false);
                    const R rcdz = R(rcdz_L);
                    Sr = (-(mZ - mZm1) * rcdz + adv_r) + lds(a.DENS_t + c);
                    // fluxX/Y_XYZ (ud3.F90:251-353)
                    const R P00 = R(sPO[0]);
                    const R Pm2 = R(sPO[-2 * KX]), Pm1 = R(sPO[-KX]), Pp1 = R(sPO[KX]), Pp2 = R(sPO[2 * KX]);
                    const R Qm2 = R(sPO[-2 * KY]), Qm1 = R(sPO[-KY]), Qp1 = R(sPO[KY]), Qp2 = R(sPO[2 * KY]);
                    const R Pm3 = W6 ? R(sPO[-3 * KX]) : R(0.0), Pp3 = W6 ? R(sPO[3 * KX]) : R(0.0);
                    const R Qm3 = W6 ? R(sPO[-3 * KY]) : R(0.0), Qp3 = W6 ? R(sPO[3 * KY]) : R(0.0);
                    const R tXe = Xe * ip6<S>(Xe, Pm2, Pm1, P00, Pp1, Pp2, Pp3) + ld(nd.TX() + c);
                    const R tXw = Xw * ip6<S>(Xw, Pm3, Pm2, Pm1, P00, Pp1, Pp2) + ld(nd.TX() + c - sI);
                    const R tYn = Yn * ip6<S>(Yn, Qm2, Qm1, P00, Qp1, Qp2, Qp3) + ld(nd.TY() + c);
                    const R tYs = Ys * ip6<S>(Ys, Qm3, Qm2, Qm1, P00, Qp1, Qp2) + ld(nd.TY() + c - sJ);
                    const R adv_t = -((tXe - tXw) * rcdx + (tYn - tYs) * rcdy); // hevi_st :646-648
                    put_flux(a, N3, 4, c, tXe, true);
                    put_flux(a, N3, 5, c, tYn, true);
                    if (i == g.IS) put_flux(a, N3, 4, c - sI, tXw, false);
                    if (j == g.JS) put_flux(a, N3, 5, c - sJ, tYs, false);
                    St = (-(tZ - tZm) * rcdz + adv_t) + lds(a.RHOT_t + c); // hevi_st :646-649
                    sSr[c] = Sr;
                    sSt[c] = St;
                    stZ[c] = tZ;
                    sPT[c] = PT;
                }
            }

            // ---- c. level k = L-1: Sw (hevi_sw :528-578) and C(k) (:698-722) ----
            {
                R Sr_k = __shfl_up_sync(FULL, Sr, 1), St_k = __shfl_up_sync(FULL, St, 1);
                if (lane == 0) { Sr_k = Sr_prev; St_k = St_prev; }
                Sr_prev = from31(Sr);
                St_prev = from31(St);
                const int k = L - 1;
                const bool vc = col_ok && (!EDGE || (k >= KS && k <= KE - 1));
                const double *cMZ = sMZ - 1, *cDN = sDN - 1, *cMX = sMX - 1, *cMY = sMY - 1; // level k
                const int ck = c - 1;
                auto vMZ = [&](int l) { return R(cMZ[l - k]); };
                // vertical w-momentum flux above level k, fluxZ_XYW (ud3.F90:358-452),
                // zero outside KS..KE-2; the one below is the previous lane's
                R q_k = R(0.0);
                if (vc && (!EDGE || k <= KE - 2)) {
                    const R vel = (R(0.5) * (vMZ(k) + vMZ(k + 1))) / R(cDN[1]);
                    q_k = J33R * vel * zf(vel, k, vMZ) + lds(nd.WZ() + col + k);
                }
                R q_km = __shfl_up_sync(FULL, q_k, 1);
                if (lane == 0) q_km = cy_qw;
                cy_qw = from31(q_k);
                const double rd1 = vb ? lds(a.REF_dens + c) : 0.0; // REF_dens(k+1)
                double rd0 = __shfl_up_sync(FULL, rd1, 1);         // REF_dens(k)
                if (lane == 0) rd0 = cy_rd;
                cy_rd = __shfl_sync(FULL, rd1, 31);
                if (vc) {
                    // horizontal w-momentum flux divergence, fluxX/Y_XYW (ud3.F90:598-748)
                    R adv_w;
                    {
                        const R f1 = R(f1_k), f2 = R(f2_k);
                        const R vXe = (f1 * R(cMX[1]) + f2 * R(cMX[0]))
                                      / (f1 * h * (R(cDN[1]) + R(cDN[1 + KX])) + f2 * h * (R(cDN[0]) + R(cDN[KX])));
                        const R vXw = (f1 * R(cMX[1 - KX]) + f2 * R(cMX[-KX]))
                                      / (f1 * h * (R(cDN[1 - KX]) + R(cDN[1])) + f2 * h * (R(cDN[-KX]) + R(cDN[0])));
                        const R vYn = (f1 * R(cMY[1]) + f2 * R(cMY[0]))
                                      / (f1 * h * (R(cDN[1]) + R(cDN[1 + KY])) + f2 * h * (R(cDN[0]) + R(cDN[KY])));
                        const R vYs = (f1 * R(cMY[1 - KY]) + f2 * R(cMY[-KY]))
                                      / (f1 * h * (R(cDN[1 - KY]) + R(cDN[1])) + f2 * h * (R(cDN[-KY]) + R(cDN[0])));
                        const R W_m2 = R(cMZ[-2 * KX]), W_m1 = R(cMZ[-KX]), W_00 = R(cMZ[0]);
                        const R W_p1 = R(cMZ[KX]), W_p2 = R(cMZ[2 * KX]);
                        const R V_m2 = R(cMZ[-2 * KY]), V_m1 = R(cMZ[-KY]), V_p1 = R(cMZ[KY]), V_p2 = R(cMZ[2 * KY]);
                        const R W_m3 = W6 ? R(cMZ[-3 * KX]) : R(0.0), W_p3 = W6 ? R(cMZ[3 * KX]) : R(0.0);
                        const R V_m3 = W6 ? R(cMZ[-3 * KY]) : R(0.0), V_p3 = W6 ? R(cMZ[3 * KY]) : R(0.0);
                        const R qXe = vXe * ip6<S>(vXe, W_m2, W_m1, W_00, W_p1, W_p2, W_p3) + ld(nd.WX() + ck);
                        const R qXw = vXw * ip6<S>(vXw, W_m3, W_m2, W_m1, W_00, W_p1, W_p2) + ld(nd.WX() + ck - sI);
                        const R qYn = vYn * ip6<S>(vYn, V_m2, V_m1, W_00, V_p1, V_p2, V_p3) + ld(nd.WY() + ck);
                        const R qYs = vYs * ip6<S>(vYs, V_m3, V_m2, V_m1, W_00, V_p1, V_p2) + ld(nd.WY() + ck - sJ);
                        adv_w = -((qXe - qXw) * rcdx + (qYn - qYs) * rcdy);
                    }
                    const R advcv = -(q_k - q_km) * R(rfdz_k);
                    const R wdmp = -R(wd_k) * R(ld(a.MOMZ0 + ck));
                    const R div = use_div ? ddc * (ld(a.DDIV + ck + 1) - ld(a.DDIV + ck)) * R(fdz_k) : R(0.0);
                    const R Sw = (advcv + adv_w) + wdmp + div + lds(a.MOMZ_t + ck);
                    const double rfdz = rfdz_k;
                    const double *rp = srp + w * NDP + lane; // RT2P at level k
                    const double RTL1 = rp[1], RTL0 = rp[0];
                    const double *dp = sdp + (ty * (TX + 1) + tx) * NDP + lane; // DPRES at level k (slot k-L0+1 = lane)
                    const double pg = -(dp[1] + RTL1 * dt * (double)St - dp[0] - RTL0 * dt * (double)St_k) * rfdz * J33G
                                      - GRAV * (f1_k * (cDN[1] - rd1 + (double)Sr * dt)
                                                + f2_k * (cDN[0] - rd0 + (double)Sr_k * dt));
                    a.colC[ck] = cMZ[0] + dt * (pg + (double)Sw);
                }
            }

            // ---- d. rho*u (hevi_momx :814-928) and rho*v (hevi_momy :934-1048) at level L ----
            {
                const double *dp = sdp + (ty * (TX + 1) + tx) * NDP + lane + 1; // DPRES at level L, this column
                auto vMX = [&](int l) { return R(sMX[l - L]); };
                auto vMY = [&](int l) { return R(sMY[l - L]); };
                const bool do_u = vb && i <= g.IEH, do_v = vb && j <= g.JEH;
                const bool zok = !EDGE || L <= KE - 1; // the face above L carries a flux
                // u: the z flux at (u,y,w) above L, fluxZ_UYZ (ud3.F90:753-859); the one
                // below is the previous lane's
                {
                    R q_k = R(0.0);
                    if (do_u && zok) {
                        const R den = R(f1_L) * h * (R(sDN[1]) + R(sDN[1 + KX]))
                                      + R(f2_L) * h * (R(sDN[0]) + R(sDN[KX]));
                        const R vel = (h * (R(sMZ[0]) + R(sMZ[KX]))) / den;
                        q_k = J33R * vel * zf(vel, L, vMX) + lds(nd.UZ() + c);
                    }
                    R q_km = __shfl_up_sync(FULL, q_k, 1);
                    if (lane == 0) q_km = cy_qu;
                    cy_qu = from31(q_k);
                    if (do_u) {
                        const R fdx = R(ld(g.FDX + i - 1));
                        const double rfdx = ld(g.RFDX + i - 1);
                        const R cor_u = R(0.125) * (R(ld(a.CORIOLI + g.c2 + (i) + (size_t)g.IA * (j - 1)))
                                                    + R(ld(a.CORIOLI + g.c2 + (i - 1) + (size_t)g.IA * (j - 1))));
                        const R U_m2 = R(sMX[-2 * KX]), U_m1 = R(sMX[-KX]), U_00 = R(sMX[0]);
                        const R U_p1 = R(sMX[KX]), U_p2 = R(sMX[2 * KX]);
                        // x flux at (x,y,z) with the index shift of fluxX_UYZ (ud3.F90:1053-1109)
                        const R vE = (h * (U_p1 + U_00)) / (R(sDN[KX]));
                        const R U_m3 = W6 ? R(sMX[-3 * KX]) : R(0.0), U_p3 = W6 ? R(sMX[3 * KX]) : R(0.0);
                        const R qXe = vE * ip6<S>(vE, U_m2, U_m1, U_00, U_p1, U_p2, U_p3) + ld(nd.UX() + c + sI);
                        const R vW = (h * (U_00 + U_m1)) / (R(sDN[0]));
                        const R qXw = vW * ip6<S>(vW, U_m3, U_m2, U_m1, U_00, U_p1, U_p2) + ld(nd.UX() + c);
                        // y flux at (u,v,z), fluxY_UYZ (ud3.F90:1113-1167)
                        const R vN = (h * (R(sMY[0]) + R(sMY[KX])))
                                     / (qr * (R(sDN[0]) + R(sDN[KX]) + R(sDN[KY]) + R(sDN[KX + KY])));
                        const R qYn = vN * ip6<S>(vN, W6 ? R(sMX[-2 * KY]) : R(0.0), R(sMX[-KY]), U_00, R(sMX[KY]),
                                                  R(sMX[2 * KY]), W6 ? R(sMX[3 * KY]) : R(0.0)) + ld(nd.UY() + c);
                        const R vS = (h * (R(sMY[-KY]) + R(sMY[KX - KY])))
                                     / (qr * (R(sDN[-KY]) + R(sDN[KX - KY]) + R(sDN[0]) + R(sDN[KX])));
                        const R qYs = vS * ip6<S>(vS, W6 ? R(sMX[-3 * KY]) : R(0.0), R(sMX[-2 * KY]), R(sMX[-KY]), U_00,
                                                  R(sMX[KY]), W6 ? R(sMX[2 * KY]) : R(0.0)) + ld(nd.UY() + c - sJ);
                        const R advcv = -(q_k - q_km) * R(rcdz_L);
                        const R advch = -((qXe - qXw) * R(rfdx) + (qYn - qYs) * rcdy);
                        const double DPe = dp[NDP]; // DPRES at (i+1, j)
                        const double pg = (DPe - dp[0]) * rfdx;
                        const R cf = cor_u * (R(sMY[KX]) + R(sMY[0]) + R(sMY[KX - KY]) + R(sMY[-KY]));
                        const R div = !use_div ? R(0.0) : ddc * (ld(a.DDIV + c + sI) - ld(a.DDIV + c)) * fdx;
                        const double val = lds(a.MOMX0 + c)
                                           + dt * (((((double)(advcv + advch)) - pg) + (double)cf) + (double)div
                                                   + (double)lds(a.MOMX_t + c));
                        put_state(a, N3, 2, a.MOMX_RK, a.MOMX0, c, val, true);
                    }
                }
                // v: the z flux at (x,v,w), fluxZ_XVZ (ud3.F90:1173-1279)
                {
                    R q_k = R(0.0);
                    if (do_v && zok) {
                        const R den = R(f1_L) * h * (R(sDN[1]) + R(sDN[1 + KY]))
                                      + R(f2_L) * h * (R(sDN[0]) + R(sDN[KY]));
                        const R vel = (h * (R(sMZ[0]) + R(sMZ[KY]))) / den;
                        q_k = J33R * vel * zf(vel, L, vMY) + lds(nd.VZ() + c);
                    }
                    R q_km = __shfl_up_sync(FULL, q_k, 1);
                    if (lane == 0) q_km = cy_qv;
                    cy_qv = from31(q_k);
                    if (do_v) {
                        const R fdy = R(ld(g.FDY + j - 1));
                        const double rfdy = ld(g.RFDY + j - 1);
                        const R cor_v = R(-0.125) * (R(ld(a.CORIOLI + g.c2 + (i - 1) + (size_t)g.IA * (j)))
                                                     + R(ld(a.CORIOLI + g.c2 + (i - 1) + (size_t)g.IA * (j - 1))));
                        const R Y_m2 = R(sMY[-2 * KY]), Y_m1 = R(sMY[-KY]), Y_00 = R(sMY[0]);
                        const R Y_p1 = R(sMY[KY]), Y_p2 = R(sMY[2 * KY]);
                        // x flux at (u,v,z), fluxX_XVZ (ud3.F90:1473-1527)
                        const R vE = (h * (R(sMX[0]) + R(sMX[KY])))
                                     / (qr * (R(sDN[0]) + R(sDN[KX]) + R(sDN[KY]) + R(sDN[KX + KY])));
                        const R qXe = vE * ip6<S>(vE, W6 ? R(sMY[-2 * KX]) : R(0.0), R(sMY[-KX]), Y_00, R(sMY[KX]),
                                                  R(sMY[2 * KX]), W6 ? R(sMY[3 * KX]) : R(0.0)) + ld(nd.VX() + c);
                        const R vW = (h * (R(sMX[-KX]) + R(sMX[KY - KX])))
                                     / (qr * (R(sDN[-KX]) + R(sDN[0]) + R(sDN[KY - KX]) + R(sDN[KY])));
                        const R qXw = vW * ip6<S>(vW, W6 ? R(sMY[-3 * KX]) : R(0.0), R(sMY[-2 * KX]), R(sMY[-KX]), Y_00,
                                                  R(sMY[KX]), W6 ? R(sMY[2 * KX]) : R(0.0)) + ld(nd.VX() + c - sI);
                        // y flux with the index shift of fluxY_XVZ (ud3.F90:1531-1587)
                        const R vN = (h * (Y_p1 + Y_00)) / (R(sDN[KY]));
                        const R Y_m3 = W6 ? R(sMY[-3 * KY]) : R(0.0), Y_p3 = W6 ? R(sMY[3 * KY]) : R(0.0);
                        const R qYn = vN * ip6<S>(vN, Y_m2, Y_m1, Y_00, Y_p1, Y_p2, Y_p3) + ld(nd.VY() + c + sJ);
                        const R vS = (h * (Y_00 + Y_m1)) / (R(sDN[0]));
                        const R qYs = vS * ip6<S>(vS, Y_m3, Y_m2, Y_m1, Y_00, Y_p1, Y_p2) + ld(nd.VY() + c);
                        const R advcv = -(q_k - q_km) * R(rcdz_L);
                        const R advch = -((qXe - qXw) * rcdx + (qYn - qYs) * R(rfdy));
                        const double DPn = dp[(TX + 1) * NDP]; // DPRES at (i, j+1)
                        const double pg = (DPn - dp[0]) * rfdy;
                        const R cf = cor_v * (R(sMX[KY]) + R(sMX[0]) + R(sMX[KY - KX]) + R(sMX[-KX]));
                        const R div = !use_div ? R(0.0) : ddc * (ld(a.DDIV + c + sJ) - ld(a.DDIV + c)) * fdy;
                        const double val = lds(a.MOMY0 + c)
                                           + dt * (((((double)(advcv + advch)) - pg) + (double)cf) + (double)div
                                                   + (double)lds(a.MOMY_t + c));
                        put_state(a, N3, 3, a.MOMY_RK, a.MOMY0, c, val, true);
                    }
                }
            }
        };
        if (interior) chunk(std::false_type{});
        else chunk(std::true_type{});
#undef rcdz_L
#undef rfdz_k
#undef f1_L
#undef f1_k
#undef f2_L
#undef f2_k
#undef fdz_k
#undef wd_k
        __syncthreads(); // every read of the staged box and of DPRES is done
        if (tid == 0 && ch + 1 < NC) issue(ch + 1);
    }

}

// =============================================================================
// k_hevi_column: the column problem of CCOLS columns per CTA
// =============================================================================
// The CTA loads C, PT and A(k) of its columns into shared memory, and the
// per-level factors B(k) and RFDZ(k) of the coefficients once for all of
// them. Warp 0 runs the Thomas solve (solve_direct :1092-1127) one lane per
// column: the coefficients of level k+1 are formed while the division of
// level k runs, so that only e(k-1) and f(k-1) chain the levels. Then all warps
// back-update rho, rho*w, rho*theta and the vertical fluxes (:728-790).
constexpr int CCOLS = 16;  // columns per CTA (consecutive in i)
constexpr int CWARPS = 8;
__host__ __device__ inline int col_pitch_c(int KA) { return KA | 1; }
__host__ __device__ inline size_t column_smem(int KA) { return ((size_t)3 * CCOLS * col_pitch_c(KA) + 2 * (size_t)KA) * sizeof(double); }

template <typename R, int NM>
__global__ void __launch_bounds__(32 * CWARPS, 4) k_hevi_column(const Grid gt, const StageArgsT<R> a, const BatchT<NM> B)
{
    extern __shared__ double csm[];
    int b;
    const Grid g = block_domain(gt, B, b);
    const int nbx = (g.IMAX + CCOLS - 1) / CCOLS;
    const int i0 = g.IS + (b % nbx) * CCOLS, j = g.JS + b / nbx;
    const int lane = threadIdx.x, w = threadIdx.y;
    const size_t N3 = n3(g);
    const int KS = g.KS, KE = g.KE, KP = col_pitch_c(g.KA);
    const double dt = a.dtrk, J33G = a.J33G, dt2 = dt * dt;
    const Nd<R> nd(a, N3);
    const R *sSr = a.colscr, *sSt = a.colscr + N3, *stZ = a.colscr + 2 * N3, *sPT = a.colscr + 3 * N3;
    // per-level arrays of the tile's columns: [array][column][level], odd pitch;
    // then B(k) and RFDZ(k) by level
    double *sC = csm, *sP = csm + (size_t)CCOLS * KP, *sA = csm + (size_t)2 * CCOLS * KP;
    double *sB = csm + (size_t)3 * CCOLS * KP, *sR = sB + g.KA;
#define CA(arr, cc, L) arr[(size_t)(cc) * KP + (L) - 1]

    // ---- load C, PT and A(k) = dt^2 J33G^2 RCDZ RT2P (:696); B(k) (:697) and RFDZ(k) ----
    for (int cc = w; cc < CCOLS; cc += CWARPS) {
        const int i = i0 + cc;
        if (i > g.IE) break;
        const int col = (int)idx3(g, 1, i, j);
        for (int L = KS + lane; L <= KE; L += 32) {
            const int c = col + L - 1;
            if (L <= KE - 1) {
                CA(sC, cc, L) = __ldcg(a.colC + c);
                CA(sP, cc, L) = (double)__ldcg(sPT + c);
            }
            CA(sA, cc, L) = dt2 * J33G * ld(g.RCDZ + L - 1) * ld(a.RT2P + c) * J33G;
        }
    }
    for (int k = KS + w * 32 + lane; k <= KE - 1; k += 32 * CWARPS) {
        sB[k - 1] = GRAV * dt2 * J33G / (ld(g.CDZ + k) + ld(g.CDZ + k - 1));
        sR[k - 1] = ld(g.RFDZ + k - 1);
    }
    __syncthreads();

    // ---- Thomas solve, one lane per column (F1..F3 of :699-709) ----
    if (w == 0 && lane < CCOLS && i0 + lane <= g.IE) {
        const int cc = lane;
        // F1, F2, F3 and C of level k (F1 is not used at KE-1, F3 not at KS)
        auto coef = [&](int k, double &F1, double &F2, double &F3, double &Ck) {
            const double rfdz = sR[k - 1], Bk = sB[k - 1];
            const double Ak = CA(sA, cc, k), Ak1 = CA(sA, cc, k + 1);
            F2 = 1.0 + (CA(sP, cc, k) * rfdz * (Ak1 + Ak));
            F1 = k <= KE - 2 ? -(CA(sP, cc, k + 1) * rfdz * Ak1 + Bk) : 0.0;
            F3 = k >= KS + 1 ? -(CA(sP, cc, k - 1) * rfdz * Ak - Bk) : 0.0;
            Ck = CA(sC, cc, k);
        };
        double F1, F2, F3, Ck;
        coef(KS, F1, F2, F3, Ck);
        double e_prev, f_prev;
        {
            const double rdenom = 1.0 / F2;
            e_prev = -F1 * rdenom;
            f_prev = Ck * rdenom;
        }
        double nF1, nF2, nF3, nC; // the next level's coefficients
        coef(KS + 1, nF1, nF2, nF3, nC);
        // levels KS+1..KE-2: one straight block per level, in which the next
        // level's coefficients fill the latency of this level's division
        for (int k = KS + 1; k <= KE - 2; ++k) {
            F1 = nF1; F2 = nF2; F3 = nF3; Ck = nC;
            CA(sA, cc, k - 1) = e_prev;
            CA(sC, cc, k - 1) = f_prev;
            coef(k + 1, nF1, nF2, nF3, nC); // reads A(k+1), A(k+2): not yet overwritten
            const double rdenom = 1.0 / (F2 + F3 * e_prev);
            e_prev = -F1 * rdenom;
            f_prev = (Ck - F3 * f_prev) * rdenom;
        }
        CA(sA, cc, KE - 2) = e_prev;
        CA(sC, cc, KE - 2) = f_prev;
        f_prev = (nC - nF3 * f_prev) / (nF2 + nF3 * e_prev); // the solution at KE-1
        CA(sA, cc, KE - 1) = e_prev;
        CA(sC, cc, KE - 1) = f_prev;
        // back substitution, C(k) = e(k) C(k+1) + f(k)
        double Cnext = f_prev;
        for (int k = KE - 2; k >= KS; --k) {
            Cnext = CA(sA, cc, k) * Cnext + CA(sC, cc, k);
            CA(sC, cc, k) = Cnext;
        }
    }
    __syncthreads();

    // ---- back-update (:728-790) ----
    for (int cc = w; cc < CCOLS; cc += CWARPS) {
        const int i = i0 + cc;
        if (i > g.IE) break;
        const int col = (int)idx3(g, 1, i, j);
        for (int m = KS + lane; m <= KE; m += 32) {
            const int c = col + m - 1;
            const double rcdz = ld(g.RCDZ + m - 1);
            double adr, adt;
            if (m == KE) {
                const double Cm1 = CA(sC, cc, m - 1);
                adr = Cm1 * J33G * rcdz;
                adt = Cm1 * CA(sP, cc, KE - 1) * J33G * rcdz;
            } else if (m == KS) {
                const double Cm = CA(sC, cc, m);
                adr = -Cm * J33G * rcdz;
                adt = -Cm * CA(sP, cc, KS) * J33G * rcdz;
            } else {
                const double Cm = CA(sC, cc, m), Cm1 = CA(sC, cc, m - 1);
                adr = -(Cm - Cm1) * J33G * rcdz;
                adt = -(Cm * CA(sP, cc, m) - Cm1 * CA(sP, cc, m - 1)) * J33G * rcdz;
            }
            put_state(a, N3, 0, a.DENS_RK, a.DENS0, c, lds(a.DENS0 + c) + dt * (adr + (double)__ldcg(sSr + c)), true);
            put_state(a, N3, 4, a.RHOT_RK, a.RHOT0, c, lds(a.RHOT0 + c) + dt * (adt + (double)__ldcg(sSt + c)), true);
            if (m <= KE - 1) {
                const double Cm = CA(sC, cc, m);
                put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, ld(a.MOMZ0 + c) + (Cm - ld(a.MOMZ + c)), true);
                put_flux(a, N3, 0, c, R((double)ld(nd.DZ() + c) + J33G * Cm), true);
                put_flux(a, N3, 3, c, R((double)__ldcg(stZ + c) + J33G * Cm * CA(sP, cc, m)), true);
            } else {
                put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, c, 0.0, false);
                put_flux(a, N3, 0, c, R(0.0), true);
                put_flux(a, N3, 3, c, R(0.0), true);
            }
        }
        if (lane == 0) {
            // rigid-lid and surface values (:753-754) and the zero fluxes at KS-1 (:371, ud3.F90:222)
            put_state(a, N3, 1, a.MOMZ_RK, a.MOMZ0, col + KS - 2, 0.0, false);
            put_flux(a, N3, 0, col + KS - 2, R(0.0), false);
            put_flux(a, N3, 3, col + KS - 2, R(0.0), false);
        }
        // hevi_mflx_z :369-393 also fills the halo column i = IS-1 with the explicit
        // part of the vertical mass flux; the solver never updates it
        if (i == g.IS && (a.rk_mode == RK_PLAIN || a.rk_mode == RK_FINAL || a.rk_mode == RK_HEUN3)) {
            const size_t chl = idx3(g, 1, g.IS - 1, j);
            for (int k = KS - 1 + lane; k <= KE; k += 32)
                a.mflx[chl + k - 1] = (k >= KS && k <= KE - 1) ? ld(nd.DZ() + chl + k - 1) : R(0.0);
        }
    }
#undef CA
}

// =============================================================================
// k_numfilter_tiled: the 15 num_diff components (ND_ORDER = 1) of a 4 x 4 tile
// of columns from shared memory
// =============================================================================
// One warp per column, lanes along k, chunks of 32 levels as in
// k_hevi_explicit. Per chunk one thread copies the five filtered quantities
// (phi, written by k_phi) and DENS over the tile, a lateral halo of 2 and the
// levels L0-2..L0+33 into shared memory (six bulk tensor copies completing on
// an mbarrier, bounded wait); numfilter_cell then forms every component from
// there, with the arithmetic of k_numfilter, so the two give identical bits.
// The vertical halo levels of each column follow with global loads.
#ifndef HEVI_ND_TX
#define HEVI_ND_TX 4
#define HEVI_ND_TY 4
#endif
constexpr int NTX = HEVI_ND_TX, NTY = HEVI_ND_TY, NWARPS = NTX * NTY; // tile columns; one warp each
constexpr int NKLO = 2;                        // box levels below the chunk's first
constexpr int NBK = KC + 4;                    // box levels: L0-2 .. L0+33
constexpr int NBW = NTX + 4, NBH = NTY + 4;    // lateral halo of 2
constexpr int NPL = NBK * NBW * NBH;           // one staged field
template <typename R> constexpr size_t nd_smem_bytes() { return (size_t)NPL * (5 * sizeof(R) + sizeof(double)) + 16; }

struct NdMaps {
    CUtensorMap m[6]; // phi q = 0..4 (type R), DENS (FP64), as (KA, IA, JA) tensors
};

// the staged filtered quantities; box element 0 is level k0, column i0, row j0
template <typename R>
struct PhiS {
    using type = R;
    const R *base;
    int k0, i0, j0;
    __device__ R operator()(int q, int k, int i, int j) const
    {
        return base[q * NPL + ((j - j0) * NBW + (i - i0)) * NBK + (k - k0)];
    }
};
// the staged density around a cell
struct DensS {
    const double *p;
    __device__ double operator()(int dk, int di, int dj) const { return p[dk + di * NBK + dj * NBK * NBW]; }
};

template <typename R>
__global__ void __launch_bounds__(32 * NWARPS, 1024 / (32 * NWARPS) > 1 ? 2 : 1)
    k_numfilter_tiled(const Grid g, const NdCoef c, const NdArgsT<R> a, unsigned *status,
                      const __grid_constant__ NdMaps maps)
{
    extern __shared__ __align__(1024) double sm[];
    R *sphi = reinterpret_cast<R *>(sm); // 5 fields, [j][i][k] each
    double *sdn = reinterpret_cast<double *>(reinterpret_cast<char *>(sm) + (size_t)5 * NPL * sizeof(R));
    uint64_t *bar = reinterpret_cast<uint64_t *>(sdn + NPL);
    __shared__ int s_ok;
    const int lane = threadIdx.x, w = threadIdx.y, tid = w * 32 + lane;
    const int tx = w % NTX, ty = w / NTX;
    const int nti = (g.IMAX + NTX - 1) / NTX;
    const int i0 = g.IS + ((int)blockIdx.x % nti) * NTX, j0 = g.JS + ((int)blockIdx.x / nti) * NTY;
    const int i = i0 + tx, j = j0 + ty;
    const bool col_ok = i <= g.IE && j <= g.JE;
    const size_t N3 = n3(g);
    const int KS = g.KS, KE = g.KE;
    const int NC = (g.KMAX + KC - 1) / KC;
    constexpr unsigned BYTES = (unsigned)(NPL * (5 * sizeof(R) + sizeof(double)));

    auto issue = [&](int ch) {
        // box origin (0-based): level L0-2 = 32*ch (KS = 3), column i0-2, row j0-2
        const int x = KC * ch + (KS - 1) - NKLO, y = i0 - 2 - 1, z = j0 - 2 - 1;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(bar, BYTES);
        for (int q = 0; q < 5; ++q) tma_load_3d(sphi + (size_t)q * NPL, &maps.m[q], x, y, z, bar);
        tma_load_3d(sdn, &maps.m[5], x, y, z, bar);
    };
    if (tid == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        issue(0);
    }
    __syncthreads();

    const R ncx = col_ok ? R(ld(c.cdx + i - 1)) : R(0.0), nfx = col_ok ? R(ld(c.fdx + i - 1)) : R(0.0);
    const R ncy = col_ok ? R(ld(c.cdy + j - 1)) : R(0.0), nfy = col_ok ? R(ld(c.fdy + j - 1)) : R(0.0);
    const R sfc = R(c.sfc);
    for (int ch = 0; ch < NC; ++ch) {
        if (tid == 0) {
            const bool ok = mbar_wait(bar, ch & 1);
            // on a timeout, wait once more (bounded) for the copies still in flight
            if (!ok) (void)mbar_wait(bar, ch & 1);
            s_ok = ok ? 1 : 0;
        }
        __syncthreads();
        if (!s_ok) {
            if (tid == 0) atomicOr(status, ST_TMA_TIMEOUT);
            return; // block-uniform
        }
        (void)mbar_try(bar, ch & 1); // completed phase: makes the copied data visible to this thread
        const int L0 = KS + KC * ch, k = L0 + lane;
        if (col_ok && k <= KE) {
            const PhiS<R> phi{sphi, L0 - NKLO, i0 - 2, j0 - 2};
            const DensS dn{sdn + ((ty + 2) * NBW + (tx + 2)) * NBK + (k - (L0 - NKLO))};
            numfilter_cell<false>(g, c, phi, dn, nullptr, a.num_diff, N3, idx3(g, k, i, j), k, i, j, ncx, nfx, ncy,
                                  nfy, sfc);
        }
        __syncthreads(); // every read of the staged box is done
        if (tid == 0 && ch + 1 < NC) issue(ch + 1);
    }
    if (col_ok) numfilter_halo_levels<false>(g, c, Phi<R>{g, a}, nullptr, a.num_diff, N3, a.DENS, i, j, lane);
}

// =============================================================================
// host side
// =============================================================================
template <int S, typename R>
cudaError_t launch_s(const Grid &g, StageArgsT<R> a, int raster, cudaStream_t st)
{
    StateMaps maps;
    const double *f[NF] = {a.DENS, a.MOMZ, a.MOMX, a.MOMY, a.RHOT};
    for (int q = 0; q < NF; ++q)
        if (!encode(&maps.m[q], f[q], g, box_k<S>(), box_w<S>(), box_h<S>())) return cudaErrorNotSupported;
    BatchT<1> B{};
    B.n = 1;
    a.raster = raster > 0 ? raster : STAGE_RASTER_DEFAULT;
    const int ntiles = ((g.IMAX + TX - 1) / TX) * ((g.JMAX + TY - 1) / TY);
    B.first[0] = 0;
    B.first[1] = ntiles;
    auto kx = k_hevi_explicit<S, R, 1>;
    cudaError_t e = open_smem(kx, smem_bytes<S>());
    if (e != cudaSuccess) return e;
    kx<<<ntiles, dim3(32, NCOL), smem_bytes<S>(), st>>>(g, a, B, maps);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    auto kc = k_hevi_column<R, 1>;
    // the attribute is set once per device, so it opens the largest size (KA = 260)
    if ((e = open_smem(kc, column_smem(260))) != cudaSuccess) return e;
    const int ncb = ((g.IMAX + CCOLS - 1) / CCOLS) * g.JMAX;
    B.first[1] = ncb;
    kc<<<ncb, dim3(32, CWARPS), column_smem(g.KA), st>>>(g, a, B);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_numfilter_s(const Grid &g, const NdCoef &c, const NdArgsT<R> &a, unsigned *status, cudaStream_t st)
{
    NdMaps maps;
    for (int q = 0; q < 5; ++q)
        if (!encode(&maps.m[q], a.phi + (size_t)q * n3(g), g, NBK, NBW, NBH)) return cudaErrorNotSupported;
    if (!encode(&maps.m[5], a.DENS, g, NBK, NBW, NBH)) return cudaErrorNotSupported;
    auto k = k_numfilter_tiled<R>;
    cudaError_t e = open_smem(k, nd_smem_bytes<R>());
    if (e != cudaSuccess) return e;
    const int ntiles = ((g.IMAX + NTX - 1) / NTX) * ((g.JMAX + NTY - 1) / NTY);
    k<<<ntiles, dim3(32, NWARPS), nd_smem_bytes<R>(), st>>>(g, c, a, status, maps);
    return cudaGetLastError();
}

}  // namespace tma

// The numerical filter's components from staged tiles where they apply: one
// domain of KHALO = 2 whose filtered quantities and density admit tensor maps
// (16-byte aligned bases and strides). cudaErrorNotSupported otherwise.
template <typename R>
cudaError_t launch_numfilter_tiled(const Grid &g, const Members &mem, const NdCoef &c, const NdArgsT<R> &a,
                                   unsigned *status, cudaStream_t st)
{
    if (mem.n > 1 || g.KS != 3 || c.order != 1 || !status) return cudaErrorNotSupported;
    return tma::launch_numfilter_s<R>(g, c, a, status, st);
}
#ifndef HEVI_FLOAT_TU
template cudaError_t launch_numfilter_tiled<double>(const Grid &, const Members &, const NdCoef &,
                                                    const NdArgsT<double> &, unsigned *, cudaStream_t);
#else
template cudaError_t launch_numfilter_tiled<float>(const Grid &, const Members &, const NdCoef &,
                                                   const NdArgsT<float> &, unsigned *, cudaStream_t);
#endif

// The tiled stage where it applies: one domain, even KA, KA <= MAXKA_TILED,
// the column scratch of the tiled kernels present and every staged field on a
// 16-byte boundary. cudaErrorNotSupported otherwise (the caller then runs the
// fused kernel).
template <typename R>
cudaError_t launch_hevi_stage_tiled(const Grid &g, const Members &mem, const StageArgsT<R> &a, int scheme, int raster,
                                    cudaStream_t st)
{
    // even KA: 16-byte strides for the tensor maps
    if (mem.n > 1 || (g.KA & 1) || g.KA > 260 || !a.colC) return cudaErrorNotSupported;
    switch (scheme) {
    case UD3: return tma::launch_s<UD3, R>(g, a, raster, st);
    case CD4: return tma::launch_s<CD4, R>(g, a, raster, st);
    case KOREN: return tma::launch_s<KOREN, R>(g, a, raster, st);
    case CD2: return tma::launch_s<CD2, R>(g, a, raster, st);
    case UD5: return tma::launch_s<UD5, R>(g, a, raster, st);
    case CD6: return tma::launch_s<CD6, R>(g, a, raster, st);
    default: return cudaErrorInvalidValue;
    }
}
#ifndef HEVI_FLOAT_TU
template cudaError_t launch_hevi_stage_tiled<double>(const Grid &, const Members &, const StageArgsT<double> &, int,
                                                     int, cudaStream_t);
#else
template cudaError_t launch_hevi_stage_tiled<float>(const Grid &, const Members &, const StageArgsT<float> &, int, int,
                                                    cudaStream_t);

#endif

}  // namespace hevi
