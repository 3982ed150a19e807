// Device bodies of the lateral and vertical halo fills (halo_column,
// vbc_column). They take their block and thread indices as arguments, so that
// the fill kernels of misc.cu and the persistent short-step kernel run the
// same code.
#pragma once
#include "hevi_kernels.cuh"

namespace hevi {

// ---- periodic halo fill: COMM_vars8 + COMM_wait on a single periodic rank ----
// (scalelib/src/communication/scale_comm_cartesC.F90:345-397, 1600-2043). Every
// halo column takes all KA levels of its periodic image; corners included. A
// block of the launch is FILL_WARPS warps, one halo column each.
constexpr int FILL_WARPS = 4;
template <typename T>
struct FieldList {
    T *f[16];
};

// halo column of field v: block x of the launch over all members, warp wy
template <typename T, int NM>
__device__ __forceinline__ void halo_column(const Grid &gt, T *v, const BatchT<NM> &B, int x, int wy, int lane)
{
    int b;
    const Grid g = block_domain(gt, B, b, x);
    const int nA = 2 * g.JHALO * g.IA;      // halo rows j < JS and j > JE, all i
    const int nB = 2 * g.IHALO * g.JMAX;    // halo columns i < IS and i > IE, interior j
    const int h = b * FILL_WARPS + wy;
    if (h >= nA + nB) return;
    int i, j;
    if (h < nA) {
        const int r = h / g.IA;
        i = 1 + h % g.IA;
        j = r < g.JHALO ? 1 + r : g.JE + 1 + (r - g.JHALO);
    } else {
        const int q = h - nA;
        const int r = q / g.JMAX;
        j = g.JS + q % g.JMAX;
        i = r < g.IHALO ? 1 + r : g.IE + 1 + (r - g.IHALO);
    }
    const int si = i < g.IS ? i + g.IMAX : (i > g.IE ? i - g.IMAX : i);
    const int sj = j < g.JS ? j + g.JMAX : (j > g.JE ? j - g.JMAX : j);
    const size_t dst = idx3(g, 1, i, j), src = idx3(g, 1, si, sj);
    for (int k = lane; k < g.KA; k += 32) v[dst + k] = v[src + k];
}
// blocks of the halo fill of one field in one domain
__host__ __device__ inline int halo_blocks(const Grid &m)
{
    return (2 * m.JHALO * m.IA + 2 * m.IHALO * m.JMAX + FILL_WARPS - 1) / FILL_WARPS;
}

// ---- vertical boundary values after a short step (scale_atmos_dyn_tstep_large_fvm_heve.F90:910-926) ----
// column i of the block's FILL_WARPS columns of row j, one lane per halo level
template <int NM>
__device__ __forceinline__ void vbc_column(const Grid &gt, double *DENS, double *MOMZ, double *MOMX, double *MOMY,
                                           double *RHOT, const BatchT<NM> &B, int x, int wy, int lane)
{
    int b;
    const Grid g = block_domain(gt, B, b, x);
    const Block2 p = split_block(b, (g.IMAX + FILL_WARPS - 1) / FILL_WARPS);
    const int i = g.IS + p.x * FILL_WARPS + wy;
    const int j = g.JS + p.y;
    if (i > g.IE) return;
    const size_t c = idx3(g, 1, i, j);
    const int k = 1 + lane;
    if (k <= g.KS - 1) {
        const size_t s = c + g.KS - 1, d = c + k - 1;
        DENS[d] = DENS[s]; MOMZ[d] = 0.0; MOMX[d] = MOMX[s]; MOMY[d] = MOMY[s]; RHOT[d] = RHOT[s];
    } else if (k <= g.KS - 1 + (g.KA - g.KE)) {
        const int kk = g.KE + (k - (g.KS - 1));
        const size_t s = c + g.KE - 1, d = c + kk - 1;
        DENS[d] = DENS[s]; MOMZ[d] = 0.0; MOMX[d] = MOMX[s]; MOMY[d] = MOMY[s]; RHOT[d] = RHOT[s];
    }
}
__host__ __device__ inline int vbc_blocks(const Grid &m) { return ((m.IMAX + FILL_WARPS - 1) / FILL_WARPS) * m.JMAX; }

}  // namespace hevi
