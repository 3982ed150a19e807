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
#include "numfilter_body.cuh"

namespace hevi {

#ifndef HEVI_ND_MINB
#define HEVI_ND_MINB 8 // minimum resident blocks per SM asked of the register allocator
#endif

template <typename R, int NM>
__global__ void __launch_bounds__(PHI_THREADS) k_phi(const Grid gt, const NdArgsT<R> a, const BatchT<NM> B)
{
    phi_point(gt, a, B, (int)blockIdx.x, (int)threadIdx.x);
}

template <typename R, int NM, bool FW = false>
__global__ void __launch_bounds__(32 * ND_WARPS, HEVI_ND_MINB)
    k_numfilter(const Grid gt, const NdCoef ct, const NdArgsT<R> a, const BatchT<NM> B, const double *W = nullptr)
{
    numfilter_column<R, NM, FW>(gt, ct, a, B, W, (int)blockIdx.x, (int)threadIdx.y, (int)threadIdx.x);
}

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
                                  cudaStream_t st, const HaloFill *fill)
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
        if (fill) { // COMM_vars8 of the work (:1557-1563)
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
            if (fill->fn(fill->ctx, reinterpret_cast<void *const *>(f), 15, (int)sizeof(double))) return cudaErrorUnknown;
        } else {
            periodic_halo(g, Members{}, f, 15, st);
        }
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
cudaError_t launch_numfilter(const Grid &g, const Members &mem, const NdCoef &c, const NdArgsT<R> &a, cudaStream_t st,
                             unsigned *status)
{
    auto nb_phi = [](const Grid &m) { return (int)(((long)m.KA * m.IA * m.JA + PHI_THREADS - 1) / PHI_THREADS); };
    auto nb_nd = [](const Grid &m) { return ((m.IMAX + 3) / 4) * m.JMAX; };
    with_batch(g, mem, nb_phi, [&](const auto &B, int nb) {
        k_phi<R, std::decay_t<decltype(B)>::NMAX><<<nb, PHI_THREADS, 0, st>>>(g, a, B);
        return cudaSuccess;
    });
    if (status) {
        // one domain: the components from staged tiles where the tensor maps apply
        const cudaError_t e = launch_numfilter_tiled(g, mem, c, a, status, st);
        if (e != cudaErrorNotSupported) return e;
    }
    with_batch(g, mem, nb_nd, [&](const auto &B, int nb) {
        k_numfilter<R, std::decay_t<decltype(B)>::NMAX><<<nb, dim3(32, 4), 0, st>>>(g, c, a, B, nullptr);
        return cudaSuccess;
    });
    return cudaGetLastError();
}
#ifdef HEVI_FLOAT_TU
template cudaError_t launch_numfilter<float>(const Grid &, const Members &, const NdCoef &, const NdArgsT<float> &,
                                             cudaStream_t, unsigned *);
#else
template cudaError_t launch_numfilter<double>(const Grid &, const Members &, const NdCoef &, const NdArgsT<double> &,
                                              cudaStream_t, unsigned *);
#endif

}  // namespace hevi
