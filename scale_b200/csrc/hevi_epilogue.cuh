// Epilogue and per-cell helpers shared by the HEVI stage kernels: the RK4/RK3
// folds of the stage outputs (put_state, put_flux), the cache-streaming loads
// and stores of single-use data, and the num_diff component table.
#pragma once
#include "hevi_stage.cuh"

#ifndef HEVI_STREAM_HINTS
#define HEVI_STREAM_HINTS 1 // evict-first loads/stores for data each cell touches once
#endif

namespace hevi {

__device__ __forceinline__ void flag_nonfinite(unsigned *status, double v)
{
    if (!isfinite(v)) atomicOr(status, ST_NONFINITE);
}

// Data a cell reads or writes once (tendencies, stage-0 state, outputs, RK sums)
// go through the cache-streaming path, so that L2 keeps the fields whose x/y
// neighbours other tiles read again.
#if HEVI_STREAM_HINTS
template <typename T> __device__ __forceinline__ T lds(const T *p) { return __ldcs(p); }
template <typename T> __device__ __forceinline__ void sts(T *p, T v) { __stcs(p, v); }
#else
template <typename T> __device__ __forceinline__ T lds(const T *p) { return __ldg(p); }
template <typename T> __device__ __forceinline__ void sts(T *p, T v) { *p = v; }
#endif

// store one prognostic value of the stage, folding in the RK4 or RK3 combine
template <typename F>
__device__ __forceinline__ void put_state(const StageArgsT<F> &a, size_t N3, int v, double *out, const double *x0,
                                          size_t c, double val, bool combine)
{
    double *acc = a.acc + (size_t)v * N3 + c;
    switch (a.rk_mode) {
    case RK_PLAIN: sts(out + c, val); flag_nonfinite(a.status, val); break;
    case RK_STAGE1: sts(out + c, val); if (combine) sts(acc, val * 2.0); break;
    case RK_STAGE2: sts(out + c, val); if (combine) sts(acc, lds(acc) + val * 4.0); break;
    case RK_STAGE3: sts(out + c, val); if (combine) sts(acc, lds(acc) + val * 2.0); break;
    case RK_HEUN1: sts(out + c, val); break;
    case RK_HEUN3: {
        double r = combine ? ((lds(acc) * 3.0 + val * 3.0) - lds(x0 + c) * 2.0) / 4.0 : val;
        sts(out + c, r);
        flag_nonfinite(a.status, r);
        break;
    }
    default: {
        double r = combine ? ((lds(acc) + val) - lds(x0 + c) * 3.0) / 6.0 : val;
        sts(out + c, r);
        flag_nonfinite(a.status, r);
    }
    }
}

// store one flux value (f: 0..2 mflx Z,X,Y; 3..5 tflx Z,X,Y); 'interior' marks the
// cells the RK4 and RK3 combines average (k in KS:KE, i in IS:IE, j in JS:JE)
template <typename F>
__device__ __forceinline__ void put_flux(const StageArgsT<F> &a, size_t N3, int f, size_t c, F val, bool interior)
{
    F *out = (f < 3 ? a.mflx : a.tflx) + (size_t)(f % 3) * N3 + c;
    F *acc = a.facc + (size_t)f * N3 + c;
    switch (a.rk_mode) {
    case RK_PLAIN: sts(out, val); break;
    case RK_STAGE1: if (interior) sts(acc, val); break;
    case RK_STAGE2:
    case RK_STAGE3: if (interior) sts(acc, lds(acc) + val * F(2.0)); break;
    case RK_HEUN1: if (interior) sts(acc, val); break;
    case RK_HEUN3: sts(out, interior ? (lds(acc) + val * F(3.0)) / F(4.0) : val); break;
    default: sts(out, interior ? (lds(acc) + val) / F(6.0) : val);
    }
}

// =============================================================================
// per-cell pieces shared by the phases (c = offset of cell (k,i,j))
// =============================================================================
// num_diff components by (quantity, direction), computed at each use from the
// kernel parameters so that no register holds fifteen pointers
template <typename F>
struct Nd {
    const F *base;
    size_t N3;
    __device__ Nd(const StageArgsT<F> &a, size_t n) : base(a.num_diff), N3(n) {}
    __device__ const F *q(int v, int dir) const { return base + N3 * (size_t)((v - 1) + 5 * (dir - 1)); }
    __device__ const F *DZ() const { return q(1, 1); }
    __device__ const F *DX() const { return q(1, 2); }
    __device__ const F *DY() const { return q(1, 3); }
    __device__ const F *WZ() const { return q(2, 1); }
    __device__ const F *WX() const { return q(2, 2); }
    __device__ const F *WY() const { return q(2, 3); }
    __device__ const F *UZ() const { return q(3, 1); }
    __device__ const F *UX() const { return q(3, 2); }
    __device__ const F *UY() const { return q(3, 3); }
    __device__ const F *VZ() const { return q(4, 1); }
    __device__ const F *VX() const { return q(4, 2); }
    __device__ const F *VY() const { return q(4, 3); }
    __device__ const F *TZ() const { return q(5, 1); }
    __device__ const F *TX() const { return q(5, 2); }
    __device__ const F *TY() const { return q(5, 3); }
};

}  // namespace hevi
