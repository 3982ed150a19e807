// Argument block of one HEVI short-step stage on the device.
#pragma once
#include "hevi_common.cuh"

namespace hevi {

// RK4 accumulation performed in the stage epilogue. The four stages of
// ATMOS_DYN_tinteg_short_rk4 (scale_atmos_dyn_tinteg_short_rk4.F90:376-560)
// write their outputs to RK buffers and the combine (:562-650) forms
//   X  = (RK1*2 + RK2*4 + RK3*2 + X4 - X0*3) / 6      (state, interior)
//   F  = (F1 + F2*2 + F3*2 + F4) / 6                    (mflx_hi/tflx_hi, interior)
// Accumulating the same sums left to right in the stage epilogues gives the
// identical IEEE results without storing RK1..RK3 fluxes or a combine pass.
enum RkMode : int {
    RK_PLAIN = 0,  // one ATMOS_DYN_Tstep_short call: outputs only
    RK_STAGE1 = 1, // acc = X*2, facc = F
    RK_STAGE2 = 2, // acc += X*4, facc += F*2
    RK_STAGE3 = 3, // acc += X*2, facc += F*2
    RK_FINAL = 4,  // X = ((acc + X) - X0*3)/6, F = (facc + F)/6 over the interior
    // Heun's RK3 (scale_atmos_dyn_tinteg_short_rk3.F90:188-576): stage 1 writes
    // RK1 to its buffer and F1 to facc; stage 2 is RK_PLAIN; stage 3 forms
    //   X = ((RK1*3 + X3*3) - X0*2)/4, F = (F1 + F3*3)/4 over the interior
    // with acc pointing at the stage-1 buffer.
    RK_HEUN1 = 5,
    RK_HEUN3 = 6,
};

// Per-level sources Sr, St and the vertical theta flux tZ of the implicit
// column problem: in shared memory (0) or in a global scratch of 3 fields (1).
#ifndef HEVI_COL_SCRATCH
#define HEVI_COL_SCRATCH 1
#endif

// F is the storage and arithmetic type of the flux-like arrays (num_diff, the
// tendencies, DDIV, the fluxes and their RK sums, the column-solve sources):
// double on the plain path, float on the mixed-precision path. The state, the
// base state and the pressure deviation are always double.
template <typename F>
struct StageArgsT {
    // outputs (RK_FINAL: the state arrays themselves, updated in place)
    double *DENS_RK, *MOMZ_RK, *MOMX_RK, *MOMY_RK, *RHOT_RK;
    F *mflx; // mflx_hi(KA,IA,JA,3): Z, X, Y
    F *tflx; // tflx_hi(KA,IA,JA,3)
    // inputs
    const double *DENS0, *MOMZ0, *MOMX0, *MOMY0, *RHOT0;
    const double *DENS, *MOMZ, *MOMX, *MOMY, *RHOT;
    const F *DENS_t, *MOMZ_t, *MOMX_t, *MOMY_t, *RHOT_t;
    const double *DPRES0, *RT2P, *CORIOLI;
    const F *num_diff;   // (KA,IA,JA,5,3)
    const double *wdamp; // (KA)
    const F *DDIV;
    const double *REF_dens, *REF_rhot;
    double divdmp_coef, J33G, dtrk;
    // RK accumulation
    int rk_mode;
    double *acc; // 5*N3: DENS, MOMZ, MOMX, MOMY, RHOT
    F *facc;     // 6*N3: mflx Z,X,Y then tflx Z,X,Y
    unsigned *status;
    F *colscr; // Sr, St, tZ (3*N3, the fused kernel) and PT (4*N3, the tiled kernels)
    double *colC; // 2*N3: right-hand side C of the column problem, then f; e (tiled kernels; null: fused only)
    int raster; // rows of tiles per raster group (set by the launcher)
};
using StageArgs = StageArgsT<double>;

}  // namespace hevi
