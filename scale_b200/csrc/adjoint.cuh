// Tangent-linear and adjoint of the HEVI short step (adjoint.cu).
#pragma once
#include "hevi_kernels.cuh"

namespace hevi {
namespace ad {

// The differentiated model: one short step (numerical filter, RK4 of four
// HEVI stages, vertical boundary values, periodic halo) of a single flat-
// terrain domain with the large-step quantities (DPRES0, RT2P, REF_*) held
// fixed and zero tendencies. Device pointers except the tables in g / nd.
struct Model {
    Grid g;
    NdCoef nd;
    double dt, J33G;
    const double *wdamp; // device (KA)
    unsigned *status;
    const double *DPRES0, *RT2P, *REF_rhot, *REF_dens, *REF_pott, *PHI, *CORIOLI;
    const double *zero;   // N3 zeros (the tendencies)
    double *scratch;      // scratch_fields() * N3
    int scheme;
    cudaStream_t stream;
};

size_t scratch_fields();
// one step through the pass form (X: DENS, MOMZ, MOMX, MOMY, RHOT, 5*N3)
cudaError_t step_forward(const Model &M, double *X);
// X and its tangent dX advanced one step
cudaError_t step_tlm(const Model &M, double *X, double *dX);
// one short step in double-double arithmetic: X_hi + X_lo in and out
cudaError_t step_dd(const Model &M, double *X_hi, double *X_lo);
// lam (adjoint of the state after the step) replaced by the adjoint of the
// state X at the step's start
cudaError_t step_adjoint(const Model &M, const double *X, double *lam);
// adjoint of the vertical boundary values and the periodic halo
cudaError_t boundary_adjoint(const Model &M, double *lam);

}  // namespace ad
}  // namespace hevi
