// Argument blocks and host launchers of every device kernel of the library.
#pragma once
#include "hevi_stage.cuh"

namespace hevi {

// ---- numerical filter (numfilter.cu) ----
// coefficient tables built on the host (grid_coef.cpp), 0-based storage of
// CNZ3(3,KA,2), CNX3(3,IA,2), CNY3(3,JA,2) and the nd_coef_* vectors
struct NdCoef {
    const double *CNZ3, *CNX3, *CNY3;
    const double *cdz, *fdz, *cdx, *fdx, *cdy, *fdy; // DIFF4 * D**4 (nd_coef_cdz, ...)
    double sfc;                                      // ND_SFC_FACT
};
template <typename R>
struct NdArgsT {
    R *num_diff;
    const double *DENS, *MOMZ, *MOMX, *MOMY, *RHOT, *REF_dens, *REF_pott;
    R *phi; // 5*N3 scratch: the five filtered quantities at every point
};
using NdArgs = NdArgsT<double>;
template <typename R>
cudaError_t launch_numfilter(const Grid &g, const NdCoef &c, const NdArgsT<R> &a, cudaStream_t st);

// ---- tracer advection (tracer.cu) ----
struct TracerArgs {
    double *QTRCo;
    const double *QTRC;   // stage input (high-order flux values)
    const double *QTRC0;  // value at the start of the large step (phi_in of the limiter)
    const double *RHOQ_t;
    const double *DENS0, *DENS;
    int dens_mode;        // density of the stage: 0 DENS, 1 DENS0+(DENS-DENS0)/3, 2 DENS0+(DENS-DENS0)*0.5
    const double *mflx;   // (KA,IA,JA,3)
    const double *ndq;    // (KA,IA,JA,3) or null for ND_COEF_Q = 0
    double dtl;
    double *phi_lo, *anti, *rjp, *rjm; // limiter scratch (anti is 3 fields)
    int along_stream;
};
cudaError_t launch_tracer_stage(const Grid &g, const TracerArgs &a, int scheme, bool fct, cudaStream_t st);

// ---- HEVI stage (hevi_stage.cu) ----
template <typename R>
cudaError_t launch_hevi_stage(const Grid &g, const StageArgsT<R> &a, int scheme, cudaStream_t st);

// ---- utilities (misc.cu) ----
template <typename T>
void periodic_halo(const Grid &g, T *const *fields, int nf, cudaStream_t st);
void divergence(const Grid &g, double *DDIV, const double *MOMZ, const double *MOMX, const double *MOMY,
                const double *RCDZ, const double *RCDX, const double *RCDY, double J33G, cudaStream_t st);
void vertical_bc(const Grid &g, double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT, cudaStream_t st);
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
void mflx_accumulate(const Grid &g, double *av, const double *mflx, cudaStream_t st);
void mflx_average(const Grid &g, double *mflx, const double *av, int nstep, cudaStream_t st);

// message returned by scale_hevi_last_error() (capi.cu)
void set_last_error(const char *msg);

}  // namespace hevi
