// Tangent-linear and adjoint of the HEVI short step (numerical filter, RK4 of
// four HEVI stages, boundary values and periodic halo), flat terrain, a single
// domain, no divergence damping.
//
// The short step is restated here as a sequence of passes over the grid that
// follows the reference's own sequence of array passes
// (ATMOS_DYN_Tstep_short_fvm_hevi, scale_atmos_dyn_tstep_short_fvm_hevi.F90:343-1048:
// hevi_pres, hevi_mflx_z/x/y, hevi_sr, the w-momentum fluxes and hevi_sw, POTT,
// the theta fluxes and hevi_st, hevi_solver with solve_direct, hevi_momx,
// hevi_momy; ATMOS_DYN_numfilter_coef, scale_atmos_dyn_common.F90:385-985;
// ATMOS_DYN_tinteg_short_rk4, scale_atmos_dyn_tinteg_short_rk4.F90:199-650).
// Every pass but the column solve computes each output cell from a small
// stencil of inputs, and is written once, generically, against an accessor IO:
//   FwdIO  doubles: the forward values (the same operations in the same order
//          as the fused stage kernel, so the trajectory is the same);
//   TlmIO  dual numbers: the tangent-linear model, value and tangent together;
//   AdjIO  jets: the pass is evaluated with one derivative slot per input it
//          loads, which gives the partial derivatives of the output cell; the
//          output's adjoint times each partial is then added to the adjoint of
//          that input (the transposed stencil, with atomic adds since several
//          outputs share an input).
// The column pass (the implicit vertical problem) has a generic forward
// (FwdIO, TlmIO) and a hand-written adjoint: the transposed tridiagonal solve
// for the right-hand side, the adjoint of the matrix entries (-y_r C_c), and
// the chain back through the face potential temperature, the buoyancy and the
// vertical pressure gradient.
//
// The adjoint is of the discrete model as computed: the UD3 upwind switch
// sign(flux) is piecewise constant, so its derivative is taken as zero.
#include <cstdio>

#include "hevi_kernels.cuh"
#include "adjoint.cuh"

namespace hevi {
namespace ad {

// ---- scalar types --------------------------------------------------------------
struct Dual {
    double v, t;
    __device__ Dual() : v(0.0), t(0.0) {}
    __device__ Dual(double x) : v(x), t(0.0) {}
    __device__ Dual(double x, double dx) : v(x), t(dx) {}
    friend __device__ Dual operator+(const Dual &a, const Dual &b) { return {a.v + b.v, a.t + b.t}; }
    friend __device__ Dual operator-(const Dual &a, const Dual &b) { return {a.v - b.v, a.t - b.t}; }
    friend __device__ Dual operator*(const Dual &a, const Dual &b) { return {a.v * b.v, a.t * b.v + a.v * b.t}; }
    friend __device__ Dual operator/(const Dual &a, const Dual &b)
    {
        const double q = a.v / b.v;
        return {q, (a.t - q * b.t) / b.v};
    }
    friend __device__ Dual operator-(const Dual &a) { return {-a.v, -a.t}; }
    friend __device__ Dual operator+(const Dual &a) { return a; }
    friend __device__ double vof(const Dual &a) { return a.v; }
    friend __device__ Dual fabs(const Dual &a) { return {::fabs(a.v), signbit(a.v) ? -a.t : a.t}; }
    friend __device__ Dual copysign(const Dual &a, const Dual &b)
    {
        return {::copysign(a.v, b.v), signbit(a.v) != signbit(b.v) ? -a.t : a.t};
    }
};

template <int N>
struct Jet {
    double v;
    double d[N];
    __device__ Jet() : v(0.0)
    {
#pragma unroll
        for (int q = 0; q < N; ++q) d[q] = 0.0;
    }
    __device__ Jet(double x) : v(x)
    {
#pragma unroll
        for (int q = 0; q < N; ++q) d[q] = 0.0;
    }
    friend __device__ Jet operator+(const Jet &a, const Jet &b)
    {
        Jet r(a.v + b.v);
#pragma unroll
        for (int q = 0; q < N; ++q) r.d[q] = a.d[q] + b.d[q];
        return r;
    }
    friend __device__ Jet operator-(const Jet &a, const Jet &b)
    {
        Jet r(a.v - b.v);
#pragma unroll
        for (int q = 0; q < N; ++q) r.d[q] = a.d[q] - b.d[q];
        return r;
    }
    friend __device__ Jet operator*(const Jet &a, const Jet &b)
    {
        Jet r(a.v * b.v);
#pragma unroll
        for (int q = 0; q < N; ++q) r.d[q] = a.d[q] * b.v + a.v * b.d[q];
        return r;
    }
    friend __device__ Jet operator/(const Jet &a, const Jet &b)
    {
        Jet r(a.v / b.v);
#pragma unroll
        for (int q = 0; q < N; ++q) r.d[q] = (a.d[q] - r.v * b.d[q]) / b.v;
        return r;
    }
    friend __device__ Jet operator-(const Jet &a)
    {
        Jet r(-a.v);
#pragma unroll
        for (int q = 0; q < N; ++q) r.d[q] = -a.d[q];
        return r;
    }
    friend __device__ Jet operator+(const Jet &a) { return a; }
    friend __device__ double vof(const Jet &a) { return a.v; }
    friend __device__ Jet fabs(const Jet &a)
    {
        Jet r = signbit(a.v) ? -a : a;
        r.v = ::fabs(a.v);
        return r;
    }
    friend __device__ Jet copysign(const Jet &a, const Jet &b)
    {
        Jet r = (signbit(a.v) != signbit(b.v)) ? -a : a;
        r.v = ::copysign(a.v, b.v);
        return r;
    }
};

// Double-double numbers (an unevaluated sum hi + lo, about 106 significant
// bits) for a forward model whose rounding lies far below the differences that
// a finite-difference check of the adjoint takes. The error-free transforms
// are Knuth's two-sum, the fast two-sum for |a| >= |b| and the product error
// through a fused multiply-add; sums, products and quotients renormalise their
// results. The unit is compiled without FMA contraction, so every expression
// here is evaluated as written.
struct DD {
    double hi, lo;
    __device__ DD() : hi(0.0), lo(0.0) {}
    __device__ DD(double x) : hi(x), lo(0.0) {}
    __device__ DD(double h, double l) : hi(h), lo(l) {}
};
__device__ __forceinline__ DD dd_two_sum(double a, double b)
{
    const double s = a + b, v = s - a;
    return {s, (a - (s - v)) + (b - v)};
}
__device__ __forceinline__ DD dd_fast_sum(double a, double b) // |a| >= |b| or a == 0
{
    const double s = a + b;
    return {s, b - (s - a)};
}
__device__ __forceinline__ DD dd_two_prod(double a, double b)
{
    const double p = a * b;
    return {p, fma(a, b, -p)};
}
__device__ __forceinline__ DD operator+(const DD &a, const DD &b)
{
    DD s = dd_two_sum(a.hi, b.hi);
    const DD t = dd_two_sum(a.lo, b.lo);
    s = dd_fast_sum(s.hi, s.lo + t.hi);
    return dd_fast_sum(s.hi, s.lo + t.lo);
}
__device__ __forceinline__ DD operator-(const DD &a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ DD operator+(const DD &a) { return a; }
__device__ __forceinline__ DD operator-(const DD &a, const DD &b) { return a + (-b); }
__device__ __forceinline__ DD operator*(const DD &a, const DD &b)
{
    const DD p = dd_two_prod(a.hi, b.hi);
    return dd_fast_sum(p.hi, p.lo + (a.hi * b.lo + a.lo * b.hi));
}
__device__ __forceinline__ DD operator/(const DD &a, const DD &b)
{
    // three quotient digits, each from the remainder of the previous ones
    const double q1 = a.hi / b.hi;
    DD r = a - b * DD(q1);
    const double q2 = r.hi / b.hi;
    r = r - b * DD(q2);
    const double q3 = r.hi / b.hi;
    return dd_fast_sum(q1, q2) + DD(q3);
}
__device__ __forceinline__ double vof(const DD &a) { return a.hi; }
__device__ __forceinline__ DD fabs(const DD &a) { return signbit(a.hi) ? -a : a; }
__device__ __forceinline__ DD copysign(const DD &a, const DD &b) { return signbit(a.hi) != signbit(b.hi) ? -a : a; }

// ---- field table ---------------------------------------------------------------------
// Every array a pass touches is a field of the table; val[f] holds its values,
// aux[f] its tangent (TlmIO) or adjoint (AdjIO), null for constants.
enum Field : int {
    X0D = 0, X0W, X0U, X0V, X0R,       // stage start state (DENS0..RHOT0)
    XD = 5, XW, XU, XV, XR,            // stage evaluation state (DENS..RHOT)
    TD = 10, TW, TU, TV, TR,           // tendencies (constants)
    ND0 = 15,                          // num_diff(v,dir) at ND0 + (v-1) + 5*(dir-1)
    DPRES0 = 30, RT2P, REFRHOT, REFDENS, REFPOTT, GEOP, CORI,   // constants
    DPRES = 37, MZ, MX, MY, SR, QWZ, QWX, QWY, SW, POTT, TZ, TX, TY, ST, QUZ, QUX, QUY, QVZ, QVX, QVY,
    ODRK = 57, OWRK, OURK, OVRK, ORRK, // stage outputs
    PH0 = 62,                          // the five filtered quantities of the numerical filter
    PTf = 67, F1f, F2f, F3f, Cf, Ef, Ff, // column work: face theta, matrix, solution, elimination
    NFLD = 74
};
__host__ __device__ constexpr int NDF(int v, int dir) { return ND0 + (v - 1) + 5 * (dir - 1); }
constexpr int N_INTER_FIRST = DPRES, N_INTER = QVY - DPRES + 1;

struct Ctx {
    Grid g;
    NdCoef nd;
    double dt, J33G;
    const double *wdamp;
    unsigned *status;
    double *val[NFLD];
    double *aux[NFLD];
};

enum : unsigned { ST_JET_OVERFLOW = 1u << 4 };

struct FwdIO {
    using T = double;
    const Ctx &x;
    __device__ FwdIO(const Ctx &c) : x(c) {}
    __device__ double in(int f, size_t c) { return x.val[f][c]; }
    __device__ double cst(int f, size_t c) { return x.val[f][c]; }
    __device__ void out(int f, size_t c, double v) { x.val[f][c] = v; }
};
struct TlmIO {
    using T = Dual;
    const Ctx &x;
    __device__ TlmIO(const Ctx &c) : x(c) {}
    __device__ Dual in(int f, size_t c) { return Dual(x.val[f][c], x.aux[f][c]); }
    __device__ Dual cst(int f, size_t c) { return Dual(x.val[f][c]); }
    __device__ void out(int f, size_t c, const Dual &v)
    {
        x.val[f][c] = v.v;
        x.aux[f][c] = v.t;
    }
};
// double-double values: hi in val, lo in aux
struct DdIO {
    using T = DD;
    const Ctx &x;
    __device__ DdIO(const Ctx &c) : x(c) {}
    __device__ DD in(int f, size_t c) { return DD(x.val[f][c], x.aux[f][c]); }
    __device__ DD cst(int f, size_t c) { return DD(x.val[f][c]); }
    __device__ void out(int f, size_t c, const DD &v)
    {
        x.val[f][c] = v.hi;
        x.aux[f][c] = v.lo;
    }
};
template <int N>
struct AdjIO {
    using T = Jet<N>;
    const Ctx &x;
    int n = 0;
    int fid[N];
    size_t off[N];
    __device__ AdjIO(const Ctx &c) : x(c) {}
    // The slots are indexed by compile-time constants only (an unrolled loop
    // with a select), so the jets and the slot table stay in registers rather
    // than in local memory.
    __device__ Jet<N> in(int f, size_t c)
    {
        Jet<N> r(x.val[f][c]);
        if (n < N) {
#pragma unroll
            for (int q = 0; q < N; ++q) {
                if (q == n) {
                    r.d[q] = 1.0;
                    fid[q] = f;
                    off[q] = c;
                }
            }
            ++n;
        } else {
            atomicOr(x.status, ST_JET_OVERFLOW);
        }
        return r;
    }
    __device__ Jet<N> cst(int f, size_t c) { return Jet<N>(x.val[f][c]); }
    __device__ void out(int f, size_t c, const Jet<N> &v)
    {
        const double l = x.aux[f][c];
        if (l == 0.0) return;
#pragma unroll
        for (int q = 0; q < N; ++q)
            if (q < n && v.d[q] != 0.0) atomicAdd(x.aux[fid[q]] + off[q], l * v.d[q]);
    }
};

// ---- launch boxes --------------------------------------------------------------------------
struct Box {
    int k0, k1, i0, i1, j0, j1;
    __host__ __device__ long long count() const
    {
        return (long long)(k1 - k0 + 1) * (i1 - i0 + 1) * (j1 - j0 + 1);
    }
};

template <class P, class IOT>
__global__ void __launch_bounds__(128) k_pass(const __grid_constant__ Ctx x, const Box b)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= b.count()) return;
    const int nk = b.k1 - b.k0 + 1, ni = b.i1 - b.i0 + 1;
    const int k = b.k0 + (int)(t % nk);
    t /= nk;
    const int i = b.i0 + (int)(t % ni);
    const int j = b.j0 + (int)(t / ni);
    IOT io(x);
    P{}(io, x, k, i, j);
}

#define PASS_BEGIN                                                          \
    using T = typename IO::T;                                               \
    const Grid &g = x.g;                                                    \
    const size_t c = idx3(g, k, i, j);                                      \
    const size_t sI = (size_t)g.KA, sJ = (size_t)g.KA * g.IA;               \
    const int KS = g.KS, KE = g.KE;                                         \
    (void)sI; (void)sJ; (void)KS; (void)KE;
#define IN(f, o) io.in(f, (o))
#define CS(f, o) io.cst(f, (o))
#define TB(p, n) T(ld((p) + (n)))

// ============================================================================
// numerical filter (numfilter.cu restated per output component)
// ============================================================================
// the five filtered quantities at every point (k_phi)
struct PassPhi {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        // every input is loaded unconditionally and in one order (the neighbour
        // of the last point of the array in a direction is replaced by the point
        // itself, whose value is then unused), so each keeps one derivative slot
        const T D = IN(XD, c);
        const T W = IN(XW, c), Dk = IN(XD, k < g.KA ? c + 1 : c);
        const T U = IN(XU, c), Di = IN(XD, i < g.IA ? c + sI : c);
        const T V = IN(XV, c), Dj = IN(XD, j < g.JA ? c + sJ : c);
        const T RT = IN(XR, c);
        io.out(PH0 + 0, c, D - CS(REFDENS, c));
        io.out(PH0 + 1, c, k < g.KA ? T(2.0) * W / (Dk + D) : T(0.0));
        io.out(PH0 + 2, c, i < g.IA ? T(2.0) * U / (Di + D) : T(0.0));
        io.out(PH0 + 3, c, j < g.JA ? T(2.0) * V / (Dj + D) : T(0.0));
        io.out(PH0 + 4, c, RT / D - CS(REFPOTT, c));
    }
};

#define CZ3(n, kk, s) TB(x.nd.CNZ3, ((n) - 1) + 3 * ((size_t)((kk) - 1) + (size_t)g.KA * ((s) - 1)))
#define CX3(n, ii, s) TB(x.nd.CNX3, ((n) - 1) + 3 * ((size_t)((ii) - 1) + (size_t)g.IA * ((s) - 1)))
#define CY3(n, jj, s) TB(x.nd.CNY3, ((n) - 1) + 3 * ((size_t)((jj) - 1) + (size_t)g.JA * ((s) - 1)))
#define PHI(q, kk, ii, jj) IN(PH0 + (q), idx3(g, kk, ii, jj))

template <class IO>
__device__ typename IO::T nd_dz0(IO &io, const Ctx &x, int q, int k, int i, int j)
{
    using T = typename IO::T;
    const Grid &g = x.g;
    const int KS = g.KS, KE = g.KE;
    auto inner = [&](int m) {
        return (+CZ3(1, m + 1, 1) * PHI(q, m + 2, i, j) - CZ3(2, m + 1, 1) * PHI(q, m + 1, i, j)
                + CZ3(3, m + 1, 1) * PHI(q, m, i, j) - CZ3(1, m, 1) * PHI(q, m - 1, i, j));
    };
    auto atKS = [&]() {
        return (+CZ3(1, KS + 1, 1) * PHI(q, KS + 2, i, j) - CZ3(2, KS + 1, 1) * PHI(q, KS + 1, i, j)
                + CZ3(3, KS + 1, 1) * PHI(q, KS, i, j) - CZ3(1, KS, 1) * PHI(q, KS + 1, i, j));
    };
    auto atKEm1 = [&]() {
        return (+CZ3(1, KE, 1) * PHI(q, KE - 1, i, j) - CZ3(2, KE, 1) * PHI(q, KE, i, j)
                + CZ3(3, KE, 1) * PHI(q, KE - 1, i, j) - CZ3(1, KE - 1, 1) * PHI(q, KE - 2, i, j));
    };
    if (k >= KS + 1 && k <= KE - 2) return inner(k);
    if (k == KS) return atKS();
    if (k == KS - 1) return -atKS();
    if (k == KS - 2) return -inner(KS + 1);
    if (k == KE - 1) return atKEm1();
    if (k == KE) return -atKEm1();
    if (k == KE + 1) return -inner(KE - 2);
    return T(0.0);
}

template <class IO>
__device__ typename IO::T nd_dz1(IO &io, const Ctx &x, int q, int k, int i, int j)
{
    const Grid &g = x.g;
    const int KS = g.KS, KE = g.KE;
    using T = typename IO::T;
    auto inner = [&](int m) {
        return (+CZ3(1, m, 2) * PHI(q, m + 1, i, j) - CZ3(2, m, 2) * PHI(q, m, i, j)
                + CZ3(3, m, 2) * PHI(q, m - 1, i, j) - CZ3(1, m - 1, 2) * PHI(q, m - 2, i, j));
    };
    auto atKSp1 = [&]() {
        return (+CZ3(1, KS + 1, 2) * PHI(q, KS + 2, i, j) - CZ3(2, KS + 1, 2) * PHI(q, KS + 1, i, j)
                + CZ3(3, KS + 1, 2) * PHI(q, KS, i, j) - CZ3(1, KS, 2) * PHI(q, KS + 1, i, j));
    };
    auto atKEm1 = [&]() {
        return (-CZ3(2, KE - 1, 2) * PHI(q, KE - 1, i, j) + CZ3(3, KE - 1, 2) * PHI(q, KE - 2, i, j)
                - CZ3(1, KE - 2, 2) * PHI(q, KE - 3, i, j));
    };
    auto atKE = [&]() {
        return (+CZ3(1, KE, 2) * PHI(q, KE - 1, i, j) + CZ3(3, KE, 2) * PHI(q, KE - 1, i, j)
                - CZ3(1, KE - 1, 2) * PHI(q, KE - 2, i, j));
    };
    if (k >= KS + 2 && k <= KE - 2) return inner(k);
    if (k == KS + 1) return atKSp1();
    if (k == KS) return -atKSp1();
    if (k == KS - 1) return -inner(KS + 2);
    if (k == KS - 2) return -inner(KS + 3);
    if (k == KE - 1) return atKEm1();
    if (k == KE) return atKE();
    if (k == KE + 1) return -atKE();
    return -atKEm1();
}

template <class IO>
__device__ typename IO::T nd_dx(IO &io, const Ctx &x, int q, int o, int k, int i, int j)
{
    const Grid &g = x.g;
    using T = typename IO::T;
    if (o == 0)
        return (+CX3(1, i + 1, 1) * PHI(q, k, i + 2, j) - CX3(2, i + 1, 1) * PHI(q, k, i + 1, j)
                + CX3(3, i + 1, 1) * PHI(q, k, i, j) - CX3(1, i, 1) * PHI(q, k, i - 1, j));
    return (+CX3(1, i, 2) * PHI(q, k, i + 1, j) - CX3(2, i, 2) * PHI(q, k, i, j)
            + CX3(3, i, 2) * PHI(q, k, i - 1, j) - CX3(1, i - 1, 2) * PHI(q, k, i - 2, j));
}
template <class IO>
__device__ typename IO::T nd_dy(IO &io, const Ctx &x, int q, int o, int k, int i, int j)
{
    const Grid &g = x.g;
    using T = typename IO::T;
    if (o == 0)
        return (+CY3(1, j + 1, 1) * PHI(q, k, i, j + 2) - CY3(2, j + 1, 1) * PHI(q, k, i, j + 1)
                + CY3(3, j + 1, 1) * PHI(q, k, i, j) - CY3(1, j, 1) * PHI(q, k, i, j - 1));
    return (+CY3(1, j, 2) * PHI(q, k, i, j + 1) - CY3(2, j, 2) * PHI(q, k, i, j)
            + CY3(3, j, 2) * PHI(q, k, i, j - 1) - CY3(1, j - 1, 2) * PHI(q, k, i, j - 2));
}

// one num_diff component (v, dir) at every level of an interior column (k_numfilter)
template <int V, int DIR>
struct PassND {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        const size_t o = c;
        const T ncz = (k >= KS - 1 && k <= KE) ? TB(x.nd.cdz, k - 1) : T(0.0);
        const T ncx = TB(x.nd.cdx, i - 1), nfx = TB(x.nd.fdx, i - 1), ncy = TB(x.nd.cdy, j - 1), nfy = TB(x.nd.fdy, j - 1);
        const T sfc = T(x.nd.sfc);
        auto sfct = [&](T v) -> T {
            if (k == KS) return v * sfc;
            if (k == KS + 1) return v * (T(1.0) + sfc) * T(0.5);
            return v;
        };
        auto DN = [&](size_t p) { return IN(XD, p); };
        const bool kin = (k >= KS && k <= KE), kz = (k >= KS && k <= KE - 1);
        T r = T(0.0);
        if (V == 1 && DIR == 1) {
            if (k >= KS - 1 && k <= KE) r = nd_dz0(io, x, 0, k, i, j) * ncz;
        } else if (V == 1 && DIR == 2) {
            if (kin) r = sfct(nd_dx(io, x, 0, 0, k, i, j) * ncx);
        } else if (V == 1 && DIR == 3) {
            if (kin) r = sfct(nd_dy(io, x, 0, 0, k, i, j) * ncy);
        } else if (V == 2 && DIR == 1) {
            if (k >= KS + 1 && k <= KE - 1) r = nd_dz1(io, x, 1, k, i, j) * TB(x.nd.fdz, k - 1) * DN(o);
        } else if (V == 2 && DIR == 2) {
            if (kz) r = sfct(nd_dx(io, x, 1, 0, k, i, j) * ncx * T(0.25) * (DN(o + 1 + sI) + DN(o + 1) + DN(o + sI) + DN(o)));
        } else if (V == 2 && DIR == 3) {
            if (kz) r = sfct(nd_dy(io, x, 1, 0, k, i, j) * ncy * T(0.25) * (DN(o + 1 + sJ) + DN(o + 1) + DN(o + sJ) + DN(o)));
        } else if (V == 3 && DIR == 1) {
            if (kz) r = nd_dz0(io, x, 2, k, i, j) * ncz * T(0.25) * (DN(o + 1 + sI) + DN(o + 1) + DN(o + sI) + DN(o));
        } else if (V == 3 && DIR == 2) {
            if (kin) r = sfct(nd_dx(io, x, 2, 1, k, i, j) * nfx * DN(o));
        } else if (V == 3 && DIR == 3) {
            if (kin) r = sfct(nd_dy(io, x, 2, 0, k, i, j) * ncy * T(0.25) * (DN(o + sI + sJ) + DN(o + sI) + DN(o + sJ) + DN(o)));
        } else if (V == 4 && DIR == 1) {
            if (kz) r = nd_dz0(io, x, 3, k, i, j) * ncz * T(0.25) * (DN(o + 1 + sJ) + DN(o + 1) + DN(o + sJ) + DN(o));
        } else if (V == 4 && DIR == 2) {
            if (kin) r = sfct(nd_dx(io, x, 3, 0, k, i, j) * ncx * T(0.25) * (DN(o + sI + sJ) + DN(o + sJ) + DN(o + sI) + DN(o)));
        } else if (V == 4 && DIR == 3) {
            if (kin) r = sfct(nd_dy(io, x, 3, 1, k, i, j) * nfy * DN(o));
        } else if (V == 5 && DIR == 1) {
            if (kz) r = nd_dz0(io, x, 4, k, i, j) * ncz * T(0.5) * (DN(o + 1) + DN(o));
            else if (k == KS - 1) r = nd_dz0(io, x, 4, k, i, j) * ncz * DN(idx3(g, KS, i, j));
            else if (k == KE) r = nd_dz0(io, x, 4, k, i, j) * ncz * DN(o);
        } else if (V == 5 && DIR == 2) {
            if (kin) r = sfct(nd_dx(io, x, 4, 0, k, i, j) * ncx * T(0.5) * (DN(o + sI) + DN(o)));
        } else {
            if (kin) r = sfct(nd_dy(io, x, 4, 0, k, i, j) * ncy * T(0.5) * (DN(o + sJ) + DN(o)));
        }
        io.out(NDF(V, DIR), o, r);
    }
};

// ============================================================================
// the HEVI stage
// ============================================================================
// hevi_pres :343-361 on the levels the flat-terrain stage reads
struct PassDPRES {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        io.out(DPRES, c, CS(DPRES0, c) + CS(RT2P, c) * (IN(XR, c) - CS(REFRHOT, c)));
    }
};

// hevi_mflx_z/x/y :365-438 (flat terrain: the explicit vertical part is num_diff)
struct PassMFLX {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        // the inputs are loaded unconditionally and in one order (one slot each)
        const T nz = IN(NDF(1, 1), c), U = IN(XU, c), nx = IN(NDF(1, 2), c), V = IN(XV, c), ny = IN(NDF(1, 3), c);
        if (j >= g.JS && i >= g.IS) io.out(MZ, c, (k == KS - 1 || k == KE) ? T(0.0) : nz);
        if (j >= g.JS && k >= KS) io.out(MX, c, U + nx);
        if (i >= g.IS && k >= KS) io.out(MY, c, V + ny);
    }
};

// hevi_sr :443-479
struct PassSR {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        const T adv_r = -((IN(MX, c) - IN(MX, c - sI)) * TB(g.RCDX, i - 1) + (IN(MY, c) - IN(MY, c - sJ)) * TB(g.RCDY, j - 1));
        io.out(SR, c, (-(IN(MZ, c) - IN(MZ, c - 1)) * TB(g.RCDZ, k - 1) + adv_r) + CS(TD, c));
    }
};

// vertical w-momentum flux above level k, fluxZ_XYW (ud3.F90:358-452)
template <int S>
struct PassQWZ {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        if (k < KS || k > KE - 2) {
            io.out(QWZ, c, T(0.0));
            return;
        }
        const T Mk = IN(XW, c), Mk1 = IN(XW, c + 1);
        const T vel = (T(0.5) * (Mk + Mk1)) / IN(XD, c + 1);
        const T Mm1 = IN(XW, c - 1), Mk2 = IN(XW, c + 2); // both branches' points, loaded in one order
        const T q = (k == KS) ? ipL<S>(vel, Mk, Mk1, Mk2) : ip4<S>(vel, Mm1, Mk, Mk1, Mk2);
        io.out(QWZ, c, T(x.J33G) * vel * q + IN(NDF(2, 1), c + 1));
    }
};

// horizontal w-momentum fluxes fluxX_XYW / fluxY_XYW (ud3.F90:598-748)
template <int S, int DIRY>
struct PassQWH {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        const size_t s = DIRY ? sJ : sI;
        const int mom = DIRY ? XV : XU;
        const T f1 = TB(g.F2H1, k - 1), f2 = TB(g.F2H2, k - 1), h = T(0.5);
        const T vel = (f1 * IN(mom, c + 1) + f2 * IN(mom, c))
                      / (f1 * h * (IN(XD, c + 1) + IN(XD, c + 1 + s)) + f2 * h * (IN(XD, c) + IN(XD, c + s)));
        io.out(DIRY ? QWY : QWX, c,
               vel * ip4<S>(vel, IN(XW, c - s), IN(XW, c), IN(XW, c + s), IN(XW, c + 2 * s)) + IN(NDF(2, DIRY ? 3 : 2), c));
    }
};

// hevi_sw :528-578
struct PassSW {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        const T advcv = -(IN(QWZ, c) - IN(QWZ, c - 1)) * TB(g.RFDZ, k - 1);
        const T adv_w = -((IN(QWX, c) - IN(QWX, c - sI)) * TB(g.RCDX, i - 1) + (IN(QWY, c) - IN(QWY, c - sJ)) * TB(g.RCDY, j - 1));
        const T wdmp = -TB(x.wdamp, k - 1) * IN(X0W, c);
        io.out(SW, c, (advcv + adv_w) + wdmp + T(0.0) + CS(TW, c));
    }
};

// POTT :586-598
struct PassPOTT {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        io.out(POTT, c, IN(XR, c) / IN(XD, c));
    }
};

// theta fluxes fluxZ_XYZ / fluxX_XYZ / fluxY_XYZ (ud3.F90:157-353) with num_diff
template <int S>
struct PassTZ {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        if (k < KS || k > KE - 1) {
            io.out(TZ, c, T(0.0));
            return;
        }
        // every branch's points are loaded first, in one order, so that each
        // input keeps one derivative slot whatever the branch (KS-1 and KE+1 are
        // in the array; an unused point contributes nothing)
        const T mZ = IN(MZ, c);
        const T Pm1 = IN(POTT, c - 1), P0 = IN(POTT, c), P1 = IN(POTT, c + 1), P2 = IN(POTT, c + 2);
        T ti;
        if (k == KS) ti = ipL<S>(mZ, P0, P1, P2);
        else if (k == KE - 1) ti = ipH<S>(mZ, P1, P0, Pm1);
        else ti = ip4<S>(mZ, Pm1, P0, P1, P2);
        io.out(TZ, c, mZ * ti + IN(NDF(5, 1), c));
    }
};
template <int S, int DIRY>
struct PassTH {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        const size_t s = DIRY ? sJ : sI;
        const T vel = IN(DIRY ? MY : MX, c);
        io.out(DIRY ? TY : TX, c,
               vel * ip4<S>(vel, IN(POTT, c - s), IN(POTT, c), IN(POTT, c + s), IN(POTT, c + 2 * s)) + IN(NDF(5, DIRY ? 3 : 2), c));
    }
};

// hevi_st :625-661
struct PassST {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        const T adv_t = -((IN(TX, c) - IN(TX, c - sI)) * TB(g.RCDX, i - 1) + (IN(TY, c) - IN(TY, c - sJ)) * TB(g.RCDY, j - 1));
        io.out(ST, c, (-(IN(TZ, c) - IN(TZ, c - 1)) * TB(g.RCDZ, k - 1) + adv_t) + CS(TR, c));
    }
};

// face potential temperature PT(k), valueW_Z (ud3.F90:98-153), k = KS..KE-1
template <int S, class IO>
__device__ typename IO::T face_theta(IO &io, const Ctx &x, size_t c, int k)
{
    using T = typename IO::T;
    const int KS = x.g.KS, KE = x.g.KE;
    const T M0 = IN(XW, c);
    if (k == KS) return ipL<S>(M0, IN(POTT, c), IN(POTT, c + 1), IN(POTT, c + 2));
    if (k == KE - 1) return ipH<S>(M0, IN(POTT, c + 1), IN(POTT, c), IN(POTT, c - 1));
    return ip4<S>(M0, IN(POTT, c - 1), IN(POTT, c), IN(POTT, c + 1), IN(POTT, c + 2));
}

// hevi_solver :665-809 for one column (forward and tangent-linear)
template <int S, class IO>
__device__ void column_forward(IO &io, const Ctx &x, int i, int j)
{
    using T = typename IO::T;
    const Grid &g = x.g;
    const int KS = g.KS, KE = g.KE;
    const size_t c1 = idx3(g, 1, i, j);
    auto C_ = [&](int k) { return c1 + (size_t)(k - 1); };
    const double dt = x.dt, J33G = x.J33G, dt2 = dt * dt;
    for (int k = KS; k <= KE - 1; ++k) io.out(PTf, C_(k), face_theta<S>(io, x, C_(k), k));
    auto Acoef = [&](int k) { return T(dt2 * J33G * ld(g.RCDZ + k - 1)) * CS(RT2P, C_(k)) * T(J33G); };
    T e_prev = T(0.0), f_prev = T(0.0);
    for (int k = KS; k <= KE - 1; ++k) {
        const T rfdz = TB(g.RFDZ, k - 1);
        const T B = T(GRAV * dt2 * J33G / (ld(g.CDZ + k) + ld(g.CDZ + k - 1)));
        const T Ak = Acoef(k), Ak1 = Acoef(k + 1);
        const T F2 = T(1.0) + (io.in(PTf, C_(k)) * rfdz * (Ak1 + Ak));
        // right-hand side C(k) (:698-722)
        const T RTL1 = CS(RT2P, C_(k + 1)), RTL0 = CS(RT2P, C_(k));
        const T pg = -(IN(DPRES, C_(k + 1)) + RTL1 * T(dt) * IN(ST, C_(k + 1)) - IN(DPRES, C_(k)) - RTL0 * T(dt) * IN(ST, C_(k)))
                         * rfdz * T(J33G)
                     - T(GRAV) * (TB(g.F2H1, k - 1) * (IN(XD, C_(k + 1)) - CS(REFDENS, C_(k + 1)) + IN(SR, C_(k + 1)) * T(dt))
                                  + TB(g.F2H2, k - 1) * (IN(XD, C_(k)) - CS(REFDENS, C_(k)) + IN(SR, C_(k)) * T(dt)));
        const T Ck = IN(XW, C_(k)) + T(dt) * (pg + IN(SW, C_(k)));
        T F1 = T(0.0), F3 = T(0.0);
        if (k <= KE - 2) F1 = -(io.in(PTf, C_(k + 1)) * rfdz * Ak1 + B);
        if (k > KS) F3 = -(io.in(PTf, C_(k - 1)) * rfdz * Ak - B);
        io.out(F1f, C_(k), F1);
        io.out(F2f, C_(k), F2);
        io.out(F3f, C_(k), F3);
        if (k == KS) {
            const T rdenom = T(1.0) / F2;
            e_prev = -F1 * rdenom;
            f_prev = Ck * rdenom;
        } else if (k <= KE - 2) {
            const T rdenom = T(1.0) / (F2 + F3 * e_prev);
            e_prev = -F1 * rdenom;
            f_prev = (Ck - F3 * f_prev) * rdenom;
        } else {
            f_prev = (Ck - F3 * f_prev) / (F2 + F3 * e_prev);
        }
        io.out(Ef, C_(k), e_prev);
        io.out(Ff, C_(k), f_prev);
    }
    // back substitution (solve_direct :1120-1124)
    T Cn = f_prev;
    io.out(Cf, C_(KE - 1), Cn);
    for (int k = KE - 2; k >= KS; --k) {
        Cn = io.in(Ef, C_(k)) * Cn + io.in(Ff, C_(k));
        io.out(Cf, C_(k), Cn);
    }
    // back-update :728-790
    for (int m = KS; m <= KE; ++m) {
        const T rcdz = TB(g.RCDZ, m - 1);
        const T Cm = m <= KE - 1 ? io.in(Cf, C_(m)) : T(0.0), Cm1 = m >= KS + 1 ? io.in(Cf, C_(m - 1)) : T(0.0);
        T adr, adt;
        if (m == KE) {
            adr = Cm1 * T(J33G) * rcdz;
            adt = Cm1 * io.in(PTf, C_(KE - 1)) * T(J33G) * rcdz;
        } else if (m == KS) {
            adr = -Cm * T(J33G) * rcdz;
            adt = -Cm * io.in(PTf, C_(KS)) * T(J33G) * rcdz;
        } else {
            adr = -(Cm - Cm1) * T(J33G) * rcdz;
            adt = -(Cm * io.in(PTf, C_(m)) - Cm1 * io.in(PTf, C_(m - 1))) * T(J33G) * rcdz;
        }
        io.out(ODRK, C_(m), IN(X0D, C_(m)) + T(dt) * (adr + IN(SR, C_(m))));
        io.out(ORRK, C_(m), IN(X0R, C_(m)) + T(dt) * (adt + IN(ST, C_(m))));
        if (m <= KE - 1) io.out(OWRK, C_(m), IN(X0W, C_(m)) + (Cm - IN(XW, C_(m))));
        else io.out(OWRK, C_(m), T(0.0));
    }
    io.out(OWRK, C_(KS - 1), T(0.0));
}

template <int S, class IOT>
__global__ void __launch_bounds__(128) k_column(const Ctx x)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= x.g.IMAX * x.g.JMAX) return;
    const int i = x.g.IS + t % x.g.IMAX, j = x.g.JS + t / x.g.IMAX;
    IOT io(x);
    column_forward<S>(io, x, i, j);
}

// adjoint of the column (values of PT, F1..F3 and C from the forward column);
// adjoints are added with plain stores: this thread alone touches its column
template <int S>
__global__ void __launch_bounds__(128) k_column_adj(const Ctx x)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= x.g.IMAX * x.g.JMAX) return;
    const Grid &g = x.g;
    const int i = g.IS + t % g.IMAX, j = g.JS + t / g.IMAX;
    const int KS = g.KS, KE = g.KE;
    const size_t c1 = idx3(g, 1, i, j);
    auto C_ = [&](int k) { return c1 + (size_t)(k - 1); };
    const double dt = x.dt, J33G = x.J33G, dt2 = dt * dt;
    double *const *V = x.val;
    double *const *L = x.aux;
    auto val = [&](int f, int k) { return V[f][C_(k)]; };
    auto lam = [&](int f, int k) -> double & { return L[f][C_(k)]; };
    // adjoint of the solution C and of PT, gathered in the column work arrays
    // (aux of Cf and PTf), then the transposed solve in Ef/Ff (values)
    for (int k = KS - 1; k <= KE; ++k) {
        lam(Cf, k) = 0.0;
        lam(PTf, k) = 0.0;
    }
    for (int m = KS; m <= KE; ++m) {
        const double rcdz = ld(g.RCDZ + m - 1);
        const double lD = lam(ODRK, m), lR = lam(ORRK, m);
        lam(X0D, m) += lD;
        lam(X0R, m) += lR;
        lam(SR, m) += dt * lD;
        lam(ST, m) += dt * lR;
        const double gD = dt * lD * J33G * rcdz, gR = dt * lR * J33G * rcdz;
        if (m == KE) {
            lam(Cf, KE - 1) += gD + gR * val(PTf, KE - 1);
            lam(PTf, KE - 1) += gR * val(Cf, KE - 1);
        } else if (m == KS) {
            lam(Cf, KS) -= gD + gR * val(PTf, KS);
            lam(PTf, KS) -= gR * val(Cf, KS);
        } else {
            lam(Cf, m) -= gD + gR * val(PTf, m);
            lam(PTf, m) -= gR * val(Cf, m);
            lam(Cf, m - 1) += gD + gR * val(PTf, m - 1);
            lam(PTf, m - 1) += gR * val(Cf, m - 1);
        }
        if (m <= KE - 1) {
            const double lW = lam(OWRK, m);
            lam(X0W, m) += lW;
            lam(Cf, m) += lW;
            lam(XW, m) -= lW;
        }
    }
    // transposed tridiagonal solve: M^T y = lam(C). Row r of M (level k) holds
    // F3(k) C(k-1) + F2(k) C(k) + F1(k) C(k+1); M^T has F1(k-1) below the
    // diagonal and F3(k+1) above it. Elimination factors in val(Ef), val(Ff).
    {
        double cp = 0.0, bp = 0.0;
        for (int k = KS; k <= KE - 1; ++k) {
            const double sub = k > KS ? val(F1f, k - 1) : 0.0;
            const double sup = k < KE - 1 ? val(F3f, k + 1) : 0.0;
            const double m = val(F2f, k) - sub * cp;
            cp = sup / m;
            bp = (lam(Cf, k) - sub * bp) / m;
            V[Ef][C_(k)] = cp;
            V[Ff][C_(k)] = bp;
        }
        double y = bp;
        lam(Ff, KE - 1) = y;
        for (int k = KE - 2; k >= KS; --k) {
            y = V[Ff][C_(k)] - V[Ef][C_(k)] * y;
            lam(Ff, k) = y; // lam(Ff) now holds y = the adjoint of the right-hand side
        }
    }
    auto Acoef = [&](int k) { return dt2 * J33G * ld(g.RCDZ + k - 1) * V[RT2P][C_(k)] * J33G; };
    for (int k = KS; k <= KE - 1; ++k) {
        const double y = lam(Ff, k);
        const double rfdz = ld(g.RFDZ + k - 1);
        const double Ak = Acoef(k), Ak1 = Acoef(k + 1);
        // matrix entries: lam(M_rc) = -y_r C_c
        const double lF2 = -y * val(Cf, k);
        lam(PTf, k) += lF2 * rfdz * (Ak1 + Ak);
        if (k <= KE - 2) lam(PTf, k + 1) -= (-y * val(Cf, k + 1)) * rfdz * Ak1;
        if (k > KS) lam(PTf, k - 1) -= (-y * val(Cf, k - 1)) * rfdz * Ak;
        // right-hand side C(k) = MOMZ(k) + dt (pg + Sw(k))
        lam(XW, k) += y;
        const double gy = dt * y;
        lam(SW, k) += gy;
        const double a = -gy * rfdz * J33G;
        lam(DPRES, k + 1) += a;
        lam(DPRES, k) -= a;
        lam(ST, k + 1) += a * V[RT2P][C_(k + 1)] * dt;
        lam(ST, k) -= a * V[RT2P][C_(k)] * dt;
        const double b = -gy * GRAV;
        const double f1 = ld(g.F2H1 + k - 1), f2 = ld(g.F2H2 + k - 1);
        lam(XD, k + 1) += b * f1;
        lam(SR, k + 1) += b * f1 * dt;
        lam(XD, k) += b * f2;
        lam(SR, k) += b * f2 * dt;
    }
    // face theta: PT(k) from POTT (the UD3 switch on MOMZ has no derivative)
    for (int k = KS; k <= KE - 1; ++k) {
        const double lpt = lam(PTf, k);
        if (lpt == 0.0) continue;
        AdjIO<5> io(x);
        const Jet<5> pt = face_theta<S>(io, x, C_(k), k);
        for (int q = 0; q < io.n; ++q)
            if (pt.d[q] != 0.0) L[io.fid[q]][io.off[q]] += lpt * pt.d[q];
    }
}

// z flux of rho*u / rho*v, fluxZ_UYZ / fluxZ_XVZ (ud3.F90:753-859, 1173-1279)
template <int S, int DIRY>
struct PassQHZ {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        const int out = DIRY ? QVZ : QUZ, val = DIRY ? XV : XU;
        if (k < KS || k > KE - 1) {
            io.out(out, c, T(0.0));
            return;
        }
        const size_t s = DIRY ? sJ : sI;
        const T h = T(0.5);
        const T den = TB(g.F2H1, k - 1) * h * (IN(XD, c + 1) + IN(XD, c + 1 + s)) + TB(g.F2H2, k - 1) * h * (IN(XD, c) + IN(XD, c + s));
        const T vel = (h * (IN(XW, c) + IN(XW, c + s))) / den;
        const T Vm1 = IN(val, c - 1), V0 = IN(val, c), V1 = IN(val, c + 1), V2 = IN(val, c + 2); // one order
        T q;
        if (k == KS) q = ipL<S>(vel, V0, V1, V2);
        else if (k == KE - 1) q = ipH<S>(vel, V1, V0, Vm1);
        else q = ip4<S>(vel, Vm1, V0, V1, V2);
        io.out(out, c, T(x.J33G) * vel * q + IN(NDF(DIRY ? 4 : 3, 1), c));
    }
};

// flux along the momentum's own direction, with the index shift of
// fluxX_UYZ (ud3.F90:1053-1109) / fluxY_XVZ (ud3.F90:1531-1587): output at
// face o is computed at the cell o+1
template <int S, int DIRY>
struct PassQHA {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        const size_t s = DIRY ? sJ : sI;
        const int m = DIRY ? XV : XU;
        const T vel = (T(0.5) * (IN(m, c + s) + IN(m, c))) / IN(XD, c + s);
        io.out(DIRY ? QVY : QUX, c,
               vel * ip4<S>(vel, IN(m, c - s), IN(m, c), IN(m, c + s), IN(m, c + 2 * s)) + IN(NDF(DIRY ? 4 : 3, DIRY ? 3 : 2), c + s));
    }
};

// flux across the other horizontal direction, fluxY_UYZ (ud3.F90:1113-1167) /
// fluxX_XVZ (ud3.F90:1473-1527)
template <int S, int DIRY>
struct PassQHC {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        // DIRY = 0: y flux of rho*u, transported by MOMY averaged to the u point;
        // DIRY = 1: x flux of rho*v, transported by MOMX averaged to the v point
        const size_t s = DIRY ? sI : sJ;     // direction of the flux
        const size_t p = DIRY ? sJ : sI;     // direction of the momentum's stagger
        const int tr = DIRY ? XU : XV, m = DIRY ? XV : XU;
        const T vel = (T(0.5) * (IN(tr, c) + IN(tr, c + p)))
                      / (T(0.25) * (IN(XD, c) + IN(XD, c + sI) + IN(XD, c + sJ) + IN(XD, c + sI + sJ)));
        io.out(DIRY ? QVX : QUY, c,
               vel * ip4<S>(vel, IN(m, c - s), IN(m, c), IN(m, c + s), IN(m, c + 2 * s)) + IN(NDF(DIRY ? 4 : 3, DIRY ? 2 : 3), c));
    }
};

// hevi_momx :814-928 / hevi_momy :934-1048 (flat terrain)
template <int DIRY>
struct PassMOM {
    template <class IO>
    __device__ void operator()(IO &io, const Ctx &x, int k, int i, int j) const
    {
        PASS_BEGIN
        const double dt = x.dt;
        const size_t c2 = (size_t)(i - 1) + (size_t)g.IA * (j - 1);
        if (!DIRY) {
            const T advcv = -(IN(QUZ, c) - IN(QUZ, c - 1)) * TB(g.RCDZ, k - 1);
            const T advch = -((IN(QUX, c) - IN(QUX, c - sI)) * TB(g.RFDX, i - 1) + (IN(QUY, c) - IN(QUY, c - sJ)) * TB(g.RCDY, j - 1));
            const T pg = (IN(DPRES, c + sI) - IN(DPRES, c)) * TB(g.RFDX, i - 1);
            const T cor = T(0.125) * (CS(CORI, c2 + 1) + CS(CORI, c2));
            const T cf = cor * (IN(XV, c + sI) + IN(XV, c) + IN(XV, c + sI - sJ) + IN(XV, c - sJ));
            io.out(OURK, c, IN(X0U, c) + T(dt) * ((((advcv + advch) - pg) + cf) + T(0.0) + CS(TU, c)));
        } else {
            const T advcv = -(IN(QVZ, c) - IN(QVZ, c - 1)) * TB(g.RCDZ, k - 1);
            const T advch = -((IN(QVX, c) - IN(QVX, c - sI)) * TB(g.RCDX, i - 1) + (IN(QVY, c) - IN(QVY, c - sJ)) * TB(g.RFDY, j - 1));
            const T pg = (IN(DPRES, c + sJ) - IN(DPRES, c)) * TB(g.RFDY, j - 1);
            const T cor = T(-0.125) * (CS(CORI, c2 + g.IA) + CS(CORI, c2));
            const T cf = cor * (IN(XU, c + sJ) + IN(XU, c) + IN(XU, c - sI + sJ) + IN(XU, c - sI));
            io.out(OVRK, c, IN(X0V, c) + T(dt) * ((((advcv + advch) - pg) + cf) + T(0.0) + CS(TV, c)));
        }
    }
};

#undef PASS_BEGIN
#undef IN
#undef CS
#undef TB
#undef CZ3
#undef CX3
#undef CY3
#undef PHI

// ============================================================================
// RK4 combine, halo and boundary adjoints
// ============================================================================
// X = ((2 X1 + 4 X2 + 2 X3) + X4 - 3 X0) / 6 on the interior (FINAL mode of
// the stage kernel); 'tan' selects the tangent arrays
struct Combine {
    double *X[5];
    const double *S1[5], *S2[5], *S3[5], *S4[5];
};
__global__ void k_combine(const Grid g, const Combine a)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = g.KMAX * g.IMAX * g.JMAX;
    if (t >= n) return;
    const int k = g.KS + t % g.KMAX, i = g.IS + (t / g.KMAX) % g.IMAX, j = g.JS + t / (g.KMAX * g.IMAX);
    const size_t c = idx3(g, k, i, j);
    for (int v = 0; v < 5; ++v) {
        if (v == 1 && k == g.KE) continue; // MOMZ: KS..KE-1 (KE keeps the stage's zero)
        const double acc = ((a.S1[v][c] * 2.0) + a.S2[v][c] * 4.0) + a.S3[v][c] * 2.0;
        a.X[v][c] = ((acc + a.S4[v][c]) - a.X[v][c] * 3.0) / 6.0;
    }
    if (k == g.KE) a.X[1][c] = a.S4[1][c];
}
// the same combine in double-double arithmetic (hi parts in a, lo parts in l)
__global__ void k_combine_dd(const Grid g, const Combine a, const Combine l)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = g.KMAX * g.IMAX * g.JMAX;
    if (t >= n) return;
    const int k = g.KS + t % g.KMAX, i = g.IS + (t / g.KMAX) % g.IMAX, j = g.JS + t / (g.KMAX * g.IMAX);
    const size_t c = idx3(g, k, i, j);
    for (int v = 0; v < 5; ++v) {
        if (v == 1 && k == g.KE) continue;
        const DD s1(a.S1[v][c], l.S1[v][c]), s2(a.S2[v][c], l.S2[v][c]), s3(a.S3[v][c], l.S3[v][c]);
        const DD s4(a.S4[v][c], l.S4[v][c]), x0(a.X[v][c], l.X[v][c]);
        const DD acc = ((s1 * DD(2.0)) + s2 * DD(4.0)) + s3 * DD(2.0);
        const DD r = ((acc + s4) - x0 * DD(3.0)) / DD(6.0);
        a.X[v][c] = r.hi;
        l.X[v][c] = r.lo;
    }
    if (k == g.KE) {
        a.X[1][c] = a.S4[1][c];
        l.X[1][c] = l.S4[1][c];
    }
}
// its adjoint: lam(Xs) = w_s lam(X)/6 and lam(X) = -3 lam(X)/6 on the interior
struct CombineAdj {
    double *L[5];
    double *LS[4][5];
};
__global__ void k_combine_adj(const Grid g, const CombineAdj a)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = g.KMAX * g.IMAX * g.JMAX;
    if (t >= n) return;
    const int k = g.KS + t % g.KMAX, i = g.IS + (t / g.KMAX) % g.IMAX, j = g.JS + t / (g.KMAX * g.IMAX);
    const size_t c = idx3(g, k, i, j);
    for (int v = 0; v < 5; ++v) {
        if (v == 1 && k == g.KE) {
            a.L[1][c] = 0.0; // MOMZ(KE) = 0
            continue;
        }
        const double l = a.L[v][c] / 6.0;
        a.LS[0][v][c] += 2.0 * l;
        a.LS[1][v][c] += 4.0 * l;
        a.LS[2][v][c] += 2.0 * l;
        a.LS[3][v][c] += l;
        a.L[v][c] = -3.0 * l;
    }
}

// adjoint of the periodic halo fill: every halo cell's adjoint goes to its
// periodic image in the interior (all KA levels) and the halo cell's is cleared
struct FieldPtrs {
    double *f[16];
};
__global__ void k_halo_adj(const Grid g, const FieldPtrs fl)
{
    const int nA = 2 * g.JHALO * g.IA, nB = 2 * g.IHALO * g.JMAX;
    const int h = blockIdx.x * blockDim.y + threadIdx.y;
    if (h >= nA + nB) return;
    int i, j;
    if (h < nA) {
        const int r = h / g.IA;
        i = 1 + h % g.IA;
        j = r < g.JHALO ? 1 + r : g.JE + 1 + (r - g.JHALO);
    } else {
        const int q = h - nA, r = q / g.JMAX;
        j = g.JS + q % g.JMAX;
        i = r < g.IHALO ? 1 + r : g.IE + 1 + (r - g.IHALO);
    }
    const int si = i < g.IS ? i + g.IMAX : (i > g.IE ? i - g.IMAX : i);
    const int sj = j < g.JS ? j + g.JMAX : (j > g.JE ? j - g.JMAX : j);
    double *v = fl.f[blockIdx.y];
    const size_t dst = idx3(g, 1, i, j), src = idx3(g, 1, si, sj);
    for (int k = threadIdx.x; k < g.KA; k += 32) {
        const double l = v[dst + k];
        if (l != 0.0) atomicAdd(v + src + k, l);
        v[dst + k] = 0.0;
    }
}
// adjoint of the vertical boundary values (k_vbc): halo levels take the value
// at KS / KE (MOMZ: zero)
__global__ void k_vbc_adj(const Grid g, const FieldPtrs fl)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.IMAX * g.JMAX) return;
    const int i = g.IS + t % g.IMAX, j = g.JS + t / g.IMAX;
    const size_t c = idx3(g, 1, i, j);
    for (int v = 0; v < 5; ++v) {
        double *L = fl.f[v];
        for (int k = 1; k <= g.KS - 1; ++k) {
            if (v != 1) L[c + g.KS - 1] += L[c + k - 1];
            L[c + k - 1] = 0.0;
        }
        for (int k = g.KE + 1; k <= g.KA; ++k) {
            if (v != 1) L[c + g.KE - 1] += L[c + k - 1];
            L[c + k - 1] = 0.0;
        }
    }
}

// ============================================================================
// host side
// ============================================================================
namespace {

enum Mode { M_FWD, M_TLM, M_ADJ, M_DD };

template <class P, class IOT>
cudaError_t pass(const Ctx &x, Box b, cudaStream_t st)
{
    const long long n = b.count();
    if (n <= 0) return cudaSuccess;
    k_pass<P, IOT><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(x, b);
    return cudaGetLastError();
}
// the same pass in forward, tangent-linear or adjoint form; NJ = derivative
// slots of the adjoint (at least the number of inputs the pass loads)
template <class P, int NJ>
cudaError_t run(Mode m, const Ctx &x, Box b, cudaStream_t st)
{
    switch (m) {
    case M_FWD: return pass<P, FwdIO>(x, b, st);
    case M_TLM: return pass<P, TlmIO>(x, b, st);
    case M_DD: return pass<P, DdIO>(x, b, st);
    default: return pass<P, AdjIO<NJ>>(x, b, st);
    }
}

#define RUN(...)                                  \
    do {                                          \
        cudaError_t e_ = (__VA_ARGS__);           \
        if (e_ != cudaSuccess) return e_;         \
    } while (0)

cudaError_t numfilter(Mode m, const Ctx &x, cudaStream_t st)
{
    const Grid &g = x.g;
    const Box all{1, g.KA, 1, g.IA, 1, g.JA}, col{1, g.KA, g.IS, g.IE, g.JS, g.JE};
    auto nd = [&](auto v, auto d) -> cudaError_t {
        // at most 8 inputs per component: 4 filtered quantities and 4 densities
        return run<PassND<decltype(v)::value, decltype(d)::value>, 8>(m, x, col, st);
    };
#define ND_(v, d) RUN(nd(std::integral_constant<int, v>{}, std::integral_constant<int, d>{}))
    if (m != M_ADJ) {
        RUN(run<PassPhi, 10>(m, x, all, st));
        ND_(1, 1); ND_(1, 2); ND_(1, 3); ND_(2, 1); ND_(2, 2); ND_(2, 3); ND_(3, 1); ND_(3, 2); ND_(3, 3);
        ND_(4, 1); ND_(4, 2); ND_(4, 3); ND_(5, 1); ND_(5, 2); ND_(5, 3);
    } else {
        ND_(5, 3); ND_(5, 2); ND_(5, 1); ND_(4, 3); ND_(4, 2); ND_(4, 1); ND_(3, 3); ND_(3, 2); ND_(3, 1);
        ND_(2, 3); ND_(2, 2); ND_(2, 1); ND_(1, 3); ND_(1, 2); ND_(1, 1);
        RUN(run<PassPhi, 10>(m, x, all, st));
    }
#undef ND_
    return cudaSuccess;
}

template <int S>
cudaError_t stage_fwd(Mode m, const Ctx &x, cudaStream_t st)
{
    const Grid &g = x.g;
    const int KS = g.KS, KE = g.KE, IS = g.IS, IE = g.IE, JS = g.JS, JE = g.JE;
    RUN(run<PassDPRES, 2>(m, x, Box{KS, KE, IS, IE + 1, JS, JE + 1}, st));
    RUN(run<PassMFLX, 6>(m, x, Box{KS - 1, KE, IS - 1, IE, JS - 1, JE}, st));
    RUN(run<PassSR, 6>(m, x, Box{KS, KE, IS, IE, JS, JE}, st));
    RUN(run<PassQWZ<S>, 8>(m, x, Box{KS - 1, KE, IS, IE, JS, JE}, st));
    RUN(run<PassQWH<S, 0>, 12>(m, x, Box{KS, KE - 1, IS - 1, IE, JS, JE}, st));
    RUN(run<PassQWH<S, 1>, 12>(m, x, Box{KS, KE - 1, IS, IE, JS - 1, JE}, st));
    RUN(run<PassSW, 8>(m, x, Box{KS, KE - 1, IS, IE, JS, JE}, st));
    RUN(run<PassPOTT, 2>(m, x, Box{KS, KE, IS - 2, IE + 2, JS - 2, JE + 2}, st));
    RUN(run<PassTZ<S>, 6>(m, x, Box{KS - 1, KE, IS, IE, JS, JE}, st));
    RUN(run<PassTH<S, 0>, 6>(m, x, Box{KS, KE, IS - 1, IE, JS, JE}, st));
    RUN(run<PassTH<S, 1>, 6>(m, x, Box{KS, KE, IS, IE, JS - 1, JE}, st));
    RUN(run<PassST, 7>(m, x, Box{KS, KE, IS, IE, JS, JE}, st));
    {
        const int n = g.IMAX * g.JMAX;
        if (m == M_TLM) k_column<S, TlmIO><<<(n + 127) / 128, 128, 0, st>>>(x);
        else if (m == M_DD) k_column<S, DdIO><<<(n + 127) / 128, 128, 0, st>>>(x);
        else k_column<S, FwdIO><<<(n + 127) / 128, 128, 0, st>>>(x);
        RUN(cudaGetLastError());
    }
    RUN(run<PassQHZ<S, 0>, 12>(m, x, Box{KS - 1, KE, IS, IE, JS, JE}, st));
    RUN(run<PassQHA<S, 0>, 10>(m, x, Box{KS, KE, IS - 1, IE, JS, JE}, st));
    RUN(run<PassQHC<S, 0>, 12>(m, x, Box{KS, KE, IS, IE, JS - 1, JE}, st));
    RUN(run<PassMOM<0>, 14>(m, x, Box{KS, KE, IS, IE, JS, JE}, st));
    RUN(run<PassQHZ<S, 1>, 12>(m, x, Box{KS - 1, KE, IS, IE, JS, JE}, st));
    RUN(run<PassQHC<S, 1>, 12>(m, x, Box{KS, KE, IS - 1, IE, JS, JE}, st));
    RUN(run<PassQHA<S, 1>, 10>(m, x, Box{KS, KE, IS, IE, JS - 1, JE}, st));
    RUN(run<PassMOM<1>, 14>(m, x, Box{KS, KE, IS, IE, JS, JE}, st));
    return cudaSuccess;
}

// reverse sweep of one stage (the forward values of its intermediates present)
template <int S>
cudaError_t stage_adj(const Ctx &x, cudaStream_t st)
{
    const Mode m = M_ADJ;
    const Grid &g = x.g;
    const int KS = g.KS, KE = g.KE, IS = g.IS, IE = g.IE, JS = g.JS, JE = g.JE;
    RUN(run<PassMOM<1>, 14>(m, x, Box{KS, KE, IS, IE, JS, JE}, st));
    RUN(run<PassQHA<S, 1>, 10>(m, x, Box{KS, KE, IS, IE, JS - 1, JE}, st));
    RUN(run<PassQHC<S, 1>, 12>(m, x, Box{KS, KE, IS - 1, IE, JS, JE}, st));
    RUN(run<PassQHZ<S, 1>, 12>(m, x, Box{KS - 1, KE, IS, IE, JS, JE}, st));
    RUN(run<PassMOM<0>, 14>(m, x, Box{KS, KE, IS, IE, JS, JE}, st));
    RUN(run<PassQHC<S, 0>, 12>(m, x, Box{KS, KE, IS, IE, JS - 1, JE}, st));
    RUN(run<PassQHA<S, 0>, 10>(m, x, Box{KS, KE, IS - 1, IE, JS, JE}, st));
    RUN(run<PassQHZ<S, 0>, 12>(m, x, Box{KS - 1, KE, IS, IE, JS, JE}, st));
    {
        const int n = g.IMAX * g.JMAX;
        k_column_adj<S><<<(n + 127) / 128, 128, 0, st>>>(x);
        RUN(cudaGetLastError());
    }
    RUN(run<PassST, 7>(m, x, Box{KS, KE, IS, IE, JS, JE}, st));
    RUN(run<PassTH<S, 1>, 6>(m, x, Box{KS, KE, IS, IE, JS - 1, JE}, st));
    RUN(run<PassTH<S, 0>, 6>(m, x, Box{KS, KE, IS - 1, IE, JS, JE}, st));
    RUN(run<PassTZ<S>, 6>(m, x, Box{KS - 1, KE, IS, IE, JS, JE}, st));
    RUN(run<PassSW, 8>(m, x, Box{KS, KE - 1, IS, IE, JS, JE}, st));
    RUN(run<PassQWH<S, 1>, 12>(m, x, Box{KS, KE - 1, IS, IE, JS - 1, JE}, st));
    RUN(run<PassQWH<S, 0>, 12>(m, x, Box{KS, KE - 1, IS - 1, IE, JS, JE}, st));
    RUN(run<PassQWZ<S>, 8>(m, x, Box{KS - 1, KE, IS, IE, JS, JE}, st));
    RUN(run<PassPOTT, 2>(m, x, Box{KS, KE, IS - 2, IE + 2, JS - 2, JE + 2}, st));
    RUN(run<PassSR, 6>(m, x, Box{KS, KE, IS, IE, JS, JE}, st));
    RUN(run<PassMFLX, 6>(m, x, Box{KS - 1, KE, IS - 1, IE, JS - 1, JE}, st));
    RUN(run<PassDPRES, 2>(m, x, Box{KS, KE, IS, IE + 1, JS, JE + 1}, st));
    return cudaSuccess;
}

cudaError_t halo_adj(const Grid &g, double *const *f, int n, cudaStream_t st)
{
    const int nh = 2 * g.JHALO * g.IA + 2 * g.IHALO * g.JMAX;
    for (int b = 0; b < n; b += 16) {
        FieldPtrs fl{};
        const int m = n - b < 16 ? n - b : 16;
        for (int q = 0; q < m; ++q) fl.f[q] = f[b + q];
        k_halo_adj<<<dim3((nh + 3) / 4, m), dim3(32, 4), 0, st>>>(g, fl);
    }
    return cudaGetLastError();
}

cudaError_t vbc_adj(const Grid &g, double *const *f, cudaStream_t st)
{
    FieldPtrs fl{};
    for (int q = 0; q < 5; ++q) fl.f[q] = f[q];
    const int n = g.IMAX * g.JMAX;
    k_vbc_adj<<<(n + 127) / 128, 128, 0, st>>>(g, fl);
    return cudaGetLastError();
}

} // namespace

// ---- the model and its scratch ------------------------------------------------------
// scratch layout (fields of N3): intermediates and column work (values, then
// tangents/adjoints), the filtered quantities and num_diff (values, aux), the
// four stage states (values, aux) and one 5-field temporary
size_t scratch_fields() { return 2 * (size_t)(N_INTER + 7) + 2 * 5 + 2 * 15 + 2 * 20 + 5; }

struct Bind {
    Ctx x;
    double *inter_v, *inter_a, *phi_v, *phi_a, *nd_v, *nd_a, *xs_v, *xs_a, *tmp;
};

static Bind make_bind(const Model &M)
{
    Bind b{};
    const size_t N3 = n3(M.g);
    double *p = M.scratch;
    b.inter_v = p; p += (size_t)(N_INTER + 7) * N3;
    b.inter_a = p; p += (size_t)(N_INTER + 7) * N3;
    b.phi_v = p; p += 5 * N3;
    b.phi_a = p; p += 5 * N3;
    b.nd_v = p; p += 15 * N3;
    b.nd_a = p; p += 15 * N3;
    b.xs_v = p; p += 20 * N3;
    b.xs_a = p; p += 20 * N3;
    b.tmp = p;
    Ctx &x = b.x;
    x.g = M.g;
    x.nd = M.nd;
    x.J33G = M.J33G;
    x.wdamp = M.wdamp;
    x.status = M.status;
    for (int q = 0; q < 5; ++q) x.val[TD + q] = const_cast<double *>(M.zero);
    x.val[DPRES0] = const_cast<double *>(M.DPRES0);
    x.val[RT2P] = const_cast<double *>(M.RT2P);
    x.val[REFRHOT] = const_cast<double *>(M.REF_rhot);
    x.val[REFDENS] = const_cast<double *>(M.REF_dens);
    x.val[REFPOTT] = const_cast<double *>(M.REF_pott);
    x.val[GEOP] = const_cast<double *>(M.PHI);
    x.val[CORI] = const_cast<double *>(M.CORIOLI);
    for (int q = 0; q < N_INTER; ++q) {
        x.val[N_INTER_FIRST + q] = b.inter_v + (size_t)q * N3;
        x.aux[N_INTER_FIRST + q] = b.inter_a + (size_t)q * N3;
    }
    for (int q = 0; q < 7; ++q) {
        x.val[PTf + q] = b.inter_v + (size_t)(N_INTER + q) * N3;
        x.aux[PTf + q] = b.inter_a + (size_t)(N_INTER + q) * N3;
    }
    for (int q = 0; q < 5; ++q) {
        x.val[PH0 + q] = b.phi_v + (size_t)q * N3;
        x.aux[PH0 + q] = b.phi_a + (size_t)q * N3;
    }
    for (int q = 0; q < 15; ++q) {
        x.val[ND0 + q] = b.nd_v + (size_t)q * N3;
        x.aux[ND0 + q] = b.nd_a + (size_t)q * N3;
    }
    return b;
}

static void bind_state(Ctx &x, int first, double *v, double *a, size_t N3)
{
    for (int q = 0; q < 5; ++q) {
        x.val[first + q] = v + (size_t)q * N3;
        x.aux[first + q] = a ? a + (size_t)q * N3 : nullptr;
    }
}

// one forward (M_FWD), tangent-linear (M_TLM: dX the tangent) or double-double
// (M_DD: dX the lo parts of X) short step in pass form
template <int S>
static cudaError_t step_tlm_impl(const Model &M, double *X, double *dX, Mode m)
{
    cudaStream_t st = M.stream;
    const size_t N3 = n3(M.g);
    Bind b = make_bind(M);
    Ctx &x = b.x;
    const bool tangent = m != M_FWD; // the aux arrays are bound and carried
    const Members one{};
    // numerical filter of the step's start state, then the halo of num_diff
    bind_state(x, XD, X, dX, N3);
    RUN(numfilter(m, x, st));
    {
        double *f[15];
        for (int q = 0; q < 15; ++q) f[q] = b.nd_v + (size_t)q * N3;
        periodic_halo(M.g, one, f, 15, st);
        if (tangent) {
            for (int q = 0; q < 15; ++q) f[q] = b.nd_a + (size_t)q * N3;
            periodic_halo(M.g, one, f, 15, st);
        }
    }
    const double dts[4] = {M.dt / 2.0, M.dt / 2.0, M.dt, M.dt};
    for (int s = 0; s < 4; ++s) {
        bind_state(x, X0D, X, dX, N3);
        if (s == 0) bind_state(x, XD, X, dX, N3);
        else bind_state(x, XD, b.xs_v + (size_t)(s - 1) * 5 * N3, b.xs_a + (size_t)(s - 1) * 5 * N3, N3);
        bind_state(x, ODRK, b.xs_v + (size_t)s * 5 * N3, b.xs_a + (size_t)s * 5 * N3, N3);
        x.dt = dts[s];
        RUN(stage_fwd<S>(m, x, st));
        if (s < 3) {
            double *f[5];
            for (int q = 0; q < 5; ++q) f[q] = b.xs_v + ((size_t)s * 5 + q) * N3;
            periodic_halo(M.g, one, f, 5, st);
            if (tangent) {
                for (int q = 0; q < 5; ++q) f[q] = b.xs_a + ((size_t)s * 5 + q) * N3;
                periodic_halo(M.g, one, f, 5, st);
            }
        }
    }
    const int n = M.g.KMAX * M.g.IMAX * M.g.JMAX;
    auto combine_of = [&](double *Xp, double *Sp) {
        Combine cb{};
        for (int q = 0; q < 5; ++q) {
            cb.X[q] = Xp + (size_t)q * N3;
            cb.S1[q] = Sp + (size_t)q * N3;
            cb.S2[q] = Sp + (size_t)(5 + q) * N3;
            cb.S3[q] = Sp + (size_t)(10 + q) * N3;
            cb.S4[q] = Sp + (size_t)(15 + q) * N3;
        }
        return cb;
    };
    if (m == M_DD) {
        k_combine_dd<<<(n + 127) / 128, 128, 0, st>>>(M.g, combine_of(X, b.xs_v), combine_of(dX, b.xs_a));
        RUN(cudaGetLastError());
    }
    for (int pass_ = 0; pass_ < (tangent ? 2 : 1); ++pass_) {
        double *Xp = pass_ ? dX : X, *Sp = pass_ ? b.xs_a : b.xs_v;
        if (m != M_DD) {
            k_combine<<<(n + 127) / 128, 128, 0, st>>>(M.g, combine_of(Xp, Sp));
            RUN(cudaGetLastError());
        }
        double *f[5];
        for (int q = 0; q < 5; ++q) f[q] = Xp + (size_t)q * N3;
        vertical_bc(M.g, one, f[0], f[1], f[2], f[3], f[4], st);
        periodic_halo(M.g, one, f, 5, st);
    }
    return cudaGetLastError();
}

template <int S>
static cudaError_t step_adj_impl(const Model &M, const double *X_in, double *lam)
{
    cudaStream_t st = M.stream;
    const size_t N3 = n3(M.g);
    Bind b = make_bind(M);
    Ctx &x = b.x;
    const Members one{};
    double *X = const_cast<double *>(X_in); // read only: bound as an input
    // ---- recompute the forward step: num_diff and the four stage states ----
    bind_state(x, XD, X, nullptr, N3);
    RUN(numfilter(M_FWD, x, st));
    {
        double *f[15];
        for (int q = 0; q < 15; ++q) f[q] = b.nd_v + (size_t)q * N3;
        periodic_halo(M.g, one, f, 15, st);
    }
    const double dts[4] = {M.dt / 2.0, M.dt / 2.0, M.dt, M.dt};
    auto bind_stage = [&](int s, bool with_adj) {
        bind_state(x, X0D, X, with_adj ? lam : nullptr, N3);
        if (s == 0) bind_state(x, XD, X, with_adj ? lam : nullptr, N3);
        else bind_state(x, XD, b.xs_v + (size_t)(s - 1) * 5 * N3, with_adj ? b.xs_a + (size_t)(s - 1) * 5 * N3 : nullptr, N3);
        bind_state(x, ODRK, b.xs_v + (size_t)s * 5 * N3, with_adj ? b.xs_a + (size_t)s * 5 * N3 : nullptr, N3);
        x.dt = dts[s];
    };
    for (int s = 0; s < 4; ++s) {
        bind_stage(s, false);
        RUN(stage_fwd<S>(M_FWD, x, st));
        if (s < 3) {
            double *f[5];
            for (int q = 0; q < 5; ++q) f[q] = b.xs_v + ((size_t)s * 5 + q) * N3;
            periodic_halo(M.g, one, f, 5, st);
        }
    }
    // ---- reverse sweep ----
    // lam holds the adjoint of the state after the step: move it to the
    // temporary, clear lam (it becomes the adjoint of the start state)
    RUN(cudaMemcpyAsync(b.tmp, lam, 5 * N3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    RUN(cudaMemsetAsync(lam, 0, 5 * N3 * sizeof(double), st));
    RUN(cudaMemsetAsync(b.xs_a, 0, 20 * N3 * sizeof(double), st));
    RUN(cudaMemsetAsync(b.nd_a, 0, 15 * N3 * sizeof(double), st));
    {
        double *f[5];
        for (int q = 0; q < 5; ++q) f[q] = b.tmp + (size_t)q * N3;
        RUN(halo_adj(M.g, f, 5, st));
        RUN(vbc_adj(M.g, f, st));
        CombineAdj ca{};
        for (int q = 0; q < 5; ++q) {
            ca.L[q] = f[q];
            for (int s = 0; s < 4; ++s) ca.LS[s][q] = b.xs_a + ((size_t)s * 5 + q) * N3;
        }
        const int n = M.g.KMAX * M.g.IMAX * M.g.JMAX;
        k_combine_adj<<<(n + 127) / 128, 128, 0, st>>>(M.g, ca);
        RUN(cudaGetLastError());
        // the start state's share of the combine
        for (int q = 0; q < 5; ++q)
            RUN(cudaMemcpyAsync(lam + (size_t)q * N3, f[q], N3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    for (int s = 3; s >= 0; --s) {
        // forward values of this stage's intermediates, then its adjoint
        bind_stage(s, false);
        RUN(stage_fwd<S>(M_FWD, x, st));
        bind_stage(s, true);
        RUN(cudaMemsetAsync(b.inter_a, 0, (size_t)(N_INTER + 7) * N3 * sizeof(double), st));
        RUN(stage_adj<S>(x, st));
        if (s > 0) {
            double *f[5];
            for (int q = 0; q < 5; ++q) f[q] = b.xs_a + ((size_t)(s - 1) * 5 + q) * N3;
            RUN(halo_adj(M.g, f, 5, st));
        }
    }
    {
        double *f[15];
        for (int q = 0; q < 15; ++q) f[q] = b.nd_a + (size_t)q * N3;
        RUN(halo_adj(M.g, f, 15, st));
    }
    RUN(cudaMemsetAsync(b.phi_a, 0, 5 * N3 * sizeof(double), st));
    bind_state(x, XD, X, lam, N3);
    RUN(numfilter(M_ADJ, x, st));
    return cudaGetLastError();
}

// the model's flux scheme as a template argument
template <class F>
static cudaError_t by_scheme(int scheme, F f)
{
    switch (scheme) {
    case UD3: return f(std::integral_constant<int, UD3>{});
    case CD4: return f(std::integral_constant<int, CD4>{});
    case KOREN: return f(std::integral_constant<int, KOREN>{});
    case CD2: return f(std::integral_constant<int, CD2>{});
    default: return cudaErrorInvalidValue;
    }
}
cudaError_t step_forward(const Model &M, double *X)
{
    return by_scheme(M.scheme, [&](auto s) { return step_tlm_impl<decltype(s)::value>(M, X, nullptr, M_FWD); });
}
cudaError_t step_tlm(const Model &M, double *X, double *dX)
{
    return by_scheme(M.scheme, [&](auto s) { return step_tlm_impl<decltype(s)::value>(M, X, dX, M_TLM); });
}
cudaError_t step_dd(const Model &M, double *X_hi, double *X_lo)
{
    return by_scheme(M.scheme, [&](auto s) { return step_tlm_impl<decltype(s)::value>(M, X_hi, X_lo, M_DD); });
}
cudaError_t step_adjoint(const Model &M, const double *X, double *lam)
{
    return by_scheme(M.scheme, [&](auto s) { return step_adj_impl<decltype(s)::value>(M, X, lam); });
}
cudaError_t boundary_adjoint(const Model &M, double *lam)
{
    const size_t N3 = n3(M.g);
    double *f[5];
    for (int q = 0; q < 5; ++q) f[q] = lam + (size_t)q * N3;
    RUN(halo_adj(M.g, f, 5, M.stream));
    return vbc_adj(M.g, f, M.stream);
}
#undef RUN

} // namespace ad
} // namespace hevi
