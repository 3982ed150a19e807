// Halo fill, vertical boundary fill, large-step preparation, metric check and
// budget reduction kernels.
#include "fill_body.cuh"

namespace hevi {

template <typename T, int NM>
__global__ void k_halo(const Grid gt, const FieldList<T> fl, const BatchT<NM> B)
{
    halo_column(gt, fl.f[blockIdx.y], B, (int)blockIdx.x, (int)threadIdx.y, (int)threadIdx.x);
}

template <typename T>
void periodic_halo(const Grid &g, const Members &mem, T *const *fields, int nf, cudaStream_t st)
{
    auto nblocks = [](const Grid &m) { return halo_blocks(m); };
    for (int base = 0; base < nf; base += 16) {
        FieldList<T> fl;
        const int n = (nf - base) < 16 ? (nf - base) : 16;
        for (int q = 0; q < n; ++q) fl.f[q] = fields[base + q];
        with_batch(g, mem, nblocks, [&](const auto &B, int nb) {
            constexpr int NM = std::decay_t<decltype(B)>::NMAX;
            k_halo<T, NM><<<dim3(nb, n), dim3(32, FILL_WARPS), 0, st>>>(g, fl, B);
            return cudaSuccess;
        });
    }
}
template void periodic_halo<double>(const Grid &, const Members &, double *const *, int, cudaStream_t);
template void periodic_halo<float>(const Grid &, const Members &, float *const *, int, cudaStream_t);

template <int NM>
__global__ void k_vbc(const Grid gt, double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT,
                      const BatchT<NM> B)
{
    vbc_column(gt, DENS, MOMZ, MOMX, MOMY, RHOT, B, (int)blockIdx.x, (int)threadIdx.y, (int)threadIdx.x);
}

void vertical_bc(const Grid &g, const Members &mem, double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT,
                 cudaStream_t st)
{
    auto nblocks = [](const Grid &m) { return vbc_blocks(m); };
    with_batch(g, mem, nblocks, [&](const auto &B, int nb) {
        constexpr int NM = std::decay_t<decltype(B)>::NMAX;
        k_vbc<NM><<<nb, dim3(32, FILL_WARPS), 0, st>>>(g, DENS, MOMZ, MOMX, MOMY, RHOT, B);
        return cudaSuccess;
    });
}

// ---- 3-D divergence for divergence damping, ATMOS_DYN_divergence
// (scale_atmos_dyn_common.F90:1437-1515) on k = KS-1..KE+1, i = IS..IE+1,
// j = JS..JE+1 with the KS and KE rows of :1487-1506. Flat terrain: the J13G/J23G
// terms are zeros and the GSQRT/MAPF factors are ones, which leaves every
// non-zero value unchanged.
__global__ void k_divergence(const Grid g, double *DDIV, const double *MOMZ, const double *MOMX, const double *MOMY,
                             const double *RCDZ, const double *RCDX, const double *RCDY, double J33G)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE + 1) return;
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const double rcdx = ld(RCDX + i - 1), rcdy = ld(RCDY + j - 1);
    for (int k = g.KS - 1 + threadIdx.x; k <= g.KE + 1; k += 32) {
        const size_t c = idx3(g, k, i, j);
        const double h = (ld(MOMX + c) - ld(MOMX + c - sI)) * rcdx + (ld(MOMY + c) - ld(MOMY + c - sJ)) * rcdy;
        double v;
        if (k == g.KS) v = J33G * (ld(MOMZ + c)) * ld(RCDZ + k - 1) + h;
        else if (k == g.KE) v = J33G * (-ld(MOMZ + c - 1)) * ld(RCDZ + k - 1) + h;
        else v = J33G * (ld(MOMZ + c) - ld(MOMZ + c - 1)) * ld(RCDZ + k - 1) + h;
        DDIV[c] = v;
    }
}

void divergence(const Grid &g, double *DDIV, const double *MOMZ, const double *MOMX, const double *MOMY,
                const double *RCDZ, const double *RCDX, const double *RCDY, double J33G, cudaStream_t st)
{
    dim3 b(32, 4), gr((g.IMAX + 1 + 3) / 4, g.JMAX + 1);
    k_divergence<<<gr, b, 0, st>>>(g, DDIV, MOMZ, MOMX, MOMY, RCDZ, RCDX, RCDY, J33G);
}

// ATMOS_DYN_divergence with terrain-following metrics (scale_atmos_dyn_common.F90:1437-1515):
// the general row for KS-1..KE+1, the rows at KS and KE written in place of it
__global__ void k_divergence_terrain(const Grid g, double *DDIV, const double *MOMZ, const double *MOMX,
                                     const double *MOMY, const Metrics M, double J33G)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE + 1) return;
    const size_t N3 = n3(g);
    const long sI = g.KA, sJ = (long)g.KA * g.IA;
    const int KS = g.KS, KE = g.KE;
    const double rcdx = ld(g.RCDX + i - 1), rcdy = ld(g.RCDY + j - 1);
    const double *GUZ = M.GSQRT + 4 * N3, *GVZ = M.GSQRT + 5 * N3; // I_UYZ, I_XVZ
    const double *J13 = M.J13G + N3, *J23 = M.J23G + N3;            // I_XYW
    const size_t NP = (size_t)g.IA * g.JA, p = (size_t)(i - 1) + (size_t)g.IA * (j - 1);
    // MAPF(i,j,a,b), b = I_XY (1), I_UY (2), I_XV (3)
#define MF(pp, aa, bb) ld(M.MAPF + (pp) + NP * ((size_t)((aa) - 1) + 2 * (size_t)((bb) - 1)))
    const double mxy = MF(p, 1, 1) * MF(p, 2, 1);
    for (int k = KS - 1 + threadIdx.x; k <= KE + 1; k += 32) {
        const size_t c = idx3(g, k, i, j);
        const double h = mxy * ((ld(MOMX + c) * ld(GUZ + c) / MF(p, 2, 2) - ld(MOMX + c - sI) * ld(GUZ + c - sI) / MF(p - 1, 2, 2)) * rcdx
                                + (ld(MOMY + c) * ld(GVZ + c) / MF(p, 1, 3) - ld(MOMY + c - sJ) * ld(GVZ + c - sJ) / MF(p - g.IA, 1, 3)) * rcdy);
        double v;
        if (k == KS) {
            v = J33G * (ld(MOMZ + c)) * ld(g.RCDZ + k - 1)
                + ((ld(MOMX + c + 1) + ld(MOMX + c + 1 - sI)) * ld(J13 + c + 1) - (ld(MOMX + c - 1) + ld(MOMX + c - sI)) * ld(J13 + c)
                   + (ld(MOMY + c + 1) + ld(MOMY + c + 1 - sJ)) * ld(J23 + c + 1) - (ld(MOMY + c) + ld(MOMY + c - sJ)) * ld(J23 + c))
                      * ld(g.RFDZ + k - 1)
                + h;
        } else if (k == KE) {
            v = J33G * (-ld(MOMZ + c - 1)) * ld(g.RCDZ + k - 1)
                + ((ld(MOMX + c) + ld(MOMX + c - sI)) * ld(J13 + c) - (ld(MOMX + c - 1) + ld(MOMX + c - 1 - sI)) * ld(J13 + c - 1)
                   + (ld(MOMY + c) + ld(MOMY + c - sJ)) * ld(J23 + c) - (ld(MOMY + c - 1) + ld(MOMY + c - 1 - sJ)) * ld(J23 + c - 1))
                      * ld(g.RFDZ + k - 1)
                + h;
        } else {
            v = J33G * (ld(MOMZ + c) - ld(MOMZ + c - 1)) * ld(g.RCDZ + k - 1)
                + ((ld(MOMX + c + 1) + ld(MOMX + c + 1 - sI)) * ld(J13 + c + 1) - (ld(MOMX + c - 1) + ld(MOMX + c - 1 - sI)) * ld(J13 + c - 1)
                   + (ld(MOMY + c + 1) + ld(MOMY + c + 1 - sJ)) * ld(J23 + c + 1) - (ld(MOMY + c - 1) + ld(MOMY + c - 1 - sJ)) * ld(J23 + c - 1))
                      / (ld(g.FDZ + k - 1) + ld(g.FDZ + k - 2))
                + h;
        }
        DDIV[c] = v;
    }
#undef MF
}

void divergence_terrain(const Grid &g, double *DDIV, const double *MOMZ, const double *MOMX, const double *MOMY,
                        const Metrics &M, double J33G, cudaStream_t st)
{
    dim3 b(32, 4), gr((g.IMAX + 1 + 3) / 4, g.JMAX + 1);
    k_divergence_terrain<<<gr, b, 0, st>>>(g, DDIV, MOMZ, MOMX, MOMY, M, J33G);
}

// ---- RT2P, DPRES0, REF_rhot once per large step (tstep_large_fvm_heve.F90:428-470, moist form) ----
__global__ void k_large_prep(const Grid g, const PrepArgs a)
{
    const int i = 1 + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = 1 + blockIdx.y;
    if (i > g.IA) return;
    const size_t N3 = n3(g), col = idx3(g, 1, i, j);
    const double P0 = 100000.0, Rdry = 287.04, CPdry = 1004.64, CVdry = CPdry - Rdry;
    for (int k = g.KS + threadIdx.x; k <= g.KE; k += 32) {
        const size_t c = col + k - 1;
        double Rtot = 0.0, CVtot = 0.0, CPtot = 0.0, QDRY = 1.0;
        for (int iq = 0; iq < a.QA; ++iq) {
            const double q = a.QTRC[c + (size_t)iq * N3];
            Rtot = Rtot + a.AQ_R[iq] * q;
            CVtot = CVtot + a.AQ_CV[iq] * q;
            CPtot = CPtot + a.AQ_CP[iq] * q;
            QDRY = QDRY - q * a.AQ_MASS[iq];
        }
        Rtot = Rtot + Rdry * QDRY;
        CVtot = CVtot + CVdry * QDRY;
        CPtot = CPtot + CPdry * QDRY;
        const double rhot = a.RHOT[c];
        const double PRES = P0 * pow(Rtot * rhot / P0, CPtot / CVtot);
        a.RT2P[c] = CPtot / CVtot * PRES / rhot;
        a.DPRES0[c] = PRES - a.REF_pres[c];
        a.REF_rhot[c] = rhot;
    }
}
__global__ void k_large_prep_edge(const Grid g, const PrepArgs a)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if (i > g.IA) return;
    const size_t col = idx3(g, 1, i, j);
    const int KS = g.KS, KE = g.KE;
    a.DPRES0[col + KS - 2] = a.DPRES0[col + KS] + (a.REF_pres[col + KS] - a.REF_pres[col + KS - 2]);
    a.DPRES0[col + KE] = a.DPRES0[col + KE - 2] + (a.REF_pres[col + KE - 2] - a.REF_pres[col + KE]);
}

void large_prep(const Grid &g, const PrepArgs &a, cudaStream_t st)
{
    dim3 b(32, 4), gr((g.IA + 3) / 4, g.JA);
    k_large_prep<<<gr, b, 0, st>>>(g, a);
    dim3 b2(128), g2((g.IA + 127) / 128, g.JA);
    k_large_prep_edge<<<g2, b2, 0, st>>>(g, a);
}

// ---- flat-terrain check of the metric arrays --------------------------------
__global__ void k_count_ne(const double *p, size_t n, double want, unsigned long long *count)
{
    unsigned long long local = 0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        local += (p[q] != want);
    if (local) atomicAdd(count, local);
}

void count_not_equal(const double *p, size_t n, double want, unsigned long long *count, cudaStream_t st)
{
    k_count_ne<<<148 * 8, 256, 0, st>>>(p, n, want, count);
}

// ---- FP64 domain budget: sum of var*CDZ*CDX*CDY over the interior ------------
// Deterministic two-level reduction: one partial per column (k summed in order),
// then a fixed-shape tree over columns.
__global__ void k_col_sum(const Grid g, const double *var, const double *CDX, const double *CDY, const double *CDZ, double *part)
{
    const int i = g.IS + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t col = idx3(g, 1, i, j);
    double s = 0.0;
    for (int k = g.KS; k <= g.KE; ++k) s += var[col + k - 1] * ld(CDZ + k - 1) * ld(CDX + i - 1) * ld(CDY + j - 1);
    part[(size_t)(i - g.IS) + (size_t)g.IMAX * (j - g.JS)] = s;
}
__global__ void k_tree_sum(const double *part, size_t n, double *out)
{
    __shared__ double sh[1024];
    double s = 0.0;
    for (size_t q = threadIdx.x; q < n; q += blockDim.x) s += part[q];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

void domain_sum(const Grid &g, const double *var, const double *CDX, const double *CDY, const double *CDZ,
                double *part, double *out, cudaStream_t st)
{
    dim3 b(128), gr((g.IMAX + 127) / 128, g.JMAX);
    k_col_sum<<<gr, b, 0, st>>>(g, var, CDX, CDY, CDZ, part);
    k_tree_sum<<<1, 1024, 0, st>>>(part, (size_t)g.IMAX * g.JMAX, out);
}

// ---- FP64 energy budget of dry air: the totals of ENGP, ENGK, ENGI and ENGT,
// scale-rm/src/atmos/mod_atmos_vars.F90:2097-2171, over the interior, each
// cell weighted by CDZ*CDX*CDY and summed in the order of k_col_sum.
// Cell-centre velocities as ATMOS_DIAGNOSTIC_CARTESC_get_vel
// (scalelib/src/atmosphere/common/scale_atmos_diagnostic_cartesC.F90:88-135) on
// flat terrain: W(KS) = MOMZ(KS)*0.5 (its flat-terrain value as written there),
// W(KE) = 0.5*MOMZ(KE-1)/DENS, U and V averaged from the faces.
// Temperature as ATMOS_THERMODYN_rhot2temp_pres (scale_atmos_thermodyn.F90:791-792)
// with Rtot = Rdry, CPtot/CVtot = CPdry/CVdry; QDRY = 1.
__global__ void k_energy_col(const Grid g, const double *DN, const double *MZ, const double *MX, const double *MY,
                             const double *RT, const double *CZ, const double *CDX, const double *CDY,
                             const double *CDZ, double *part)
{
    constexpr double Rdry = 287.04, CPdry = 1004.64, CVdry = CPdry - Rdry, PRE00 = 100000.0;
    const int i = g.IS + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t col = idx3(g, 1, i, j), ncol = (size_t)g.IMAX * g.JMAX;
    const size_t sI = g.KA, sJ = (size_t)g.KA * g.IA;
    double sp = 0.0, sk = 0.0, si = 0.0, st = 0.0;
    for (int k = g.KS; k <= g.KE; ++k) {
        const size_t c = col + k - 1;
        const double dn = DN[c];
        double w;
        if (k == g.KS) w = MZ[c] * 0.5;
        else if (k == g.KE) w = 0.5 * (MZ[c - 1]) / dn;
        else w = 0.5 * (MZ[c - 1] + MZ[c]) / dn;
        const double u = 0.5 * (MX[c - sI] + MX[c]) / dn;
        const double v = 0.5 * (MY[c - sJ] + MY[c]) / dn;
        const double pres = PRE00 * pow(RT[c] * Rdry / PRE00, CPdry / CVdry);
        const double temp = pres / (dn * Rdry);
        const double engp = dn * GRAV * ld(CZ + k - 1);
        const double engk = 0.5 * dn * (w * w + u * u + v * v);
        const double engi = dn * 1.0 * temp * CVdry;
        const double engt = engp + engk + engi;
        sp += engp * ld(CDZ + k - 1) * ld(CDX + i - 1) * ld(CDY + j - 1);
        sk += engk * ld(CDZ + k - 1) * ld(CDX + i - 1) * ld(CDY + j - 1);
        si += engi * ld(CDZ + k - 1) * ld(CDX + i - 1) * ld(CDY + j - 1);
        st += engt * ld(CDZ + k - 1) * ld(CDX + i - 1) * ld(CDY + j - 1);
    }
    const size_t q = (size_t)(i - g.IS) + (size_t)g.IMAX * (j - g.JS);
    part[q] = st;
    part[q + ncol] = sp;
    part[q + 2 * ncol] = sk;
    part[q + 3 * ncol] = si;
}

void energy_sum(const Grid &g, const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY,
                const double *RHOT, const double *CZ, const double *CDX, const double *CDY, const double *CDZ,
                double *part, double *out, cudaStream_t st)
{
    const size_t ncol = (size_t)g.IMAX * g.JMAX;
    dim3 b(128), gr((g.IMAX + 127) / 128, g.JMAX);
    k_energy_col<<<gr, b, 0, st>>>(g, DENS, MOMZ, MOMX, MOMY, RHOT, CZ, CDX, CDY, CDZ, part);
    for (int n = 0; n < 4; ++n) k_tree_sum<<<1, 1024, 0, st>>>(part + n * ncol, ncol, out + n);
}

// ---- short-step average of the mass flux for tracer advection
// (tstep_large_fvm_heve.F90:960-967 and :1012-1019), interior cells ----
__global__ void k_mflx_acc(const Grid g, double *av, const double *mflx, int nstep, int mode)
{
    const int i = g.IS + blockIdx.x * blockDim.y + threadIdx.y;
    const int j = g.JS + blockIdx.y;
    if (i > g.IE) return;
    const size_t N3 = n3(g), col = idx3(g, 1, i, j);
    for (int k = g.KS + threadIdx.x; k <= g.KE; k += 32)
        for (int n = 0; n < 3; ++n) {
            const size_t c = col + k - 1 + (size_t)n * N3;
            if (mode == 0) av[c] = av[c] + mflx[c];
            else ((double *)mflx)[c] = av[c] / nstep;
        }
}
void mflx_accumulate(const Grid &g, double *av, const double *mflx, cudaStream_t st)
{
    dim3 b(32, 4), gr((g.IMAX + 3) / 4, g.JMAX);
    k_mflx_acc<<<gr, b, 0, st>>>(g, av, mflx, 1, 0);
}
void mflx_average(const Grid &g, double *mflx, const double *av, int nstep, cudaStream_t st)
{
    dim3 b(32, 4), gr((g.IMAX + 3) / 4, g.JMAX);
    k_mflx_acc<<<gr, b, 0, st>>>(g, (double *)av, mflx, nstep, 1);
}

}  // namespace hevi
