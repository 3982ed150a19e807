// ATMOS_DYN_Tstep_short_fvm_hevi_b200_noalloc: one HEVI stage that allocates
// no device memory.
//
// Some callers cannot let a library allocate GPU memory:
//   - a host model that takes the whole device budget up front and then hands
//     out pieces of it; a cudaMalloc in the middle of a run would fail there,
//     or would upset its accounting;
//   - a caller that is not allowed to call scale_hevi_setup at all.
// For them this entry keeps its scratch in one fixed, statically sized device
// array (g_noalloc_scratch below). That array is part of the library's device
// image, so the CUDA runtime creates it when it loads the module, not this code.
//
// Usage notes:
//   - Every call looks up the array's device address with cudaGetSymbolAddress,
//     with the caller's device current (a recreated context gets its own copy
//     of the array, so no address is kept between calls). The first lookup on a
//     device can make the runtime load the module, so make the first call
//     before any stream capture. The entry synchronises its stream before it
//     returns, so it cannot itself be captured into a graph.
//   - The scratch is shared by every call on a device, so calls that overlap in
//     time (two host threads, or two streams in flight) race on it.
//   - Flat terrain only. The first call with a given set of metric arrays
//     (device, GSQRT, J13G, J23G, MAPF pointers) counts their non-flat values
//     on the device; a set found flat is remembered in host memory and later
//     calls with the same pointers skip the check. The cache assumes that the
//     contents of those arrays do not change between calls.
//   - The 4-point flux schemes (UD3, CD4, UD3KOREN1993, CD2) on a halo of 2.
//   - The scratch holds a 256-byte header (status word, terrain-check counter),
//     three per-level fields of the column solve (3*KA*IA*JA doubles) and the
//     1-D grid tables (7*KA + 4*IA + 4*JA doubles); at most
//     SCALE_HEVI_NOALLOC_SCRATCH_BYTES. Larger domains are rejected with
//     SCALE_HEVI_ERR_ARG.
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/scale_hevi.h"
#include "grid_coef.h"
#include "hevi_kernels.cuh"

namespace {

using namespace hevi;

constexpr size_t kScratchBytes = SCALE_HEVI_NOALLOC_SCRATCH_BYTES;
constexpr size_t kHeader = 256; // status word (offset 0) and terrain-check counter (offset 8)
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// metric sets (device, GSQRT, J13G, J23G, MAPF) already found flat; host memory
struct FlatKey {
    int dev;
    const void *p[4];
};
constexpr int kFlatSets = 64;
FlatKey g_flat[kFlatSets];
int g_nflat = 0;

int err(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    set_last_error(buf);
    return code;
}

#define NA_CU(call)                                                                                 \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return err(SCALE_HEVI_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

int scratch_for_current_device(unsigned char **out)
{
    void *p = nullptr;
    NA_CU(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    *out = static_cast<unsigned char *>(p);
    return SCALE_HEVI_OK;
}

bool known_flat(int dev, const void *const p[4])
{
    for (int q = 0; q < g_nflat; ++q)
        if (g_flat[q].dev == dev && !memcmp(g_flat[q].p, p, sizeof g_flat[q].p)) return true;
    return false;
}

void remember_flat(int dev, const void *const p[4])
{
    FlatKey &k = g_flat[g_nflat < kFlatSets ? g_nflat++ : (g_nflat - 1)]; // a full cache replaces its last entry
    k.dev = dev;
    memcpy(k.p, p, sizeof k.p);
}

int parse_scheme(const char *s, int *out)
{
    if (!s) return err(SCALE_HEVI_ERR_ARG, "flux scheme name is NULL");
    size_t n = strlen(s);
    while (n > 0 && s[n - 1] == ' ') --n; // Fortran blank padding
    const struct { const char *name; int id; } known[] = {{"UD3", UD3}, {"CD4", CD4}, {"UD3KOREN1993", KOREN}, {"CD2", CD2}};
    for (const auto &k : known)
        if (n == strlen(k.name) && strncmp(s, k.name, n) == 0) { *out = k.id; return SCALE_HEVI_OK; }
    return err(SCALE_HEVI_ERR_UNSUPPORTED,
               "flux scheme '%.*s' is not supported by the no-alloc entry (UD3, CD4, UD3KOREN1993, CD2 on a halo of 2)",
               (int)n, s);
}

// copy n doubles of a host vector into the device table (n may be 0)
int put_vec(double *dst, const double *src, int n, cudaStream_t st)
{
    if (n > 0) NA_CU(cudaMemcpyAsync(dst, src, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
    return SCALE_HEVI_OK;
}

}  // namespace

extern "C" int ATMOS_DYN_Tstep_short_fvm_hevi_b200_noalloc(const scale_hevi_index *idx, const char *flux_type,
                                                           void *stream, SCALE_HEVI_TSTEP_SHORT_ARGS)
{
    (void)PROG_RK; (void)PROG0; (void)PROG; (void)FLAG_FCT_MOMENTUM; (void)FLAG_FCT_T; (void)FLAG_FCT_ALONG_STREAM;
    (void)last; (void)PHI;
    if (!idx) return err(SCALE_HEVI_ERR_ARG, "index set is NULL");
    const scale_hevi_index &x = *idx;
    if (x.KHALO != 2 || x.IHALO != 2 || x.JHALO != 2) return err(SCALE_HEVI_ERR_UNSUPPORTED, "halo width must be 2");
    if (x.KA != x.KMAX + 2 * x.KHALO || x.IA != x.IMAX + 2 * x.IHALO || x.JA != x.JMAX + 2 * x.JHALO ||
        x.KS != 1 + x.KHALO || x.KE != x.KMAX + x.KHALO || x.IS != 1 + x.IHALO || x.IE != x.IMAX + x.IHALO ||
        x.JS != 1 + x.JHALO || x.JE != x.JMAX + x.JHALO)
        return err(SCALE_HEVI_ERR_ARG, "index set is inconsistent (KA=%d KMAX=%d IA=%d IMAX=%d JA=%d JMAX=%d)",
                   x.KA, x.KMAX, x.IA, x.IMAX, x.JA, x.JMAX);
    if (x.KMAX < 4 || x.KA > 260) return err(SCALE_HEVI_ERR_UNSUPPORTED, "KMAX must be in 4..256 (got %d)", x.KMAX);
    if (x.IMAX < 2 || x.JMAX < 2) return err(SCALE_HEVI_ERR_ARG, "IMAX and JMAX must be >= IHALO, JHALO");
    if ((x.IBLOCK > 0 && x.IBLOCK != x.IMAX) || (x.JBLOCK > 0 && x.JBLOCK != x.JMAX))
        return err(SCALE_HEVI_ERR_UNSUPPORTED, "only the default IBLOCK=IMAX, JBLOCK=JMAX blocking is supported");
    if ((BND_W && *BND_W) || (BND_E && *BND_E) || (BND_S && *BND_S) || (BND_N && *BND_N))
        return err(SCALE_HEVI_ERR_UNSUPPORTED, "non-periodic lateral boundaries (BND_*=.true.) are not supported");
    if (*divdmp_coef != 0.0 && !DDIV) return err(SCALE_HEVI_ERR_ARG, "divdmp_coef is nonzero but DDIV is NULL");
    if (!CDZ || !FDZ || !RCDZ || !RFDZ || !FDX || !RCDX || !RFDX || !FDY || !RCDY || !RFDY)
        return err(SCALE_HEVI_ERR_ARG, "a 1-D grid vector is NULL");
    int scheme = UD3;
    if (int rc = parse_scheme(flux_type, &scheme)) return rc;

    const int KA = x.KA, IA = x.IA, JA = x.JA;
    const size_t N3 = (size_t)KA * IA * JA;
    const size_t ntab = 7 * (size_t)KA + 4 * (size_t)IA + 4 * (size_t)JA;
    const size_t ncol = HEVI_COL_SCRATCH ? 3 * N3 : 0;
    const size_t need = kHeader + (ncol + ntab) * sizeof(double);
    if (need > kScratchBytes)
        return err(SCALE_HEVI_ERR_ARG,
                   "domain %dx%dx%d needs %zu bytes of scratch; the no-alloc entry holds at most %zu bytes",
                   x.IMAX, x.JMAX, x.KMAX, need, kScratchBytes);

    unsigned char *scr = nullptr;
    if (int rc = scratch_for_current_device(&scr)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned *status = reinterpret_cast<unsigned *>(scr);
    unsigned long long *count = reinterpret_cast<unsigned long long *>(scr + 8);
    double *colscr = reinterpret_cast<double *>(scr + kHeader);
    double *tab = colscr + ncol;

    // flat terrain only (GSQRT = 1, J13G = J23G = 0, MAPF = 1): the general-metric
    // stage of the other entries keeps 24 work fields, which this entry does not have
    NA_CU(cudaMemsetAsync(scr, 0, kHeader, st)); // status and counter start at zero
    int dev = 0;
    NA_CU(cudaGetDevice(&dev));
    const void *metrics[4] = {GSQRT, J13G, J23G, MAPF};
    if (!known_flat(dev, metrics)) {
        const size_t n7 = 7 * N3, nm = (size_t)IA * JA * 2 * 4;
        if (GSQRT) count_not_equal(GSQRT, n7, 1.0, count, st);
        if (J13G) count_not_equal(J13G, n7, 0.0, count, st);
        if (J23G) count_not_equal(J23G, n7, 0.0, count, st);
        if (MAPF) count_not_equal(MAPF, nm, 1.0, count, st);
        NA_CU(cudaGetLastError());
        unsigned long long bad = 0;
        NA_CU(cudaMemcpyAsync(&bad, count, sizeof bad, cudaMemcpyDeviceToHost, st));
        NA_CU(cudaStreamSynchronize(st));
        if (bad)
            return err(SCALE_HEVI_ERR_UNSUPPORTED,
                       "terrain-following metrics (%llu values of GSQRT/J13G/J23G/MAPF differ from flat terrain) are not supported",
                       bad);
        remember_flat(dev, metrics);
    }

    // 1-D tables: CDZ FDZ RCDZ RFDZ F2H1 F2H2 wdamp (KA each) | FDX RCDX RFDX (IA) | FDY RCDY RFDY (JA);
    // the face weights are built on this call's stack: a copy from pageable host
    // memory has read its source by the time cudaMemcpyAsync returns
    double f2h[2 * 260];
    build_f2h(KA, CDZ, f2h, f2h + KA);
    NA_CU(cudaMemsetAsync(tab, 0, ntab * sizeof(double), st)); // the unused last entries of FDZ/RFDZ/FDX/... stay 0
    double *z = tab, *xs = tab + 7 * (size_t)KA, *ys = xs + 4 * (size_t)IA;
    int rc = SCALE_HEVI_OK;
    if ((rc = put_vec(z, CDZ, KA, st)) || (rc = put_vec(z + KA, FDZ, KA - 1, st)) ||
        (rc = put_vec(z + 2 * KA, RCDZ, KA, st)) || (rc = put_vec(z + 3 * KA, RFDZ, KA - 1, st)) ||
        (rc = put_vec(z + 4 * KA, f2h, 2 * KA, st)) || (wdamp_coef && (rc = put_vec(z + 6 * KA, wdamp_coef, KA, st))) ||
        (rc = put_vec(xs, FDX, IA - 1, st)) || (rc = put_vec(xs + IA, RCDX, IA, st)) ||
        (rc = put_vec(xs + 2 * IA, RFDX, IA - 1, st)) || (rc = put_vec(ys, FDY, JA - 1, st)) ||
        (rc = put_vec(ys + JA, RCDY, JA, st)) || (rc = put_vec(ys + 2 * JA, RFDY, JA - 1, st)))
        return rc;

    Grid g{};
    g.KA = KA; g.IA = IA; g.JA = JA;
    g.KS = x.KS; g.KE = x.KE; g.IS = x.IS; g.IE = x.IE; g.JS = x.JS; g.JE = x.JE;
    g.KMAX = x.KMAX; g.IMAX = x.IMAX; g.JMAX = x.JMAX; g.IHALO = x.IHALO; g.JHALO = x.JHALO;
    g.IEH = x.IE; g.JEH = x.JE; // BND_E = BND_N = .false.
    g.CDZ = z; g.FDZ = z + KA; g.RCDZ = z + 2 * KA; g.RFDZ = z + 3 * KA; g.F2H1 = z + 4 * KA; g.F2H2 = z + 5 * KA;
    g.FDX = xs; g.RCDX = xs + IA; g.RFDX = xs + 2 * IA;
    g.FDY = ys; g.RCDY = ys + JA; g.RFDY = ys + 2 * JA;
    g.stride = (size_t)KA * IA * JA;

    StageArgs a{};
    a.DENS_RK = DENS_RK; a.MOMZ_RK = MOMZ_RK; a.MOMX_RK = MOMX_RK; a.MOMY_RK = MOMY_RK; a.RHOT_RK = RHOT_RK;
    a.mflx = mflx_hi; a.tflx = tflx_hi;
    a.DENS0 = DENS0; a.MOMZ0 = MOMZ0; a.MOMX0 = MOMX0; a.MOMY0 = MOMY0; a.RHOT0 = RHOT0;
    a.DENS = DENS; a.MOMZ = MOMZ; a.MOMX = MOMX; a.MOMY = MOMY; a.RHOT = RHOT;
    a.DENS_t = DENS_t; a.MOMZ_t = MOMZ_t; a.MOMX_t = MOMX_t; a.MOMY_t = MOMY_t; a.RHOT_t = RHOT_t;
    a.DPRES0 = DPRES0; a.RT2P = RT2P; a.CORIOLI = CORIOLI; a.num_diff = num_diff;
    a.wdamp = z + 6 * KA; a.DDIV = DDIV; a.REF_dens = REF_dens; a.REF_rhot = REF_rhot;
    a.divdmp_coef = *divdmp_coef; a.J33G = *J33G; a.dtrk = *dtrk;
    a.rk_mode = RK_PLAIN; a.acc = nullptr; a.facc = nullptr; a.status = status;
    a.colscr = HEVI_COL_SCRATCH ? colscr : nullptr;

    NA_CU(launch_hevi_stage(g, Members{}, a, scheme, StageShape{}, st));
    unsigned flags = 0;
    NA_CU(cudaMemcpyAsync(&flags, status, sizeof flags, cudaMemcpyDeviceToHost, st));
    NA_CU(cudaStreamSynchronize(st));
    if (flags & ST_NONFINITE) return err(SCALE_HEVI_ERR_NONFINITE, "a prognostic output became NaN or Inf");
    return SCALE_HEVI_OK;
}
