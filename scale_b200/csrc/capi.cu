// C-ABI of libscale_hevi.so: library state, argument checks, host<->device
// staging of the host-array entries, and the RK4 / tracer-RK3 / large-step
// drivers that sequence the device kernels. Declarations and the reference
// procedure each entry replaces are in include/scale_hevi.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "../../include/scale_hevi.h"
#include "adjoint.cuh"
#include "grid_coef.h"
#include "hevi_kernels.cuh"


using namespace hevi;

namespace {

struct LargeHooks;

struct Ctx {
    bool ready = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    scale_hevi_index idx{};
    Grid g{};
    int scheme = UD3, scheme_tracer = UD3;
    int short_type = 0;  // the registered short step of the RK4 and large-step entries: 0 HEVI, 1 HEVE
    int tinteg_type = 0; // the short integrator of the large step: 0 RK4, 1 RK3 (Heun), 2 RK3WS2002
    scale_hevi_halo_fn halo_fn = nullptr; // lateral halo exchange of a decomposed domain (null: periodic)
    void *halo_user = nullptr;
    size_t N3 = 0;   // points of one 3-D field (all members)
    // ensemble members sharing the pooled arrays (one entry for a single domain)
    std::vector<MemberGeom> members;
    std::vector<scale_hevi_index> member_idx;
    size_t N2 = 0;                   // points of one 2-D field (all members)
    int ZT = 0, XT = 0, YT = 0;      // lengths of the pooled z/x/y vectors
    StageShape shape[2];             // stage launch shape, FP64 [0] and mixed [1] path (tuned or set)
    int autotune = 0;                // tune the shape at the next short-step call (per path)
    bool tuned[2] = {false, false};
    std::string tune_text;           // JSON record of the last tuning
    long long launches = 0;
    long long h2d_bytes = 0, d2h_bytes = 0; // host<->device copies of the host-array entries
    // 1-D tables on the device: CDZ FDZ RCDZ RFDZ F2H1 F2H2 wdamp (KA each),
    // FDX RCDX RFDX CDX (IA), FDY RCDY RFDY CDY (JA)
    double *d_tab = nullptr;
    std::vector<double> h_tab;
    bool tab_valid = false;
    double *d_wdamp = nullptr;
    // numerical filter tables
    double *d_nd = nullptr;
    std::vector<double> nd_key;
    NdCoef ndc{};
    // scratch
    double *rk[2] = {nullptr, nullptr}; // 5*N3 each
    double *acc = nullptr;          // 5*N3
    double *facc = nullptr;         // 6*N3
    double *colscr = nullptr;       // 4*N3: Sr, St, tZ (fused and tiled stage), PT (tiled stage)
    double *colC = nullptr;         // 2*N3: the column problem's right-hand side, then f, and e (tiled stage)
    double *phi = nullptr;          // numerical filter: 5*N3 (allocated on first use)
    double *ndw = nullptr;          // numerical filter at ND_ORDER > 1: 2 x 15*N3 work (on first use)
    // mixed-precision path (allocated on first use): flux RK sums, column-solve
    // sources and the filtered quantities in FP32
    float *facc_f = nullptr, *colscr_f = nullptr, *phi_f = nullptr;
    float *tr_f = nullptr;          // mixed tracer limiter: phi_lo, anti(3), rjp, rjm = 6*N3 (on first use)
    double *tr = nullptr;           // tracer: RK1, RK2, phi_lo, anti(3), rjp, rjm = 8*N3
    double *lg = nullptr;           // large step: DENS00, RT2P, DPRES0, REF_rhot, mflx_av(3), DDIV = 8*N3
    double *sum_part = nullptr, *sum_out = nullptr;
    double *eng_part = nullptr;     // energy budget: 4*IMAX*JMAX column sums + 4 totals (on first use)
    // terrain-following metrics of the current call (the general-metric stage runs when set)
    bool terrain = false;
    Metrics tm{};
    TerrainWork tw{};
    double *tw_buf = nullptr; // TERRAIN_WORK_FIELDS * N3 (allocated on first use)
    std::vector<std::vector<const void *>> nonflat; // metric sets already seen to be non-flat
    unsigned *status = nullptr;
    unsigned long long *count = nullptr;
    // metric check cache (pointer tuples already verified flat)
    std::vector<std::vector<const void *>> flat_ok;
    // staging buffers of the host-array entries
    std::map<std::string, std::pair<double *, size_t>> stage;
    // host-array large step: a second stream carries the host<->device copies so
    // that they overlap the kernels on `stream` (created on first use)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_ev[6] = {};
    LargeHooks *large_hooks = nullptr; // set only inside the host-array large step
    // section timers (scale_hevi_profile): event pairs recorded around launches
    bool prof_on = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<std::pair<std::string, size_t>> prof_marks; // name, index of the start event
    std::string prof_text;
    // CUDA graph of a captured call sequence (scale_hevi_capture_*)
    cudaGraphExec_t graph_exec = nullptr;
    bool capturing = false;
    long long capture_from = 0, graph_launches = 0; // kernel launches recorded in the graph
    // differentiated short step (scale_hevi_adjoint_setup)
    bool ad_ready = false;
    ad::Model adm{};
    double *ad_scratch = nullptr, *ad_zero = nullptr, *ad_nd = nullptr, *ad_flx = nullptr;
    std::vector<double> ad_vec[12]; // CDZ CDX CDY FDZ FDX FDY RCDZ RCDX RCDY RFDZ RFDX RFDY
    std::vector<double> ad_wdamp;
    double ad_ndcoef = 0.0, ad_sfc = 1.0;
    // persistent short step: the barrier and work counters, the barrier time
    // limit and the extra arrivals a test of that limit asks for
    unsigned *pbar = nullptr;
    double pwait_s = 2.0;
    unsigned pextra = 0;
    int pgrid = 0; // CTAs of the last persistent launch
    bool nd_tiled = true; // the filter's tiled form where it applies (scale_hevi_numfilter_form)
    bool fct_fused = true; // the limiter's fused form where it applies (scale_hevi_tracer_fct_form)
};

Ctx C;
std::string g_err;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CU(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(SCALE_HEVI_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
#define CK(expr)                      \
    do {                              \
        int rc_ = (expr);             \
        if (rc_ != SCALE_HEVI_OK) return rc_; \
    } while (0)

int need_setup()
{
    if (!C.ready) return fail(SCALE_HEVI_ERR_NOT_SETUP, "scale_hevi_setup() has not been called");
    return SCALE_HEVI_OK;
}

Members mem() { return Members{C.members.data(), (int)C.members.size()}; }

// entries that only a single domain supports
int need_single(const char *what)
{
    CK(need_setup());
    if (C.members.size() > 1)
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "%s is not available for an ensemble (%zu members)", what,
                    C.members.size());
    return SCALE_HEVI_OK;
}

// Record a CUDA event pair around the launches of one section (the library's
// counterpart of PROF_rapstart/PROF_rapend, scalelib/src/common/scale_prof.F90:156,209).
template <class F>
int timed(const char *name, F &&launch)
{
    if (!C.prof_on) return launch();
    while (C.ev_pool.size() < C.ev_used + 2) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return fail(SCALE_HEVI_ERR_CUDA, "cudaEventCreate failed");
        C.ev_pool.push_back(e);
    }
    const size_t i0 = C.ev_used;
    C.ev_used += 2;
    cudaEventRecord(C.ev_pool[i0], C.stream);
    int rc = launch();
    cudaEventRecord(C.ev_pool[i0 + 1], C.stream);
    C.prof_marks.emplace_back(name, i0);
    return rc;
}

int dalloc(double **p, size_t n)
{
    if (cudaMalloc((void **)p, n * sizeof(double)) != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(SCALE_HEVI_ERR_ALLOC, "cudaMalloc of %zu doubles failed", n);
    }
    return SCALE_HEVI_OK;
}

int falloc(float **p, size_t n)
{
    if (cudaMalloc((void **)p, n * sizeof(float)) != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(SCALE_HEVI_ERR_ALLOC, "cudaMalloc of %zu floats failed", n);
    }
    return SCALE_HEVI_OK;
}

void free_all()
{
    double *bufs[] = {C.eng_part, C.phi, C.ndw, C.colscr, C.colC, C.d_tab, C.d_nd, C.rk[0], C.rk[1], C.acc, C.facc, C.tr, C.lg, C.sum_part, C.sum_out,
                      C.tw_buf};
    for (double *b : bufs) if (b) cudaFree(b);
    for (auto &kv : C.stage) cudaFree(kv.second.first);
    for (float *b : {C.facc_f, C.colscr_f, C.phi_f, C.tr_f}) if (b) cudaFree(b);
    for (double *b : {C.ad_scratch, C.ad_zero, C.ad_nd, C.ad_flx}) if (b) cudaFree(b);
    if (C.status) cudaFree(C.status);
    if (C.count) cudaFree(C.count);
    if (C.pbar) cudaFree(C.pbar);
    for (cudaEvent_t e : C.ev_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : C.copy_ev) if (e) cudaEventDestroy(e);
    if (C.copy_stream) cudaStreamDestroy(C.copy_stream);
    if (C.capturing) {
        cudaGraph_t g = nullptr;
        if (cudaStreamEndCapture(C.stream, &g) == cudaSuccess && g) cudaGraphDestroy(g);
        cudaGetLastError();
    }
    if (C.graph_exec) cudaGraphExecDestroy(C.graph_exec);
    if (C.stream) cudaStreamDestroy(C.stream);
    C = Ctx();
}

int parse_scheme(const char *s, int *out)
{
    if (!s) return fail(SCALE_HEVI_ERR_ARG, "flux scheme name is NULL");
    std::string n(s);
    while (!n.empty() && n.back() == ' ') n.pop_back(); // Fortran blank padding
    if (n == "UD3") { *out = UD3; return SCALE_HEVI_OK; }
    if (n == "CD4") { *out = CD4; return SCALE_HEVI_OK; }
    if (n == "UD3KOREN1993") { *out = KOREN; return SCALE_HEVI_OK; }
    if (n == "CD2") { *out = CD2; return SCALE_HEVI_OK; }
    if (n == "UD5") { *out = UD5; return SCALE_HEVI_OK; }
    if (n == "CD6") { *out = CD6; return SCALE_HEVI_OK; }
    return fail(SCALE_HEVI_ERR_UNSUPPORTED,
                "flux scheme '%s' is not supported (UD3, CD4, UD3KOREN1993, CD2, UD5, CD6)", n.c_str());
}

// host-array entries: a device buffer per argument role, grown on demand
int stage_buf(const char *name, size_t n, double **out)
{
    auto &e = C.stage[name];
    if (e.second < n) {
        if (e.first) cudaFree(e.first);
        e.first = nullptr;
        e.second = 0;
        CK(dalloc(&e.first, n));
        e.second = n;
    }
    *out = e.first;
    return SCALE_HEVI_OK;
}
// copies on `st`, or on the library stream when st is null
int h2d(const char *name, const double *h, size_t n, double **d, cudaStream_t st = nullptr)
{
    CK(stage_buf(name, n, d));
    CU(cudaMemcpyAsync(*d, h, n * sizeof(double), cudaMemcpyHostToDevice, st ? st : C.stream));
    C.h2d_bytes += (long long)(n * sizeof(double));
    return SCALE_HEVI_OK;
}
int d2h(double *h, const double *d, size_t n, cudaStream_t st = nullptr)
{
    CU(cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, st ? st : C.stream));
    C.d2h_bytes += (long long)(n * sizeof(double));
    return SCALE_HEVI_OK;
}

int check_bnd(const int *W, const int *E, const int *S, const int *N)
{
    if ((W && *W) || (E && *E) || (S && *S) || (N && *N))
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "non-periodic lateral boundaries (BND_*=.true.) are not supported");
    return SCALE_HEVI_OK;
}

// Whether the metric arrays are those of flat terrain (GSQRT == 1, J13G ==
// J23G == 0, MAPF == 1), counted once per distinct set of arrays.
int metrics_flat(const double *GSQRT, const double *J13G, const double *J23G, const double *MAPF, bool on_device,
                 bool *flat, unsigned long long *nbad = nullptr)
{
    std::vector<const void *> key = {GSQRT, J13G, J23G, MAPF, (const void *)(size_t)on_device};
    for (auto &k : C.flat_ok) if (k == key) { *flat = true; return SCALE_HEVI_OK; }
    for (auto &k : C.nonflat) if (k == key) { *flat = false; return SCALE_HEVI_OK; }
    const size_t n7 = 7 * C.N3, nm = C.N2 * 2 * 4;
    unsigned long long bad = 0;
    if (on_device) {
        CU(cudaMemsetAsync(C.count, 0, sizeof(unsigned long long), C.stream));
        if (GSQRT) { count_not_equal(GSQRT, n7, 1.0, C.count, C.stream); ++C.launches; }
        if (J13G) { count_not_equal(J13G, n7, 0.0, C.count, C.stream); ++C.launches; }
        if (J23G) { count_not_equal(J23G, n7, 0.0, C.count, C.stream); ++C.launches; }
        if (MAPF) { count_not_equal(MAPF, nm, 1.0, C.count, C.stream); ++C.launches; }
        CU(cudaMemcpyAsync(&bad, C.count, sizeof bad, cudaMemcpyDeviceToHost, C.stream));
        CU(cudaStreamSynchronize(C.stream));
    } else {
        for (size_t q = 0; GSQRT && q < n7; ++q) bad += GSQRT[q] != 1.0;
        for (size_t q = 0; J13G && q < n7; ++q) bad += J13G[q] != 0.0;
        for (size_t q = 0; J23G && q < n7; ++q) bad += J23G[q] != 0.0;
        for (size_t q = 0; MAPF && q < nm; ++q) bad += MAPF[q] != 1.0;
    }
    *flat = bad == 0;
    if (nbad) *nbad = bad;
    (*flat ? C.flat_ok : C.nonflat).push_back(key);
    return SCALE_HEVI_OK;
}

// Entries without a general-metric path: flat terrain only.
int check_flat(const double *GSQRT, const double *J13G, const double *J23G, const double *MAPF, bool on_device)
{
    C.terrain = false;
    bool flat = false;
    unsigned long long bad = 0;
    CK(metrics_flat(GSQRT, J13G, J23G, MAPF, on_device, &flat, &bad));
    if (!flat)
        return fail(SCALE_HEVI_ERR_UNSUPPORTED,
                    "terrain-following metrics (GSQRT/J13G/J23G/MAPF of non-flat terrain) are not supported by this entry");
    return SCALE_HEVI_OK;
}

// Entries of the HEVI stage and the short integrators: flat metrics select the
// fused kernels, any others the general-metric stage (FP64, one domain), which
// also reads PHI. Host arrays are copied to the device first.
int use_metrics(const double *GSQRT, const double *J13G, const double *J23G, const double *MAPF, const double *PHI,
                bool on_device)
{
    C.terrain = false;
    bool flat = false;
    CK(metrics_flat(GSQRT, J13G, J23G, MAPF, on_device, &flat));
    if (flat) return SCALE_HEVI_OK;
    if (C.members.size() > 1)
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "terrain-following metrics are supported for a single domain");
    if (!GSQRT || !J13G || !J23G || !MAPF || !PHI)
        return fail(SCALE_HEVI_ERR_ARG, "terrain-following metrics need GSQRT, J13G, J23G, MAPF and PHI");
    if (on_device) {
        C.tm = Metrics{GSQRT, J13G, J23G, MAPF, PHI};
    } else {
        double *g7, *j13, *j23, *mp, *ph;
        CK(h2d("GSQRT", GSQRT, 7 * C.N3, &g7));
        CK(h2d("J13G", J13G, 7 * C.N3, &j13));
        CK(h2d("J23G", J23G, 7 * C.N3, &j23));
        CK(h2d("MAPF", MAPF, C.N2 * 2 * 4, &mp));
        CK(h2d("PHI", PHI, C.N3, &ph));
        C.tm = Metrics{g7, j13, j23, mp, ph};
    }
    if (!C.tw_buf) {
        CK(dalloc(&C.tw_buf, (size_t)TERRAIN_WORK_FIELDS * C.N3));
        double *q = C.tw_buf;
        double **f[TERRAIN_WORK_FIELDS] = {&C.tw.POTT, &C.tw.DPRES, &C.tw.qZ, &C.tw.qX, &C.tw.qY, &C.tw.qJ13, &C.tw.qJ23,
                                           &C.tw.Sr, &C.tw.Sw, &C.tw.St, &C.tw.mZ, &C.tw.mX, &C.tw.mY, &C.tw.tZ,
                                           &C.tw.tX, &C.tw.tY, &C.tw.A, &C.tw.PT, &C.tw.F1, &C.tw.F2, &C.tw.F3,
                                           &C.tw.C, &C.tw.e, &C.tw.f};
        for (int q2 = 0; q2 < TERRAIN_WORK_FIELDS; ++q2) *f[q2] = q + (size_t)q2 * C.N3;
    }
    C.terrain = true;
    return SCALE_HEVI_OK;
}

// Upload the 1-D grid vectors (host arrays) when they change and point the
// Grid's table pointers at the device copies.
int prepare_tables(const double *CDZ, const double *FDZ, const double *RCDZ, const double *RFDZ,
                   const double *FDX, const double *RCDX, const double *RFDX,
                   const double *FDY, const double *RCDY, const double *RFDY, const double *wdamp,
                   const double *CDX, const double *CDY)
{
    // pooled layout: table t of the z vectors at t*ZT, member m's values at z0
    // of it (KA slots; FDZ/RFDZ use KA-1); likewise x (IA) and y (JA)
    const size_t ZT = C.ZT, XT = C.XT, YT = C.YT;
    std::vector<double> h(7 * ZT + 4 * XT + 4 * YT, 0.0);
    double *z = h.data(), *x = z + 7 * ZT, *y = x + 4 * XT;
    if (!CDZ || !FDZ || !RCDZ || !RFDZ || !FDX || !RCDX || !RFDX || !FDY || !RCDY || !RFDY)
        return fail(SCALE_HEVI_ERR_ARG, "a 1-D grid vector is NULL");
    const int H = C.g.IHALO; // lateral halo of every member
    for (const MemberGeom &m : C.members) {
        const int KA = m.KMAX + 4, IA = m.IMAX + 2 * H, JA = m.JMAX + 2 * H, z0 = m.z0, x0 = m.x0, y0 = m.y0;
        std::memcpy(z + z0, CDZ + z0, KA * sizeof(double));
        std::memcpy(z + ZT + z0, FDZ + z0, (KA - 1) * sizeof(double));
        std::memcpy(z + 2 * ZT + z0, RCDZ + z0, KA * sizeof(double));
        std::memcpy(z + 3 * ZT + z0, RFDZ + z0, (KA - 1) * sizeof(double));
        build_f2h(KA, CDZ + z0, z + 4 * ZT + z0, z + 5 * ZT + z0);
        if (wdamp) std::memcpy(z + 6 * ZT + z0, wdamp + z0, KA * sizeof(double));
        std::memcpy(x + x0, FDX + x0, (IA - 1) * sizeof(double));
        std::memcpy(x + XT + x0, RCDX + x0, IA * sizeof(double));
        std::memcpy(x + 2 * XT + x0, RFDX + x0, (IA - 1) * sizeof(double));
        if (CDX) std::memcpy(x + 3 * XT + x0, CDX + x0, IA * sizeof(double));
        std::memcpy(y + y0, FDY + y0, (JA - 1) * sizeof(double));
        std::memcpy(y + YT + y0, RCDY + y0, JA * sizeof(double));
        std::memcpy(y + 2 * YT + y0, RFDY + y0, (JA - 1) * sizeof(double));
        if (CDY) std::memcpy(y + 3 * YT + y0, CDY + y0, JA * sizeof(double));
    }
    if (!C.tab_valid || h != C.h_tab) {
        CU(cudaMemcpyAsync(C.d_tab, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, C.stream));
        CU(cudaStreamSynchronize(C.stream)); // the host vector is freed on return
        C.h_tab.swap(h);
        C.tab_valid = true;
    }
    double *dz = C.d_tab, *dx = dz + 7 * ZT, *dy = dx + 4 * XT;
    C.g.CDZ = dz; C.g.FDZ = dz + ZT; C.g.RCDZ = dz + 2 * ZT; C.g.RFDZ = dz + 3 * ZT;
    C.g.F2H1 = dz + 4 * ZT; C.g.F2H2 = dz + 5 * ZT; C.d_wdamp = dz + 6 * ZT;
    C.g.FDX = dx; C.g.RCDX = dx + XT; C.g.RFDX = dx + 2 * XT;
    C.g.FDY = dy; C.g.RCDY = dy + YT; C.g.RFDY = dy + 2 * YT;
    return SCALE_HEVI_OK;
}

int prepare_nd(const double *CDZ, const double *CDX, const double *CDY, const double *FDZ, const double *FDX,
               const double *FDY, double DT, double ND_COEF, int ND_ORDER, double SFC)
{
    // calc_diff3 of the w-point quantity mirrors levels KS+2 and KS+3 into KS-1
    // and KS-2 (scale_atmos_dyn_common.F90:1695-1696) before it writes them when
    // KMAX < 6, so the result there would depend on what the work array held;
    // calc_diff4 (ND_ORDER > 1) reads those levels
    if (ND_ORDER > 1)
        for (const MemberGeom &m : C.members)
            if (m.KMAX < 6)
                return fail(SCALE_HEVI_ERR_UNSUPPORTED, "ND_ORDER > 1 needs KMAX >= 6 (got %d)", m.KMAX);
    const size_t ZT = C.ZT, XT = C.XT, YT = C.YT;
    std::vector<double> key;
    key.insert(key.end(), CDZ, CDZ + ZT); key.insert(key.end(), FDZ, FDZ + ZT - 1);
    key.insert(key.end(), CDX, CDX + XT); key.insert(key.end(), FDX, FDX + XT - 1);
    key.insert(key.end(), CDY, CDY + YT); key.insert(key.end(), FDY, FDY + YT - 1);
    key.push_back(DT); key.push_back(ND_COEF); key.push_back((double)ND_ORDER);
    // pooled layout: CNZ3 (6 values per level), CNX3, CNY3, then cdz fdz (ZT
    // each), cdx fdx (XT), cdy fdy (YT); member m at 6*z0 / z0 / ...
    const size_t oX3 = 6 * ZT, oY3 = oX3 + 6 * XT, ocdz = oY3 + 6 * YT, ofdz = ocdz + ZT, ocdx = ofdz + ZT,
                 ofdx = ocdx + XT, ocdy = ofdx + XT, ofdy = ocdy + YT;
    // then the calc_diff4 coefficients CNZ4, CNX4, CNY4 (10 values per level or point)
    const size_t oZ4 = ofdy + YT, oX4 = oZ4 + 10 * ZT, oY4 = oX4 + 10 * XT, oend = oY4 + 10 * YT;
    if (key != C.nd_key) {
        std::vector<double> h(oend, 0.0);
        const int H = C.g.IHALO; // lateral halo of every member
        for (const MemberGeom &m : C.members) {
            const int KA = m.KMAX + 4, IA = m.IMAX + 2 * H, JA = m.JMAX + 2 * H, z0 = m.z0, x0 = m.x0, y0 = m.y0;
            NdGrid gr{KA, IA, JA, 3, m.KMAX + 2, H + 1, m.IMAX + H, H + 1, m.JMAX + H,
                      CDZ + z0, FDZ + z0, CDX + x0, FDX + x0, CDY + y0, FDY + y0};
            NdTables t;
            build_nd_tables(gr, DT, ND_COEF, ND_ORDER, t);
            auto put = [&](const std::vector<double> &v, size_t at) { std::copy(v.begin(), v.end(), h.begin() + at); };
            put(t.CNZ3, 6 * (size_t)z0); put(t.CNX3, oX3 + 6 * (size_t)x0); put(t.CNY3, oY3 + 6 * (size_t)y0);
            put(t.cdz, ocdz + z0); put(t.fdz, ofdz + z0); put(t.cdx, ocdx + x0); put(t.fdx, ofdx + x0);
            put(t.cdy, ocdy + y0); put(t.fdy, ofdy + y0);
            put(t.CNZ4, oZ4 + 10 * (size_t)z0); put(t.CNX4, oX4 + 10 * (size_t)x0); put(t.CNY4, oY4 + 10 * (size_t)y0);
        }
        CU(cudaMemcpyAsync(C.d_nd, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, C.stream));
        CU(cudaStreamSynchronize(C.stream));
        C.nd_key.swap(key);
    }
    const double *p = C.d_nd;
    C.ndc.CNZ3 = p; C.ndc.CNX3 = p + oX3; C.ndc.CNY3 = p + oY3;
    C.ndc.cdz = p + ocdz; C.ndc.fdz = p + ofdz; C.ndc.cdx = p + ocdx; C.ndc.fdx = p + ofdx;
    C.ndc.cdy = p + ocdy; C.ndc.fdy = p + ofdy;
    C.ndc.sfc = SFC;
    C.ndc.CNZ4 = p + oZ4; C.ndc.CNX4 = p + oX4; C.ndc.CNY4 = p + oY4;
    C.ndc.order = ND_ORDER;
    return SCALE_HEVI_OK;
}

template <typename T>
int halo(T *const *f, int n)
{
    if (C.halo_fn) {
        // the exchange of a decomposed domain, with the library's stream idle
        CU(cudaStreamSynchronize(C.stream));
        std::vector<void *> p(f, f + n);
        const int rc = C.halo_fn(p.data(), n, (int)sizeof(T), C.halo_user);
        if (rc) return fail(SCALE_HEVI_ERR_CUDA, "the halo exchange hook returned %d", rc);
        return SCALE_HEVI_OK;
    }
    C.launches += (n + 15) / 16;
    return timed("halo", [&] {
        periodic_halo(C.g, mem(), f, n, C.stream);
        return SCALE_HEVI_OK;
    });
}

// the halo fill that launch_tracer_stage and launch_numfilter_high call between
// their kernels while a halo exchange hook is set; ctx: the int that receives
// halo()'s status
static int hook_fill(void *ctx, void *const *f, int n, int elem)
{
    const int rc = elem == (int)sizeof(double) ? halo(reinterpret_cast<double *const *>(f), n)
                                               : halo(reinterpret_cast<float *const *>(f), n);
    *static_cast<int *>(ctx) = rc;
    return rc;
}

// ---- one stage ---------------------------------------------------------------
// F: type of the flux-like arrays (double: plain path, float: mixed precision)
template <typename F>
struct StageInT {
    const double *DENS0, *MOMZ0, *MOMX0, *MOMY0, *RHOT0;
    const double *DENS, *MOMZ, *MOMX, *MOMY, *RHOT;
    const F *DENS_t, *MOMZ_t, *MOMX_t, *MOMY_t, *RHOT_t;
    const double *DPRES0, *RT2P, *CORIOLI;
    const F *num_diff, *DDIV;
    const double *REF_dens, *REF_rhot;
    double divdmp, J33G;
};
using StageIn = StageInT<double>;

// the flux RK sums and the column-solve scratch of each precision
template <typename F> F *facc_buf();
template <typename F> F *colscr_buf();
template <> double *facc_buf<double>() { return C.facc; }
template <> float *facc_buf<float>() { return C.facc_f; }
template <> double *colscr_buf<double>() { return C.colscr; }
template <> float *colscr_buf<float>() { return C.colscr_f; }

template <typename F>
StageArgsT<F> stage_args(const StageInT<F> &in, double *const out[5], F *mflx, F *tflx, double dtrk, int mode)
{
    StageArgsT<F> a{};
    a.DENS_RK = out[0]; a.MOMZ_RK = out[1]; a.MOMX_RK = out[2]; a.MOMY_RK = out[3]; a.RHOT_RK = out[4];
    a.mflx = mflx; a.tflx = tflx;
    a.DENS0 = in.DENS0; a.MOMZ0 = in.MOMZ0; a.MOMX0 = in.MOMX0; a.MOMY0 = in.MOMY0; a.RHOT0 = in.RHOT0;
    a.DENS = in.DENS; a.MOMZ = in.MOMZ; a.MOMX = in.MOMX; a.MOMY = in.MOMY; a.RHOT = in.RHOT;
    a.DENS_t = in.DENS_t; a.MOMZ_t = in.MOMZ_t; a.MOMX_t = in.MOMX_t; a.MOMY_t = in.MOMY_t; a.RHOT_t = in.RHOT_t;
    a.DPRES0 = in.DPRES0; a.RT2P = in.RT2P; a.CORIOLI = in.CORIOLI; a.num_diff = in.num_diff;
    a.wdamp = C.d_wdamp; a.DDIV = in.DDIV; a.REF_dens = in.REF_dens; a.REF_rhot = in.REF_rhot;
    a.divdmp_coef = in.divdmp; a.J33G = in.J33G; a.dtrk = dtrk;
    a.rk_mode = mode; a.acc = mode == RK_HEUN3 ? C.rk[0] : C.acc; a.facc = facc_buf<F>(); a.status = C.status;
    a.colscr = colscr_buf<F>();
    a.colC = C.colC;
    return a;
}

// Stage-shape autotuner: times the tiled stage (where it applies) and every
// compiled tile width of the fused kernel, each at three raster heights, on
// the caller's own inputs (one plain stage whose outputs go to the library's
// scratch: the RK buffer, the flux RK sums, the column scratch; nothing the
// caller holds is written) and keeps the fastest for this path.
template <typename F>
int autotune_stage(const StageInT<F> &in, double dtrk)
{
    const int p = sizeof(F) == sizeof(double) ? 0 : 1;
    double *out[5];
    for (int v = 0; v < 5; ++v) out[v] = C.rk[0] + (size_t)v * C.N3;
    F *fs = facc_buf<F>();
    const StageArgsT<F> a = stage_args(in, out, fs, fs + 3 * C.N3, dtrk, RK_PLAIN);
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    constexpr int RASTERS[3] = {4, 16, 64}, REPS = 3;
    StageShape best{};
    float best_ms = 1e30f;
    std::string rows;
    int rc = SCALE_HEVI_OK;
    constexpr int FORMS[4] = {0, STAGE_TILE_XS[0], STAGE_TILE_XS[1], STAGE_TILE_XS[2]};
    for (int tx : FORMS) {
        for (int r : RASTERS) {
            const StageShape sh{tx, r};
            int nl = 1;
            bool tiled = false;
            cudaError_t e = launch_hevi_stage(C.g, mem(), a, C.scheme, sh, C.stream, &nl, &tiled); // warm-up
            if (e == cudaSuccess && tx == 0 && !tiled) break; // the tiled stage does not apply here
            cudaEventRecord(e0, C.stream);
            for (int q = 0; q < REPS && e == cudaSuccess; ++q) e = launch_hevi_stage(C.g, mem(), a, C.scheme, sh, C.stream);
            cudaEventRecord(e1, C.stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) {
                rc = fail(SCALE_HEVI_ERR_CUDA, "stage autotune (tile %d, raster %d): %s", tx, r, cudaGetErrorString(e));
                break;
            }
            ms /= REPS;
            C.launches += (long long)nl * (1 + REPS);
            char buf[96];
            snprintf(buf, sizeof buf, "%s[%d, %d, %.4f]", rows.empty() ? "" : ", ", tx, r, ms);
            rows += buf;
            if (ms < best_ms) { best_ms = ms; best = sh; }
        }
        if (rc != SCALE_HEVI_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != SCALE_HEVI_OK) return rc;
    C.shape[p] = best;
    C.tuned[p] = true;
    char head[160];
    snprintf(head, sizeof head, "{\"path\": \"%s\", \"chosen\": [%d, %d, %.4f], \"candidates\": [",
             p ? "mixed" : "fp64", best.tile_x, best.raster, best_ms);
    C.tune_text = std::string(head) + rows + "]}";
    return SCALE_HEVI_OK;
}

template <typename F>
// kind: 0 HEVI, 1 HEVE, -1 the registered short step (scale_hevi_short_type)
int run_stage(const StageInT<F> &in, double *const out[5], F *mflx, F *tflx, double dtrk, int mode, int kind = -1)
{
    if (in.divdmp != 0.0 && !in.DDIV) return fail(SCALE_HEVI_ERR_ARG, "divdmp_coef is nonzero but DDIV is NULL");
    if (in.divdmp != 0.0 && C.members.size() > 1)
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "divergence damping is not available for an ensemble");
    if (kind < 0) kind = C.short_type;
    if (C.terrain) {
        if constexpr (sizeof(F) != sizeof(double)) {
            return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the mixed-precision path takes flat terrain only");
        } else {
            const StageArgsT<double> a = stage_args(in, out, mflx, tflx, dtrk, mode);
            const bool heve = kind == 1;
            CK(timed(heve ? "heve_stage_terrain" : "hevi_stage_terrain", [&] {
                CU(heve ? launch_terrain_heve_stage(C.g, a, C.tm, C.tw, C.scheme, C.stream)
                        : launch_terrain_stage(C.g, a, C.tm, C.tw, C.scheme, C.stream));
                return SCALE_HEVI_OK;
            }));
            C.launches += heve ? TERRAIN_HEVE_LAUNCHES : TERRAIN_STAGE_LAUNCHES;
            return SCALE_HEVI_OK;
        }
    }
    if (kind == 1) {
        if constexpr (sizeof(F) != sizeof(double)) {
            return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the mixed-precision path takes the HEVI short step only");
        } else {
            const StageArgsT<double> a = stage_args(in, out, mflx, tflx, dtrk, mode);
            CK(timed("heve_stage", [&] {
                CU(launch_heve_stage(C.g, mem(), a, C.scheme, C.stream));
                return SCALE_HEVI_OK;
            }));
            ++C.launches;
            return SCALE_HEVI_OK;
        }
    }
    const int p = sizeof(F) == sizeof(double) ? 0 : 1;
    if (C.autotune && !C.tuned[p] && !C.capturing) CK(autotune_stage(in, dtrk));
    const StageArgsT<F> a = stage_args(in, out, mflx, tflx, dtrk, mode);
    int nl = 1;
    CK(timed(sizeof(F) == sizeof(double) ? "hevi_stage" : "hevi_stage_mixed", [&] {
        CU(launch_hevi_stage(C.g, mem(), a, C.scheme, C.shape[p], C.stream, &nl));
        return SCALE_HEVI_OK;
    }));
    C.launches += nl;
    return SCALE_HEVI_OK;
}

// RK4 short step on device arrays (tinteg_short_rk4.F90:199-650): stage s reads
// the previous stage's buffer (halo filled on the device) and X0 = the input
// state; the last stage writes the combined state in place.
template <typename F>
int run_rk4(double *X[5], F *mflx, F *tflx, const StageInT<F> &base, double dt)
{
    StageInT<F> in = base;
    in.DENS0 = X[0]; in.MOMZ0 = X[1]; in.MOMX0 = X[2]; in.MOMY0 = X[3]; in.RHOT0 = X[4];
    const double dts[4] = {dt / 2.0, dt / 2.0, dt, dt};
    const double *src[5] = {X[0], X[1], X[2], X[3], X[4]};
    for (int s = 0; s < 4; ++s) {
        in.DENS = src[0]; in.MOMZ = src[1]; in.MOMX = src[2]; in.MOMY = src[3]; in.RHOT = src[4];
        double *out[5];
        if (s < 3) {
            double *b = C.rk[s % 2];
            for (int v = 0; v < 5; ++v) out[v] = b + (size_t)v * C.N3;
        } else {
            for (int v = 0; v < 5; ++v) out[v] = X[v];
        }
        CK(run_stage(in, out, mflx, tflx, dts[s], RK_STAGE1 + s));
        if (s < 3) {
            CK(halo(out, 5)); // COMM_vars8 of the stage buffers (rk4.F90:401-425)
            for (int v = 0; v < 5; ++v) src[v] = out[v];
        }
    }
    return SCALE_HEVI_OK;
}

// RK3 short step on device arrays (tinteg_short_rk3.F90:188-576): stages at
// dt/3, dt*fact_dt2 and dt; stage 1 writes C.rk[0], stage 2 C.rk[1] (each then
// halo-filled, :391-406 and :444-459), stage 3 the state in place. Heun's RK3
// (fact_dt2 = 2/3) combines RK1 and the third stage in the last epilogue
// (:486-566); RK3WS2002 (fact_dt2 = 1/2) keeps the third stage. Stages 1-2 of
// RK3WS2002 and stage 2 of Heun's write their fluxes to mflx/tflx, where stage 3
// overwrites them at the same cells.
template <typename F>
int run_rk3(double *X[5], F *mflx, F *tflx, const StageInT<F> &base, double dt, bool ws2002)
{
    StageInT<F> in = base;
    in.DENS0 = X[0]; in.MOMZ0 = X[1]; in.MOMX0 = X[2]; in.MOMY0 = X[3]; in.RHOT0 = X[4];
    const double fact_dt1 = 1.0 / 3.0, fact_dt2 = ws2002 ? 1.0 / 2.0 : 2.0 / 3.0;
    const double dts[3] = {dt * fact_dt1, dt * fact_dt2, dt};
    const int modes[3] = {ws2002 ? RK_PLAIN : RK_HEUN1, RK_PLAIN, ws2002 ? RK_PLAIN : RK_HEUN3};
    const double *src[5] = {X[0], X[1], X[2], X[3], X[4]};
    for (int s = 0; s < 3; ++s) {
        in.DENS = src[0]; in.MOMZ = src[1]; in.MOMX = src[2]; in.MOMY = src[3]; in.RHOT = src[4];
        double *out[5];
        if (s < 2) {
            for (int v = 0; v < 5; ++v) out[v] = C.rk[s] + (size_t)v * C.N3;
        } else {
            for (int v = 0; v < 5; ++v) out[v] = X[v];
        }
        CK(run_stage(in, out, mflx, tflx, dts[s], modes[s]));
        if (s < 2) {
            CK(halo(out, 5));
            for (int v = 0; v < 5; ++v) src[v] = out[v];
        }
    }
    return SCALE_HEVI_OK;
}

// the registered short integrator (ATMOS_DYN_tinteg_short, scale_atmos_dyn_tinteg_short.F90)
template <typename F>
int run_short(double *X[5], F *mflx, F *tflx, const StageInT<F> &base, double dt)
{
    if (C.tinteg_type == 0) return run_rk4(X, mflx, tflx, base, dt);
    return run_rk3(X, mflx, tflx, base, dt, C.tinteg_type == 2);
}

template <typename R>
int run_numfilter(R *num_diff, const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY,
                  const double *RHOT, const double *REF_dens, const double *REF_pott)
{
    R *phi;
    if (sizeof(R) == sizeof(double)) {
        if (!C.phi) CK(dalloc(&C.phi, 5 * C.N3));
        phi = reinterpret_cast<R *>(C.phi);
    } else {
        if (!C.phi_f) CK(falloc(&C.phi_f, 5 * C.N3));
        phi = reinterpret_cast<R *>(C.phi_f);
    }
    if (C.ndc.order > 1) {
        if (sizeof(R) != sizeof(double))
            return fail(SCALE_HEVI_ERR_UNSUPPORTED, "ND_ORDER > 1 is supported on the FP64 path only");
        if (C.members.size() > 1) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "ND_ORDER > 1 is not available for an ensemble");
        if (!C.ndw) CK(dalloc(&C.ndw, 30 * C.N3));
        NdArgs ah{reinterpret_cast<double *>(num_diff), DENS, MOMZ, MOMX, MOMY, RHOT, REF_dens, REF_pott,
                  reinterpret_cast<double *>(phi)};
        // a decomposed domain exchanges the work arrays through the hook
        int hrc = SCALE_HEVI_OK;
        const HaloFill hf{hook_fill, &hrc};
        const cudaError_t e = launch_numfilter_high(C.g, C.ndc, ah, C.ndw, C.ndw + 15 * C.N3, C.stream,
                                                    C.halo_fn ? &hf : nullptr);
        if (hrc != SCALE_HEVI_OK) return hrc;
        CU(e);
        C.launches += 3 + 2 * (C.ndc.order - 1);
        R *f[15];
        for (int q = 0; q < 15; ++q) f[q] = num_diff + (size_t)q * C.N3;
        return halo(f, 15);
    }
    NdArgsT<R> a{num_diff, DENS, MOMZ, MOMX, MOMY, RHOT, REF_dens, REF_pott, phi};
    CK(timed(sizeof(R) == sizeof(double) ? "numfilter" : "numfilter_mixed", [&] {
        CU(launch_numfilter(C.g, mem(), C.ndc, a, C.stream, C.nd_tiled ? C.status : nullptr));
        return SCALE_HEVI_OK;
    }));
    C.launches += 2;
    R *f[15];
    for (int q = 0; q < 15; ++q) f[q] = num_diff + (size_t)q * C.N3;
    return halo(f, 15);
}

// ATMOS_DYN_divergence on device arrays; RCDZ/RCDX/RCDY are device vectors
int run_divergence(double *DDIV, const double *MOMZ, const double *MOMX, const double *MOMY, const double *RCDZ,
                   const double *RCDX, const double *RCDY, double J33G)
{
    CK(timed("divergence", [&] {
        if (C.terrain) divergence_terrain(C.g, DDIV, MOMZ, MOMX, MOMY, C.tm, J33G, C.stream);
        else divergence(C.g, DDIV, MOMZ, MOMX, MOMY, RCDZ, RCDX, RCDY, J33G, C.stream);
        CU(cudaGetLastError());
        return SCALE_HEVI_OK;
    }));
    ++C.launches;
    return SCALE_HEVI_OK;
}

// RK3 tracer integrator (tinteg_tracer_rk3.F90:92-210) on device arrays
// the limiter scratch of each precision: phi_lo, anti (3), rjp, rjm
template <typename R> void limiter_scratch(TracerArgsT<R> &a);
template <> void limiter_scratch<double>(TracerArgsT<double> &a)
{
    a.phi_lo = C.tr + 2 * C.N3; a.anti = C.tr + 3 * C.N3; a.rjp = C.tr + 6 * C.N3; a.rjm = C.tr + 7 * C.N3;
}
template <> void limiter_scratch<float>(TracerArgsT<float> &a)
{
    a.phi_lo = C.tr_f; a.anti = C.tr_f + C.N3; a.rjp = C.tr_f + 4 * C.N3; a.rjm = C.tr_f + 5 * C.N3;
}

template <typename R>
int run_tracer_rk3(double *QTRC, const double *QTRC0, const R *RHOQ_t, const double *DENS0, const double *DENS,
                   const R *mflx, const R *ndq, double dtl, bool fct, bool along)
{
    TracerArgsT<R> a{};
    a.QTRC0 = QTRC0; a.RHOQ_t = RHOQ_t; a.DENS0 = DENS0; a.DENS = DENS; a.mflx = mflx; a.ndq = ndq;
    limiter_scratch(a);
    a.along_stream = along ? 1 : 0;
    // terrain-following metrics of the large step (the mass-point MAPF slice comes first)
    a.GS = C.terrain ? C.tm.GSQRT : nullptr;
    a.MAPF = C.terrain ? C.tm.MAPF : nullptr;
    double *rk1 = C.tr, *rk2 = C.tr + C.N3; // the tracer's RK stage values stay FP64
    const char *sec = sizeof(R) == sizeof(double) ? "tracer" : "tracer_mixed";
    const char *sec_fct = sizeof(R) == sizeof(double) ? "tracer_fct" : "tracer_fct_mixed";
    // stage 1: dt/3 with DENS0 + (DENS-DENS0)/3
    a.QTRCo = rk1; a.QTRC = QTRC; a.dens_mode = 1; a.dtl = dtl / 3.0;
    CK(timed(sec, [&] { CU(launch_tracer_stage(C.g, a, C.scheme_tracer, false, C.stream)); return SCALE_HEVI_OK; }));
    ++C.launches;
    CK(halo(&rk1, 1));
    // stage 2: dt/2 with DENS0 + (DENS-DENS0)*0.5
    a.QTRCo = rk2; a.QTRC = rk1; a.dens_mode = 2; a.dtl = dtl / 2.0;
    CK(timed(sec, [&] { CU(launch_tracer_stage(C.g, a, C.scheme_tracer, false, C.stream)); return SCALE_HEVI_OK; }));
    ++C.launches;
    CK(halo(&rk2, 1));
    // stage 3: dt with DENS, FCT when requested
    a.QTRCo = QTRC; a.QTRC = rk2; a.dens_mode = 0; a.dtl = dtl;
    a.status = C.fct_fused ? C.status : nullptr;
    int nk = 0;
    if (fct && C.halo_fn) {
        // a decomposed domain: R+/R- go through the exchange between the limiter's kernels
        int hrc = SCALE_HEVI_OK;
        const HaloFill hf{hook_fill, &hrc};
        const cudaError_t e = launch_tracer_stage(C.g, a, C.scheme_tracer, fct, C.stream, &hf, &nk);
        if (hrc != SCALE_HEVI_OK) return hrc;
        CU(e);
    } else {
        CK(timed(fct ? sec_fct : sec, [&] {
            CU(launch_tracer_stage(C.g, a, C.scheme_tracer, fct, C.stream, nullptr, &nk));
            return SCALE_HEVI_OK;
        }));
    }
    C.launches += nk;
    return SCALE_HEVI_OK;
}

size_t n3() { return C.N3; }

}  // namespace

void hevi::set_last_error(const char *msg) { g_err = msg ? msg : ""; }

// =============================================================================
// exported entry points
// =============================================================================
extern "C" {

// checks of one index set (of a domain or an ensemble member)
static int check_index(const scale_hevi_index &x)
{
    if (x.KHALO != 2 || x.IHALO != x.JHALO || x.IHALO < 2 || x.IHALO > 3)
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "halo widths must be KHALO = 2 and IHALO = JHALO = 2 or 3 (got %d, %d, %d)",
                    x.KHALO, x.IHALO, x.JHALO);
    if (x.KA != x.KMAX + 2 * x.KHALO || x.IA != x.IMAX + 2 * x.IHALO || x.JA != x.JMAX + 2 * x.JHALO ||
        x.KS != 1 + x.KHALO || x.KE != x.KMAX + x.KHALO || x.IS != 1 + x.IHALO || x.IE != x.IMAX + x.IHALO ||
        x.JS != 1 + x.JHALO || x.JE != x.JMAX + x.JHALO)
        return fail(SCALE_HEVI_ERR_ARG, "index set is inconsistent (KA=%d KMAX=%d KS=%d KE=%d IA=%d IMAX=%d JA=%d JMAX=%d)",
                    x.KA, x.KMAX, x.KS, x.KE, x.IA, x.IMAX, x.JA, x.JMAX);
    if (x.KMAX < 4 || x.KA > 260) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "KMAX must be in 4..256 (got %d)", x.KMAX);
    if (x.IMAX < x.IHALO || x.JMAX < x.JHALO) return fail(SCALE_HEVI_ERR_ARG, "IMAX and JMAX must be >= IHALO, JHALO");
    if ((x.IBLOCK > 0 && x.IBLOCK != x.IMAX) || (x.JBLOCK > 0 && x.JBLOCK != x.JMAX))
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "only the default IBLOCK=IMAX, JBLOCK=JMAX blocking is supported");
    return SCALE_HEVI_OK;
}

int scale_hevi_ensemble_setup(int n, const scale_hevi_index *idx, const char *flux_type, const char *flux_tracer_type,
                              int device)
{
    if (C.ready) free_all();
    g_err.clear();
    if (!idx) return fail(SCALE_HEVI_ERR_ARG, "index set is NULL");
    if (n < 1 || n > HEVI_MAX_MEMBERS) return fail(SCALE_HEVI_ERR_ARG, "ensemble of %d members (1..%d)", n, HEVI_MAX_MEMBERS);
    std::vector<MemberGeom> mem(n);
    size_t N3 = 0, N2 = 0;
    long long ZT = 0, XT = 0, YT = 0;
    for (int m = 0; m < n; ++m) {
        const scale_hevi_index &x = idx[m];
        CK(check_index(x));
        if (x.IHALO != idx[0].IHALO) return fail(SCALE_HEVI_ERR_ARG, "ensemble members must share one halo width");
        mem[m] = MemberGeom{x.KMAX, x.IMAX, x.JMAX, (int)ZT, (int)XT, (int)YT, (int)N3, (int)N2};
        N3 += (size_t)x.KA * x.IA * x.JA;
        N2 += (size_t)x.IA * x.JA;
        ZT += x.KA; XT += x.IA; YT += x.JA;
        if ((double)N3 >= 2147483648.0)
            return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the fields of the domain%s exceed 2^31 points", n > 1 ? "s" : "");
    }
    int s1, s2;
    CK(parse_scheme(flux_type, &s1));
    CK(parse_scheme(flux_tracer_type, &s2));
    // the 6-point schemes read three points on each side (scale_atmos_dyn_fvm_flux.F90:742-749)
    if ((wide_scheme(s1) || wide_scheme(s2)) && idx[0].IHALO < 3)
        return fail(SCALE_HEVI_ERR_ARG, "the UD5 and CD6 schemes need IHALO = JHALO = 3 (got %d)", idx[0].IHALO);
    // their near-wall forms at KS+1 and KE-2 read five levels of the interior
    for (int m = 0; m < n; ++m)
        if ((wide_scheme(s1) || wide_scheme(s2)) && idx[m].KMAX < 5)
            return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the UD5 and CD6 schemes need KMAX >= 5 (got %d)", idx[m].KMAX);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SCALE_HEVI_ERR_CUDA, "no CUDA device is available");
    }
    if (device < 0 || device >= ndev) return fail(SCALE_HEVI_ERR_ARG, "device %d out of range (%d devices)", device, ndev);
    CU(cudaSetDevice(device));
    C.device = device;
    const scale_hevi_index &x = idx[0];
    C.idx = x;
    C.member_idx.assign(idx, idx + n);
    C.members = mem;
    C.scheme = s1;
    C.scheme_tracer = s2;
    Grid &g = C.g;
    g.KA = x.KA; g.IA = x.IA; g.JA = x.JA;
    g.KS = x.KS; g.KE = x.KE; g.IS = x.IS; g.IE = x.IE; g.JS = x.JS; g.JE = x.JE;
    g.KMAX = x.KMAX; g.IMAX = x.IMAX; g.JMAX = x.JMAX; g.IHALO = x.IHALO; g.JHALO = x.JHALO;
    g.IEH = x.IE; g.JEH = x.JE; // BND_E = BND_N = .false.
    g.cell0 = g.c2 = g.z0 = g.x0 = g.y0 = 0;
    g.stride = N3;
    C.N3 = N3;
    C.N2 = N2;
    C.ZT = (int)ZT; C.XT = (int)XT; C.YT = (int)YT;
    // a blocking stream: its work is ordered with the legacy default stream,
    // on which callers such as torch enqueue the producers and consumers of
    // the device arrays handed to the _dev entries
    CU(cudaStreamCreate(&C.stream));
    int rc = SCALE_HEVI_OK;
    if ((rc = dalloc(&C.d_tab, 7 * (size_t)ZT + 4 * (size_t)XT + 4 * (size_t)YT)) ||
        (rc = dalloc(&C.d_nd, 18 * (size_t)ZT + 18 * (size_t)XT + 18 * (size_t)YT)) ||
        (rc = dalloc(&C.rk[0], 5 * N3)) || (rc = dalloc(&C.rk[1], 5 * N3)) ||
        (rc = dalloc(&C.acc, 5 * N3)) || (rc = dalloc(&C.facc, 6 * N3)) ||
        (rc = dalloc(&C.colscr, 4 * N3)) || (rc = dalloc(&C.colC, 2 * N3)) ||
        (rc = dalloc(&C.sum_part, (size_t)x.IMAX * x.JMAX)) || (rc = dalloc(&C.sum_out, 1))) {
        free_all();
        return rc;
    }
    if (cudaMalloc((void **)&C.status, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc((void **)&C.count, sizeof(unsigned long long)) != cudaSuccess) {
        free_all();
        return fail(SCALE_HEVI_ERR_ALLOC, "cudaMalloc of status words failed");
    }
    cudaMemset(C.status, 0, sizeof(unsigned));
    C.ready = true;
    return SCALE_HEVI_OK;
}

int scale_hevi_setup(const scale_hevi_index *idx, const char *flux_type, const char *flux_tracer_type, int device)
{
    return scale_hevi_ensemble_setup(1, idx, flux_type, flux_tracer_type, device);
}

int scale_hevi_ensemble_layout(long long *cell0, long long *col0, long long *z0, long long *x0, long long *y0)
{
    CK(need_setup());
    const size_t n = C.members.size();
    for (size_t m = 0; m <= n; ++m) {
        const bool end = m == n;
        const MemberGeom &g = C.members[end ? 0 : m];
        if (cell0) cell0[m] = end ? (long long)C.N3 : g.cell0;
        if (col0) col0[m] = end ? (long long)C.N2 : g.c2;
        if (z0) z0[m] = end ? C.ZT : g.z0;
        if (x0) x0[m] = end ? C.XT : g.x0;
        if (y0) y0[m] = end ? C.YT : g.y0;
    }
    return SCALE_HEVI_OK;
}

int scale_hevi_short_type(const char *type)
{
    CK(need_setup());
    if (!type) return fail(SCALE_HEVI_ERR_ARG, "short-step type is NULL");
    std::string n(type);
    while (!n.empty() && n.back() == ' ') n.pop_back(); // Fortran blank padding
    if (n == "HEVI" || n == "FVM-HEVI") { C.short_type = 0; return SCALE_HEVI_OK; }
    if (n == "HEVE" || n == "FVM-HEVE") { C.short_type = 1; return SCALE_HEVI_OK; }
    return fail(SCALE_HEVI_ERR_UNSUPPORTED, "short-step type '%s' is not supported (HEVI, HEVE)", n.c_str());
}

int scale_hevi_set_halo_exchange(scale_hevi_halo_fn fn, void *user)
{
    CK(need_setup());
    if (fn) CK(need_single("a halo exchange hook"));
    C.halo_fn = fn;
    C.halo_user = user;
    return SCALE_HEVI_OK;
}

int scale_hevi_tinteg_short_type(const char *type)
{
    CK(need_setup());
    if (!type) return fail(SCALE_HEVI_ERR_ARG, "short integrator type is NULL");
    std::string n(type);
    while (!n.empty() && n.back() == ' ') n.pop_back(); // Fortran blank padding
    if (n == "RK4") { C.tinteg_type = 0; return SCALE_HEVI_OK; }
    if (n == "RK3") { C.tinteg_type = 1; return SCALE_HEVI_OK; }
    if (n == "RK3WS2002") { C.tinteg_type = 2; return SCALE_HEVI_OK; }
    return fail(SCALE_HEVI_ERR_UNSUPPORTED, "short integrator '%s' is not supported (RK4, RK3, RK3WS2002)", n.c_str());
}

int scale_hevi_stage_shape(int tile_x, int raster)
{
    CK(need_setup());
    bool ok = tile_x == 0;
    for (int t : STAGE_TILE_XS) ok |= tile_x == t;
    if (!ok || raster < 0) return fail(SCALE_HEVI_ERR_ARG, "tile width %d / raster %d is not a compiled shape", tile_x, raster);
    C.shape[0] = C.shape[1] = StageShape{tile_x, raster};
    C.autotune = 0;
    return SCALE_HEVI_OK;
}

int scale_hevi_stage_autotune(int enable)
{
    CK(need_setup());
    C.autotune = enable != 0;
    C.tuned[0] = C.tuned[1] = false;
    C.tune_text.clear();
    return SCALE_HEVI_OK;
}

int scale_hevi_stage_shape_get(int *tile_x, int *raster, int mixed)
{
    CK(need_setup());
    const StageShape &s = C.shape[mixed ? 1 : 0];
    if (tile_x) *tile_x = s.tile_x; // 0: the tiled stage where it applies
    if (raster) *raster = s.raster > 0 ? s.raster : STAGE_RASTER_DEFAULT;
    return SCALE_HEVI_OK;
}

int scale_hevi_finalize(void)
{
    if (C.ready && C.stream) cudaStreamSynchronize(C.stream);
    free_all();
    return SCALE_HEVI_OK;
}

const char *scale_hevi_last_error(void) { return g_err.c_str(); }
void *scale_hevi_stream(void) { return (void *)C.stream; }
long long scale_hevi_kernel_launches(void) { return C.launches; }

int scale_hevi_transfer_bytes(long long *h2d_bytes, long long *d2h_bytes)
{
    if (h2d_bytes) *h2d_bytes = C.h2d_bytes;
    if (d2h_bytes) *d2h_bytes = C.d2h_bytes;
    return SCALE_HEVI_OK;
}

int scale_hevi_check(void)
{
    CK(need_setup());
    unsigned st = 0;
    CU(cudaMemcpyAsync(&st, C.status, sizeof st, cudaMemcpyDeviceToHost, C.stream));
    CU(cudaStreamSynchronize(C.stream));
    CU(cudaMemsetAsync(C.status, 0, sizeof(unsigned), C.stream));
    if (st & ST_TMA_TIMEOUT)
        return fail(SCALE_HEVI_ERR_CUDA, "a bulk tensor copy of the tiled stage did not complete within its wait limit");
    if (st & ST_BARRIER_TIMEOUT)
        return fail(SCALE_HEVI_ERR_CUDA, "a grid barrier of the persistent short step did not complete within its wait limit");
    if (st & ST_NONFINITE) return fail(SCALE_HEVI_ERR_NONFINITE, "a prognostic output became NaN or Inf");
    if (st & (1u << 4)) return fail(SCALE_HEVI_ERR_CUDA, "an adjoint pass loaded more inputs than its derivative slots");
    return SCALE_HEVI_OK;
}

// ---- HEVI stage --------------------------------------------------------------
#define SCALE_HEVI_TSTEP_SHORT_NAMES                                                                            \
    DENS_RK, MOMZ_RK, MOMX_RK, MOMY_RK, RHOT_RK, PROG_RK, mflx_hi, tflx_hi, DENS0, MOMZ0, MOMX0, MOMY0, RHOT0, \
        DENS, MOMZ, MOMX, MOMY, RHOT, DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, PROG0, PROG, DPRES0, RT2P,        \
        CORIOLI, num_diff, wdamp_coef, divdmp_coef, DDIV, FLAG_FCT_MOMENTUM, FLAG_FCT_T, FLAG_FCT_ALONG_STREAM, \
        CDZ, FDZ, FDX, FDY, RCDZ, RCDX, RCDY, RFDZ, RFDX, RFDY, PHI, GSQRT, J13G, J23G, J33G, MAPF, REF_dens,   \
        REF_rhot, BND_W, BND_E, BND_S, BND_N, dtrk, last
static int stage_host(SCALE_HEVI_TSTEP_SHORT_ARGS, int kind);

int ATMOS_DYN_Tstep_short_fvm_hevi_b200_dev(SCALE_HEVI_TSTEP_SHORT_ARGS)
{
    (void)PROG_RK; (void)PROG0; (void)PROG; (void)FLAG_FCT_MOMENTUM; (void)FLAG_FCT_T; (void)FLAG_FCT_ALONG_STREAM;
    (void)last; (void)PHI;
    CK(need_setup());
    CK(check_bnd(BND_W, BND_E, BND_S, BND_N));
    CK(use_metrics(GSQRT, J13G, J23G, MAPF, PHI, true));
    CK(prepare_tables(CDZ, FDZ, RCDZ, RFDZ, FDX, RCDX, RFDX, FDY, RCDY, RFDY, wdamp_coef, nullptr, nullptr));
    StageIn in{DENS0, MOMZ0, MOMX0, MOMY0, RHOT0, DENS, MOMZ, MOMX, MOMY, RHOT,
               DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, DPRES0, RT2P, CORIOLI, num_diff, DDIV, REF_dens, REF_rhot,
               *divdmp_coef, *J33G};
    double *out[5] = {DENS_RK, MOMZ_RK, MOMX_RK, MOMY_RK, RHOT_RK};
    return run_stage(in, out, mflx_hi, tflx_hi, *dtrk, RK_PLAIN, 0);
}

int ATMOS_DYN_Tstep_short_fvm_hevi_b200(SCALE_HEVI_TSTEP_SHORT_ARGS)
{
    return stage_host(SCALE_HEVI_TSTEP_SHORT_NAMES, 0);
}

// ---- HEVE stage (ATMOS_DYN_Tstep_short_fvm_heve, scale_atmos_dyn_tstep_short_fvm_heve.F90:109-1518) ----
static int check_heve_fct(const int *FLAG_FCT_MOMENTUM, const int *FLAG_FCT_T)
{
    if ((FLAG_FCT_MOMENTUM && *FLAG_FCT_MOMENTUM) || (FLAG_FCT_T && *FLAG_FCT_T))
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the HEVE momentum/theta FCT is not supported");
    return SCALE_HEVI_OK;
}

int ATMOS_DYN_Tstep_short_fvm_heve_b200_dev(SCALE_HEVI_TSTEP_SHORT_ARGS)
{
    (void)PROG_RK; (void)PROG0; (void)PROG; (void)FLAG_FCT_ALONG_STREAM; (void)last; (void)PHI;
    CK(need_setup());
    CK(check_heve_fct(FLAG_FCT_MOMENTUM, FLAG_FCT_T));
    CK(check_bnd(BND_W, BND_E, BND_S, BND_N));
    CK(use_metrics(GSQRT, J13G, J23G, MAPF, PHI, true));
    CK(prepare_tables(CDZ, FDZ, RCDZ, RFDZ, FDX, RCDX, RFDX, FDY, RCDY, RFDY, wdamp_coef, nullptr, nullptr));
    StageIn in{DENS0, MOMZ0, MOMX0, MOMY0, RHOT0, DENS, MOMZ, MOMX, MOMY, RHOT,
               DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, DPRES0, RT2P, CORIOLI, num_diff, DDIV, REF_dens, REF_rhot,
               *divdmp_coef, *J33G};
    double *out[5] = {DENS_RK, MOMZ_RK, MOMX_RK, MOMY_RK, RHOT_RK};
    return run_stage(in, out, mflx_hi, tflx_hi, *dtrk, RK_PLAIN, 1);
}

int ATMOS_DYN_Tstep_short_fvm_heve_b200(SCALE_HEVI_TSTEP_SHORT_ARGS)
{
    CK(check_heve_fct(FLAG_FCT_MOMENTUM, FLAG_FCT_T));
    return stage_host(SCALE_HEVI_TSTEP_SHORT_NAMES, 1);
}

// host-array form of one stage (kind 0 HEVI, 1 HEVE): copies in, runs, copies back
static int stage_host(SCALE_HEVI_TSTEP_SHORT_ARGS, int kind)
{
    CK(need_single("the host-array stage entry"));
    CK(check_bnd(BND_W, BND_E, BND_S, BND_N));
    CK(use_metrics(GSQRT, J13G, J23G, MAPF, PHI, false));
    const size_t N3 = n3(), N2 = (size_t)C.g.IA * C.g.JA;
    const bool use_div = *divdmp_coef != 0.0;
    double *o[5], *mf, *tf, *i0[5], *iv[5], *it[5], *dp0, *rt, *cor, *nd, *ddiv = nullptr, *rd, *rr;
    const double *hin0[5] = {DENS0, MOMZ0, MOMX0, MOMY0, RHOT0};
    const double *hin[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    const double *htt[5] = {DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t};
    double *hout[5] = {DENS_RK, MOMZ_RK, MOMX_RK, MOMY_RK, RHOT_RK};
    static const char *n_o[5] = {"o0", "o1", "o2", "o3", "o4"}, *n_0[5] = {"a0", "a1", "a2", "a3", "a4"};
    static const char *n_v[5] = {"b0", "b1", "b2", "b3", "b4"}, *n_t[5] = {"t0", "t1", "t2", "t3", "t4"};
    for (int v = 0; v < 5; ++v) {
        CK(h2d(n_o[v], hout[v], N3, &o[v])); // cells the stage does not write keep their contents
        CK(h2d(n_0[v], hin0[v], N3, &i0[v]));
        CK(h2d(n_v[v], hin[v], N3, &iv[v]));
        CK(h2d(n_t[v], htt[v], N3, &it[v]));
    }
    CK(h2d("mflx", mflx_hi, 3 * N3, &mf));
    CK(h2d("tflx", tflx_hi, 3 * N3, &tf));
    CK(h2d("DPRES0", DPRES0, N3, &dp0));
    CK(h2d("RT2P", RT2P, N3, &rt));
    CK(h2d("CORIOLI", CORIOLI, N2, &cor));
    CK(h2d("num_diff", num_diff, 15 * N3, &nd));
    if (use_div) CK(h2d("DDIV", DDIV, N3, &ddiv));
    CK(h2d("REF_dens", REF_dens, N3, &rd));
    CK(h2d("REF_rhot", REF_rhot, N3, &rr));
    CK(prepare_tables(CDZ, FDZ, RCDZ, RFDZ, FDX, RCDX, RFDX, FDY, RCDY, RFDY, wdamp_coef, nullptr, nullptr));
    StageIn in{i0[0], i0[1], i0[2], i0[3], i0[4], iv[0], iv[1], iv[2], iv[3], iv[4],
               it[0], it[1], it[2], it[3], it[4], dp0, rt, cor, nd, ddiv, rd, rr, *divdmp_coef, *J33G};
    CK(run_stage(in, o, mf, tf, *dtrk, RK_PLAIN, kind));
    for (int v = 0; v < 5; ++v) CK(d2h(hout[v], o[v], N3));
    CK(d2h(mflx_hi, mf, 3 * N3));
    CK(d2h(tflx_hi, tf, 3 * N3));
    CU(cudaStreamSynchronize(C.stream));
    (void)PROG_RK; (void)PROG0; (void)PROG; (void)FLAG_FCT_MOMENTUM; (void)FLAG_FCT_T; (void)FLAG_FCT_ALONG_STREAM; (void)last; (void)PHI;
    return scale_hevi_check();
}

// ---- RK4 short step ------------------------------------------------------------
int ATMOS_DYN_Tinteg_short_rk4_b200_dev(SCALE_HEVI_TINTEG_SHORT_ARGS)
{
    (void)PROG; (void)FLAG_FCT_ALONG_STREAM; (void)PHI;
    CK(need_setup());
    if (C.short_type == 1) CK(check_heve_fct(FLAG_FCT_MOMENTUM, FLAG_FCT_T));
    CK(check_bnd(BND_W, BND_E, BND_S, BND_N));
    CK(use_metrics(GSQRT, J13G, J23G, MAPF, PHI, true));
    CK(prepare_tables(CDZ, FDZ, RCDZ, RFDZ, FDX, RCDX, RFDX, FDY, RCDY, RFDY, wdamp_coef, nullptr, nullptr));
    double *X[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    StageIn base{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                 DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, DPRES0, RT2P, CORIOLI, num_diff, DDIV, REF_dens, REF_rhot,
                 *divdmp_coef, *J33G};
    return run_rk4(X, mflx_hi, tflx_hi, base, *dt);
}

int ATMOS_DYN_Tinteg_short_rk4_b200(SCALE_HEVI_TINTEG_SHORT_ARGS)
{
    CK(need_single("the host-array RK4 entry"));
    if (C.short_type == 1) CK(check_heve_fct(FLAG_FCT_MOMENTUM, FLAG_FCT_T));
    CK(check_bnd(BND_W, BND_E, BND_S, BND_N));
    CK(use_metrics(GSQRT, J13G, J23G, MAPF, PHI, false));
    const size_t N3 = n3(), N2 = (size_t)C.g.IA * C.g.JA;
    double *hx[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    const double *htt[5] = {DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t};
    static const char *n_x[5] = {"x0", "x1", "x2", "x3", "x4"}, *n_t[5] = {"t0", "t1", "t2", "t3", "t4"};
    double *X[5], *T[5], *mf, *tf, *dp0, *rt, *cor, *nd, *ddiv = nullptr, *rd, *rr;
    for (int v = 0; v < 5; ++v) {
        CK(h2d(n_x[v], hx[v], N3, &X[v]));
        CK(h2d(n_t[v], htt[v], N3, &T[v]));
    }
    CK(h2d("mflx", mflx_hi, 3 * N3, &mf));
    CK(h2d("tflx", tflx_hi, 3 * N3, &tf));
    CK(h2d("DPRES0", DPRES0, N3, &dp0));
    CK(h2d("RT2P", RT2P, N3, &rt));
    CK(h2d("CORIOLI", CORIOLI, N2, &cor));
    CK(h2d("num_diff", num_diff, 15 * N3, &nd));
    if (*divdmp_coef != 0.0) CK(h2d("DDIV", DDIV, N3, &ddiv));
    CK(h2d("REF_dens", REF_dens, N3, &rd));
    CK(h2d("REF_rhot", REF_rhot, N3, &rr));
    CK(prepare_tables(CDZ, FDZ, RCDZ, RFDZ, FDX, RCDX, RFDX, FDY, RCDY, RFDY, wdamp_coef, nullptr, nullptr));
    StageIn base{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                 T[0], T[1], T[2], T[3], T[4], dp0, rt, cor, nd, ddiv, rd, rr, *divdmp_coef, *J33G};
    CK(run_rk4(X, mf, tf, base, *dt));
    for (int v = 0; v < 5; ++v) CK(d2h(hx[v], X[v], N3));
    CK(d2h(mflx_hi, mf, 3 * N3));
    CK(d2h(tflx_hi, tf, 3 * N3));
    CU(cudaStreamSynchronize(C.stream));
    (void)PROG; (void)FLAG_FCT_MOMENTUM; (void)FLAG_FCT_T; (void)FLAG_FCT_ALONG_STREAM; (void)PHI;
    return scale_hevi_check();
}

// ---- RK3 short step (Heun's RK3 or RK3WS2002) -----------------------------------
// the RK3 variant chosen by ATMOS_DYN_Tinteg_short_rk3_setup (tinteg_short_rk3.F90:104-132),
// here by scale_hevi_tinteg_short_type
static int rk3_type(bool *ws2002)
{
    if (C.tinteg_type == 0)
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the registered short integrator is RK4; register RK3 or RK3WS2002 first");
    *ws2002 = C.tinteg_type == 2;
    return SCALE_HEVI_OK;
}

int ATMOS_DYN_Tinteg_short_rk3_b200_dev(SCALE_HEVI_TINTEG_SHORT_ARGS)
{
    (void)PROG; (void)FLAG_FCT_ALONG_STREAM; (void)PHI;
    CK(need_setup());
    bool ws2002;
    CK(rk3_type(&ws2002));
    if (C.short_type == 1) CK(check_heve_fct(FLAG_FCT_MOMENTUM, FLAG_FCT_T));
    CK(check_bnd(BND_W, BND_E, BND_S, BND_N));
    CK(use_metrics(GSQRT, J13G, J23G, MAPF, PHI, true));
    CK(prepare_tables(CDZ, FDZ, RCDZ, RFDZ, FDX, RCDX, RFDX, FDY, RCDY, RFDY, wdamp_coef, nullptr, nullptr));
    double *X[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    StageIn base{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                 DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, DPRES0, RT2P, CORIOLI, num_diff, DDIV, REF_dens, REF_rhot,
                 *divdmp_coef, *J33G};
    return run_rk3(X, mflx_hi, tflx_hi, base, *dt, ws2002);
}

int ATMOS_DYN_Tinteg_short_rk3_b200(SCALE_HEVI_TINTEG_SHORT_ARGS)
{
    CK(need_single("the host-array RK3 entry"));
    bool ws2002;
    CK(rk3_type(&ws2002));
    if (C.short_type == 1) CK(check_heve_fct(FLAG_FCT_MOMENTUM, FLAG_FCT_T));
    CK(check_bnd(BND_W, BND_E, BND_S, BND_N));
    CK(use_metrics(GSQRT, J13G, J23G, MAPF, PHI, false));
    const size_t N3 = n3(), N2 = (size_t)C.g.IA * C.g.JA;
    double *hx[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    const double *htt[5] = {DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t};
    static const char *n_x[5] = {"x0", "x1", "x2", "x3", "x4"}, *n_t[5] = {"t0", "t1", "t2", "t3", "t4"};
    double *X[5], *T[5], *mf, *tf, *dp0, *rt, *cor, *nd, *ddiv = nullptr, *rd, *rr;
    for (int v = 0; v < 5; ++v) {
        CK(h2d(n_x[v], hx[v], N3, &X[v]));
        CK(h2d(n_t[v], htt[v], N3, &T[v]));
    }
    CK(h2d("mflx", mflx_hi, 3 * N3, &mf));
    CK(h2d("tflx", tflx_hi, 3 * N3, &tf));
    CK(h2d("DPRES0", DPRES0, N3, &dp0));
    CK(h2d("RT2P", RT2P, N3, &rt));
    CK(h2d("CORIOLI", CORIOLI, N2, &cor));
    CK(h2d("num_diff", num_diff, 15 * N3, &nd));
    if (*divdmp_coef != 0.0) CK(h2d("DDIV", DDIV, N3, &ddiv));
    CK(h2d("REF_dens", REF_dens, N3, &rd));
    CK(h2d("REF_rhot", REF_rhot, N3, &rr));
    CK(prepare_tables(CDZ, FDZ, RCDZ, RFDZ, FDX, RCDX, RFDX, FDY, RCDY, RFDY, wdamp_coef, nullptr, nullptr));
    StageIn base{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                 T[0], T[1], T[2], T[3], T[4], dp0, rt, cor, nd, ddiv, rd, rr, *divdmp_coef, *J33G};
    CK(run_rk3(X, mf, tf, base, *dt, ws2002));
    for (int v = 0; v < 5; ++v) CK(d2h(hx[v], X[v], N3));
    CK(d2h(mflx_hi, mf, 3 * N3));
    CK(d2h(tflx_hi, tf, 3 * N3));
    CU(cudaStreamSynchronize(C.stream));
    (void)PROG; (void)FLAG_FCT_MOMENTUM; (void)FLAG_FCT_T; (void)FLAG_FCT_ALONG_STREAM; (void)PHI;
    return scale_hevi_check();
}

// ---- mixed precision: FP32 flux arithmetic, FP64 state and solve -----------------
int ATMOS_DYN_Tinteg_short_rk4_b200_mixed_dev(SCALE_HEVI_TINTEG_SHORT_MIXED_ARGS)
{
    (void)PROG; (void)FLAG_FCT_ALONG_STREAM; (void)PHI;
    CK(need_setup());
    if (C.short_type == 1) CK(check_heve_fct(FLAG_FCT_MOMENTUM, FLAG_FCT_T));
    CK(check_bnd(BND_W, BND_E, BND_S, BND_N));
    CK(check_flat(GSQRT, J13G, J23G, MAPF, true));
    CK(prepare_tables(CDZ, FDZ, RCDZ, RFDZ, FDX, RCDX, RFDX, FDY, RCDY, RFDY, wdamp_coef, nullptr, nullptr));
    if (!C.facc_f) CK(falloc(&C.facc_f, 6 * C.N3));
    if (!C.colscr_f) CK(falloc(&C.colscr_f, 4 * C.N3));
    double *X[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    StageInT<float> base{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                         DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t, DPRES0, RT2P, CORIOLI, num_diff, DDIV, REF_dens, REF_rhot,
                         *divdmp_coef, *J33G};
    return run_rk4(X, mflx_hi, tflx_hi, base, *dt);
}

int ATMOS_DYN_numfilter_coef_b200_mixed_dev(SCALE_HEVI_NUMFILTER_MIXED_ARGS)
{
    CK(need_setup());
    if (*ND_ORDER != 1) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "ND_ORDER=%d is not supported (1 only)", *ND_ORDER);
    if (!*ND_USE_RS) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "ND_USE_RS=.false. is not supported");
    CK(prepare_nd(CDZ, CDX, CDY, FDZ, FDX, FDY, *DT, *ND_COEF, *ND_ORDER, *ND_SFC_FACT));
    return run_numfilter(num_diff, DENS, MOMZ, MOMX, MOMY, RHOT, REF_dens, REF_pott);
}

// ---- the persistent short step ------------------------------------------------
// numerical filter + RK4 HEVI + vertical boundary values + halo as one
// cooperative launch over all members (persist.cu)
extern "C++" {
template <typename R>
int short_step_persistent(double *X[5], R *mflx, R *tflx, R *num_diff, const R *const tend[5],
                          const double *DPRES0, const double *RT2P, const double *CORIOLI, const double *wdamp_coef,
                          const double *CDZ, const double *CDX, const double *CDY, const double *FDZ,
                          const double *FDX, const double *FDY, const double *RCDZ, const double *RCDX,
                          const double *RCDY, const double *RFDZ, const double *RFDX, const double *RFDY,
                          const double *REF_dens, const double *REF_pott, const double *REF_rhot, double nd_coef,
                          double sfc, double dt)
{
    CK(need_setup());
    if (C.short_type != 0 || C.tinteg_type != 0)
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the persistent short step runs RK4 of HEVI stages only");
    if (C.halo_fn) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the persistent short step does not take a halo exchange hook");
    CK(prepare_nd(CDZ, CDX, CDY, FDZ, FDX, FDY, dt, nd_coef, 1, sfc));
    CK(prepare_tables(CDZ, FDZ, RCDZ, RFDZ, FDX, RCDX, RFDX, FDY, RCDY, RFDY, wdamp_coef, nullptr, nullptr));
    R *phi;
    if constexpr (sizeof(R) == sizeof(double)) {
        if (!C.phi) CK(dalloc(&C.phi, 5 * C.N3));
        phi = C.phi;
    } else {
        if (!C.phi_f) CK(falloc(&C.phi_f, 5 * C.N3));
        if (!C.facc_f) CK(falloc(&C.facc_f, 6 * C.N3));
        if (!C.colscr_f) CK(falloc(&C.colscr_f, 4 * C.N3));
        phi = C.phi_f;
    }
    if (!C.pbar && cudaMalloc((void **)&C.pbar, PERSIST_WORDS * sizeof(unsigned)) != cudaSuccess) {
        C.pbar = nullptr;
        cudaGetLastError();
        return fail(SCALE_HEVI_ERR_ALLOC, "cudaMalloc of the persistent step's counters failed");
    }
    PersistStepT<R> p{};
    p.ndc = C.ndc;
    p.nd = NdArgsT<R>{num_diff, X[0], X[1], X[2], X[3], X[4], REF_dens, REF_pott, phi};
    StageInT<R> in{X[0], X[1], X[2], X[3], X[4], nullptr, nullptr, nullptr, nullptr, nullptr,
                   tend[0], tend[1], tend[2], tend[3], tend[4], DPRES0, RT2P, CORIOLI, num_diff, nullptr, REF_dens,
                   REF_rhot, 0.0, 1.0};
    const double dts[4] = {dt / 2.0, dt / 2.0, dt, dt};
    const double *src[5] = {X[0], X[1], X[2], X[3], X[4]};
    for (int s = 0; s < 4; ++s) {
        in.DENS = src[0]; in.MOMZ = src[1]; in.MOMX = src[2]; in.MOMY = src[3]; in.RHOT = src[4];
        double *out[5];
        for (int v = 0; v < 5; ++v) out[v] = s < 3 ? C.rk[s % 2] + (size_t)v * C.N3 : X[v];
        p.st[s] = stage_args(in, out, mflx, tflx, dts[s], RK_STAGE1 + s);
        if (s < 3)
            for (int v = 0; v < 5; ++v) { p.rk[s][v] = out[v]; src[v] = out[v]; }
    }
    for (int v = 0; v < 5; ++v) p.X[v] = X[v];
    p.bar = C.pbar;
    p.status = C.status;
    p.raster = C.shape[sizeof(R) == sizeof(double) ? 0 : 1].raster;
    p.wait_s = C.pwait_s;
    p.extra = C.pextra;
    CK(timed(sizeof(R) == sizeof(double) ? "short_step_persistent" : "short_step_persistent_mixed", [&] {
        CU(launch_short_step_persistent(C.g, mem(), p, C.scheme, C.stream, &C.pgrid));
        return SCALE_HEVI_OK;
    }));
    ++C.launches;
    return SCALE_HEVI_OK;
}
} // extern "C++"

#define SCALE_HEVI_SHORT_STEP_CALL                                                                              \
    DPRES0, RT2P, CORIOLI, wdamp_coef, CDZ, CDX, CDY, FDZ, FDX, FDY, RCDZ, RCDX, RCDY, RFDZ, RFDX, RFDY,       \
        REF_dens, REF_pott, REF_rhot, *ND_COEF, *ND_SFC_FACT, *dt

int scale_hevi_short_step_persistent_dev(SCALE_HEVI_SHORT_STEP_ARGS)
{
    double *X[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    const double *tend[5] = {DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t};
    return short_step_persistent<double>(X, mflx_hi, tflx_hi, num_diff, tend, SCALE_HEVI_SHORT_STEP_CALL);
}

int scale_hevi_short_step_persistent_mixed_dev(SCALE_HEVI_SHORT_STEP_MIXED_ARGS)
{
    double *X[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    const float *tend[5] = {DENS_t, MOMZ_t, MOMX_t, MOMY_t, RHOT_t};
    return short_step_persistent<float>(X, mflx_hi, tflx_hi, num_diff, tend, SCALE_HEVI_SHORT_STEP_CALL);
}

int scale_hevi_persistent_wait(const double *seconds, const int *extra_arrivals)
{
    CK(need_setup());
    if (!(*seconds > 0.0) || *seconds > 60.0) return fail(SCALE_HEVI_ERR_ARG, "the wait limit must lie in (0, 60] s");
    if (*extra_arrivals < 0 || *extra_arrivals > 1) return fail(SCALE_HEVI_ERR_ARG, "extra_arrivals must be 0 or 1");
    C.pwait_s = *seconds;
    C.pextra = (unsigned)*extra_arrivals;
    return SCALE_HEVI_OK;
}

int scale_hevi_numfilter_form(int tiled)
{
    CK(need_setup());
    C.nd_tiled = tiled != 0;
    return SCALE_HEVI_OK;
}

int scale_hevi_tracer_fct_form(int fused)
{
    CK(need_setup());
    C.fct_fused = fused != 0;
    return SCALE_HEVI_OK;
}

int scale_hevi_persistent_grid(int *ctas)
{
    CK(need_setup());
    *ctas = C.pgrid;
    return SCALE_HEVI_OK;
}

// ---- numerical filter --------------------------------------------------------
int ATMOS_DYN_numfilter_coef_b200_dev(SCALE_HEVI_NUMFILTER_ARGS)
{
    CK(need_setup());
    if (*ND_ORDER < 1 || *ND_ORDER > 8) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "ND_ORDER=%d is not supported (1..8)", *ND_ORDER);
    if (!*ND_USE_RS) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "ND_USE_RS=.false. is not supported");
    CK(prepare_nd(CDZ, CDX, CDY, FDZ, FDX, FDY, *DT, *ND_COEF, *ND_ORDER, *ND_SFC_FACT));
    return run_numfilter(num_diff, DENS, MOMZ, MOMX, MOMY, RHOT, REF_dens, REF_pott);
}

int ATMOS_DYN_numfilter_coef_b200(SCALE_HEVI_NUMFILTER_ARGS)
{
    CK(need_single("the host-array numerical filter"));
    const size_t N3 = n3();
    double *nd, *d[5], *rd, *rp;
    const double *h[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    static const char *nm[5] = {"x0", "x1", "x2", "x3", "x4"};
    for (int v = 0; v < 5; ++v) CK(h2d(nm[v], h[v], N3, &d[v]));
    CK(h2d("REF_dens", REF_dens, N3, &rd));
    CK(h2d("REF_pott", REF_pott, N3, &rp));
    CK(stage_buf("num_diff", 15 * N3, &nd));
    int rc = ATMOS_DYN_numfilter_coef_b200_dev(nd, d[0], d[1], d[2], d[3], d[4], CDZ, CDX, CDY, FDZ, FDX, FDY, DT, rd, rp,
                                               ND_COEF, ND_ORDER, ND_SFC_FACT, ND_USE_RS);
    if (rc) return rc;
    CK(d2h(num_diff, nd, 15 * N3));
    CU(cudaStreamSynchronize(C.stream));
    return SCALE_HEVI_OK;
}

// ---- tracer ------------------------------------------------------------------
// Metrics of the tracer entries: GSQRT (KA,IA,JA,7) and the (IA,JA,2) MAPF slice
// at (x,y). Flat ones (GSQRT = 1, MAPF = 1) take the plain factors; others
// enter the tracer kernels (TracerArgs::GS/MAPF), on the device. *dGS/*dMAPF
// receive the device arrays of non-flat metrics (null on flat terrain); host
// arrays are copied to the device first.
static int tracer_metrics(const double *GSQRT, const double *MAPF, bool on_device, const double **dGS,
                          const double **dMAPF)
{
    CK(need_single("tracer advection"));
    C.terrain = false;
    *dGS = *dMAPF = nullptr;
    bool flat_g = true, flat_m = true;
    if (GSQRT) CK(metrics_flat(GSQRT, nullptr, nullptr, nullptr, on_device, &flat_g));
    if (MAPF) {
        std::vector<const void *> key = {MAPF, (const void *)(size_t)(on_device ? 3 : 2)};
        bool seen = false;
        for (auto &k : C.flat_ok) if (k == key) { seen = true; flat_m = true; }
        for (auto &k : C.nonflat) if (k == key) { seen = true; flat_m = false; }
        if (!seen) {
            const size_t n = (size_t)C.g.IA * C.g.JA * 2;
            unsigned long long bad = 0;
            if (on_device) {
                CU(cudaMemsetAsync(C.count, 0, sizeof bad, C.stream));
                count_not_equal(MAPF, n, 1.0, C.count, C.stream);
                ++C.launches;
                CU(cudaMemcpyAsync(&bad, C.count, sizeof bad, cudaMemcpyDeviceToHost, C.stream));
                CU(cudaStreamSynchronize(C.stream));
            } else {
                for (size_t q = 0; q < n; ++q) bad += MAPF[q] != 1.0;
            }
            flat_m = bad == 0;
            (flat_m ? C.flat_ok : C.nonflat).push_back(key);
        }
    }
    if (!C.tr) CK(dalloc(&C.tr, 8 * C.N3));
    if (flat_g && flat_m) return SCALE_HEVI_OK;
    if (!GSQRT || !MAPF) return fail(SCALE_HEVI_ERR_ARG, "terrain-following metrics need GSQRT and MAPF");
    if (on_device) {
        *dGS = GSQRT;
        *dMAPF = MAPF;
    } else {
        double *g7, *mp;
        CK(h2d("GSQRT", GSQRT, 7 * C.N3, &g7));
        CK(h2d("MAPF_XY", MAPF, C.N2 * 2, &mp));
        *dGS = g7;
        *dMAPF = mp;
    }
    return SCALE_HEVI_OK;
}

int ATMOS_DYN_Tstep_tracer_fvm_heve_b200_dev(SCALE_HEVI_TSTEP_TRACER_ARGS)
{
    const double *dGS, *dMAPF;
    CK(tracer_metrics(GSQRT, MAPF, true, &dGS, &dMAPF));
    // the 1-D vectors this step needs; the others keep their last values
    std::vector<double> one(C.g.KA > C.g.IA ? (C.g.KA > C.g.JA ? C.g.KA : C.g.JA) : (C.g.IA > C.g.JA ? C.g.IA : C.g.JA), 1.0);
    CK(prepare_tables(CDZ, one.data(), RCDZ, one.data(), one.data(), RCDX, one.data(), one.data(), RCDY, one.data(),
                      nullptr, nullptr, nullptr));
    TracerArgs a{};
    a.QTRCo = QTRCo; a.QTRC = QTRC; a.QTRC0 = QTRC0; a.RHOQ_t = RHOQ_t; a.DENS0 = DENS0; a.DENS = DENS;
    a.dens_mode = 0; a.mflx = mflx_hi; a.ndq = num_diff; a.dtl = *dtl;
    a.phi_lo = C.tr + 2 * C.N3; a.anti = C.tr + 3 * C.N3; a.rjp = C.tr + 6 * C.N3; a.rjm = C.tr + 7 * C.N3;
    a.along_stream = *FLAG_FCT_ALONG_STREAM ? 1 : 0;
    a.GS = dGS;
    a.MAPF = dMAPF;
    a.status = C.fct_fused ? C.status : nullptr;
    const bool fct = *FLAG_FCT_TRACER != 0;
    int hrc = SCALE_HEVI_OK, nk = 0;
    const HaloFill hf{hook_fill, &hrc};
    const cudaError_t e = launch_tracer_stage(C.g, a, C.scheme_tracer, fct, C.stream, C.halo_fn ? &hf : nullptr, &nk);
    if (hrc != SCALE_HEVI_OK) return hrc;
    CU(e);
    C.launches += nk;
    return SCALE_HEVI_OK;
}

int ATMOS_DYN_Tstep_tracer_fvm_heve_b200(SCALE_HEVI_TSTEP_TRACER_ARGS)
{
    const double *dGS, *dMAPF;
    CK(tracer_metrics(GSQRT, MAPF, false, &dGS, &dMAPF));
    const size_t N3 = n3();
    double *qo, *q, *q0, *rq, *d0, *d, *mf, *nd = nullptr;
    CK(h2d("q_out", QTRCo, N3, &qo));
    CK(h2d("q_in", QTRC, N3, &q));
    CK(h2d("q0", QTRC0, N3, &q0));
    CK(h2d("rhoq_t", RHOQ_t, N3, &rq));
    CK(h2d("DENS0", DENS0, N3, &d0));
    CK(h2d("DENS", DENS, N3, &d));
    CK(h2d("mflx", mflx_hi, 3 * N3, &mf));
    if (num_diff) CK(h2d("ndq", num_diff, 3 * N3, &nd));
    int rc = ATMOS_DYN_Tstep_tracer_fvm_heve_b200_dev(qo, q, (QTRC0 == QTRCo) ? qo : q0, rq, d0, d, mf, nd, dGS, dMAPF,
                                                      CDZ, RCDZ, RCDX, RCDY, dtl, FLAG_FCT_TRACER, FLAG_FCT_ALONG_STREAM);
    if (rc) return rc;
    CK(d2h(QTRCo, qo, N3));
    CU(cudaStreamSynchronize(C.stream));
    return SCALE_HEVI_OK;
}

int ATMOS_DYN_Tinteg_tracer_rk3_b200_dev(SCALE_HEVI_TINTEG_TRACER_ARGS)
{
    CK(check_bnd(BND_W, BND_E, BND_S, BND_N));
    const double *dGS, *dMAPF;
    CK(tracer_metrics(GSQRT, MAPF, true, &dGS, &dMAPF));
    if (dGS) { // run_tracer_rk3 takes the metrics of the call from the library state
        C.terrain = true;
        C.tm.GSQRT = dGS;
        C.tm.MAPF = dMAPF;
    }
    std::vector<double> one(C.g.KA > C.g.IA ? (C.g.KA > C.g.JA ? C.g.KA : C.g.JA) : (C.g.IA > C.g.JA ? C.g.IA : C.g.JA), 1.0);
    CK(prepare_tables(CDZ, one.data(), RCDZ, one.data(), one.data(), RCDX, one.data(), one.data(), RCDY, one.data(),
                      nullptr, nullptr, nullptr));
    return run_tracer_rk3(QTRC, QTRC0, RHOQ_t, DENS0, DENS, mflx_hi, num_diff, *dtl, *FLAG_FCT_TRACER != 0,
                          *FLAG_FCT_ALONG_STREAM != 0);
}

// the tracer RK3 with FP32 flux and limiter arithmetic (the tracer and the
// densities stay FP64); flat terrain
int ATMOS_DYN_Tinteg_tracer_rk3_b200_mixed_dev(SCALE_HEVI_TINTEG_TRACER_MIXED_ARGS)
{
    CK(check_bnd(BND_W, BND_E, BND_S, BND_N));
    const double *dGS, *dMAPF;
    CK(tracer_metrics(GSQRT, MAPF, true, &dGS, &dMAPF));
    if (dGS) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the mixed-precision tracer advection takes flat terrain only");
    if (!C.tr_f) CK(falloc(&C.tr_f, 6 * C.N3));
    std::vector<double> one(C.g.KA > C.g.IA ? (C.g.KA > C.g.JA ? C.g.KA : C.g.JA) : (C.g.IA > C.g.JA ? C.g.IA : C.g.JA), 1.0);
    CK(prepare_tables(CDZ, one.data(), RCDZ, one.data(), one.data(), RCDX, one.data(), one.data(), RCDY, one.data(),
                      nullptr, nullptr, nullptr));
    return run_tracer_rk3(QTRC, QTRC0, RHOQ_t, DENS0, DENS, mflx_hi, num_diff, *dtl, *FLAG_FCT_TRACER != 0,
                          *FLAG_FCT_ALONG_STREAM != 0);
}

int ATMOS_DYN_Tinteg_tracer_rk3_b200(SCALE_HEVI_TINTEG_TRACER_ARGS)
{
    CK(check_bnd(BND_W, BND_E, BND_S, BND_N));
    const double *dGS, *dMAPF;
    CK(tracer_metrics(GSQRT, MAPF, false, &dGS, &dMAPF));
    const size_t N3 = n3();
    double *q, *q0, *rq, *d0, *d, *mf, *nd = nullptr;
    CK(h2d("q_out", QTRC, N3, &q));
    CK(h2d("q0", QTRC0, N3, &q0));
    CK(h2d("rhoq_t", RHOQ_t, N3, &rq));
    CK(h2d("DENS0", DENS0, N3, &d0));
    CK(h2d("DENS", DENS, N3, &d));
    CK(h2d("mflx", mflx_hi, 3 * N3, &mf));
    if (num_diff) CK(h2d("ndq", num_diff, 3 * N3, &nd));
    int rc = ATMOS_DYN_Tinteg_tracer_rk3_b200_dev(q, (QTRC0 == QTRC) ? q : q0, rq, d0, d, mf, nd, dGS, dMAPF,
                                                  CDZ, RCDZ, RCDX, RCDY, BND_W, BND_E, BND_S, BND_N, dtl,
                                                  FLAG_FCT_TRACER, FLAG_FCT_ALONG_STREAM);
    if (rc) return rc;
    CK(d2h(QTRC, q, N3));
    CU(cudaStreamSynchronize(C.stream));
    return SCALE_HEVI_OK;
}

// ---- halo --------------------------------------------------------------------
// ---- divergence ------------------------------------------------------------------
int ATMOS_DYN_divergence_b200_dev(SCALE_HEVI_DIVERGENCE_ARGS)
{
    CK(need_single("the divergence"));
    if (!RCDZ || !RCDX || !RCDY || !FDZ) return fail(SCALE_HEVI_ERR_ARG, "a 1-D grid vector is NULL");
    bool flat = false;
    CK(metrics_flat(GSQRT, J13G, J23G, MAPF, true, &flat));
    C.terrain = false;
    if (!flat) {
        // terrain: the metric divergence (k_divergence_terrain), which reads the
        // library's 1-D tables; the vectors this entry does not take are ones there
        if (!GSQRT || !J13G || !J23G || !MAPF || !RFDZ)
            return fail(SCALE_HEVI_ERR_ARG, "terrain-following metrics need GSQRT, J13G, J23G, MAPF and RFDZ");
        const int n = C.g.KA > C.g.IA ? (C.g.KA > C.g.JA ? C.g.KA : C.g.JA) : (C.g.IA > C.g.JA ? C.g.IA : C.g.JA);
        std::vector<double> one(n, 1.0);
        CK(prepare_tables(one.data(), FDZ, RCDZ, RFDZ, one.data(), RCDX, one.data(), one.data(), RCDY, one.data(),
                          nullptr, nullptr, nullptr));
        C.terrain = true;
        C.tm = Metrics{GSQRT, J13G, J23G, MAPF, nullptr};
        return run_divergence(DDIV, MOMZ, MOMX, MOMY, C.g.RCDZ, C.g.RCDX, C.g.RCDY, *J33G);
    }
    const int KA = C.g.KA, IA = C.g.IA, JA = C.g.JA;
    double *t;
    CK(stage_buf("div_tab", (size_t)KA + IA + JA, &t));
    CU(cudaMemcpyAsync(t, RCDZ, KA * sizeof(double), cudaMemcpyHostToDevice, C.stream));
    CU(cudaMemcpyAsync(t + KA, RCDX, IA * sizeof(double), cudaMemcpyHostToDevice, C.stream));
    CU(cudaMemcpyAsync(t + KA + IA, RCDY, JA * sizeof(double), cudaMemcpyHostToDevice, C.stream));
    return run_divergence(DDIV, MOMZ, MOMX, MOMY, t, t + KA, t + KA + IA, *J33G);
}

int ATMOS_DYN_divergence_b200(SCALE_HEVI_DIVERGENCE_ARGS)
{
    CK(need_single("the divergence"));
    bool flat = false;
    CK(metrics_flat(GSQRT, J13G, J23G, MAPF, false, &flat));
    const double *dGS = nullptr, *dJ13 = nullptr, *dJ23 = nullptr, *dMAPF = nullptr;
    if (!flat) {
        if (!GSQRT || !J13G || !J23G || !MAPF)
            return fail(SCALE_HEVI_ERR_ARG, "terrain-following metrics need GSQRT, J13G, J23G and MAPF");
        double *g7, *j13, *j23, *mp;
        CK(h2d("GSQRT", GSQRT, 7 * C.N3, &g7));
        CK(h2d("J13G", J13G, 7 * C.N3, &j13));
        CK(h2d("J23G", J23G, 7 * C.N3, &j23));
        CK(h2d("MAPF", MAPF, C.N2 * 2 * 4, &mp));
        dGS = g7; dJ13 = j13; dJ23 = j23; dMAPF = mp;
    }
    const size_t N3 = n3();
    double *dd, *mz, *mx, *my;
    CK(h2d("DDIV", DDIV, N3, &dd)); // cells the divergence does not write keep their contents
    CK(h2d("x1", MOMZ, N3, &mz));
    CK(h2d("x2", MOMX, N3, &mx));
    CK(h2d("x3", MOMY, N3, &my));
    int rc = ATMOS_DYN_divergence_b200_dev(dd, mz, mx, my, dGS, dJ13, dJ23, J33G, dMAPF, RCDZ, RCDX, RCDY, RFDZ, FDZ);
    if (rc) return rc;
    CK(d2h(DDIV, dd, N3));
    CU(cudaStreamSynchronize(C.stream));
    return SCALE_HEVI_OK;
}

int COMM_vars8_b200_dev(double *var, const int *nfields)
{
    CK(need_setup());
    if (!var || !nfields || *nfields < 1) return fail(SCALE_HEVI_ERR_ARG, "COMM_vars8: bad field list");
    std::vector<double *> f(*nfields);
    for (int q = 0; q < *nfields; ++q) f[q] = var + (size_t)q * C.N3;
    return halo(f.data(), *nfields);
}

// ---- large step ----------------------------------------------------------------
#define SCALE_HEVI_LARGE_ARGS                                                                                      \
    double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT, double *QTRC, const int *QA,             \
        double *mflx_hi, double *tflx_hi, double *num_diff, const double *DENS_tp, const double *MOMZ_tp,          \
        const double *MOMX_tp, const double *MOMY_tp, const double *RHOT_tp, const double *RHOQ_tp,                \
        const double *CORIOLI, const double *CDZ, const double *CDX, const double *CDY, const double *FDZ,         \
        const double *FDX, const double *FDY, const double *RCDZ, const double *RCDX, const double *RCDY,          \
        const double *RFDZ, const double *RFDX, const double *RFDY, const double *PHI, const double *GSQRT,        \
        const double *J13G, const double *J23G, const double *J33G, const double *MAPF, const double *AQ_R,        \
        const double *AQ_CV, const double *AQ_CP, const double *AQ_MASS, const double *REF_dens,                   \
        const double *REF_pott, const double *REF_pres, const double *ND_COEF, const int *ND_ORDER,                \
        const double *ND_SFC_FACT, const int *ND_USE_RS, const double *wdamp_coef, const double *divdmp_coef,      \
        const int *FLAG_FCT_TRACER, const int *FLAG_FCT_ALONG_STREAM, const double *DTLS, const double *DTSS

// Copy/compute overlap of the host-array large step. The device body waits on
// in[g] before the first use of input group g (0: DENS RHOT QTRC REF_pres for
// the preparation; 1: MOMZ MOMX MOMY REF_dens REF_pott for the filter; 2: the
// tendencies and CORIOLI for the short steps; 3: RHOQ_tp for the tracers) and
// calls done() as soon as a group of outputs holds its final values (0:
// num_diff after the last filter; 1: the state and tflx_hi after the last
// short step; 2: mflx_hi; 3: tracer q after its advection and halo).
namespace {
struct LargeHooks {
    cudaEvent_t in[4] = {};
    std::function<int(int what, int q)> done;
};
}  // namespace

int ATMOS_DYN_Tstep_large_fvm_heve_b200_dev(SCALE_HEVI_LARGE_ARGS)
{
    (void)PHI;
    CK(need_single("the large step"));
    const int qa = *QA;
    if (qa < 0 || qa > 8) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "QA=%d (0..8 supported)", qa);
    if (*ND_COEF != 0.0 && (*ND_ORDER < 1 || *ND_ORDER > 8))
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "ND_ORDER=%d is not supported (1..8)", *ND_ORDER);
    if (*ND_COEF != 0.0 && !*ND_USE_RS) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "ND_USE_RS=.false. is not supported");
    CK(use_metrics(GSQRT, J13G, J23G, MAPF, PHI, true));
    const size_t N3 = C.N3;
    if (!C.lg) CK(dalloc(&C.lg, 8 * N3));
    if (!C.tr) CK(dalloc(&C.tr, 8 * N3));
    double *DENS00 = C.lg, *RT2P = C.lg + N3, *DPRES0 = C.lg + 2 * N3, *REF_rhot = C.lg + 3 * N3, *mflx_av = C.lg + 4 * N3;
    double *DDIV = C.lg + 7 * N3;
    const bool use_div = *divdmp_coef > 0.0;

    // time steps, :373-376
    double dts = *DTSS;
    const double dtl = *DTLS;
    const int nstep = (int)std::ceil((dtl - EPS) / dts);
    dts = dtl / nstep;

    LargeHooks *hk = C.large_hooks;
    auto wait_in = [&](int grp) -> int {
        if (hk && hk->in[grp]) CU(cudaStreamWaitEvent(C.stream, hk->in[grp], 0));
        return SCALE_HEVI_OK;
    };
    auto done = [&](int what, int q) -> int { return hk ? hk->done(what, q) : SCALE_HEVI_OK; };

    CK(wait_in(0));
    CU(cudaMemcpyAsync(DENS00, DENS, N3 * sizeof(double), cudaMemcpyDeviceToDevice, C.stream));
    CU(cudaMemsetAsync(mflx_av, 0, 3 * N3 * sizeof(double), C.stream));
    // RT2P / DPRES0 / REF_rhot, :428-470
    PrepArgs pa{};
    pa.RT2P = RT2P; pa.DPRES0 = DPRES0; pa.REF_rhot = REF_rhot; pa.RHOT = RHOT; pa.QTRC = QTRC; pa.REF_pres = REF_pres;
    pa.QA = qa;
    for (int q = 0; q < qa; ++q) { pa.AQ_R[q] = AQ_R[q]; pa.AQ_CV[q] = AQ_CV[q]; pa.AQ_CP[q] = AQ_CP[q]; pa.AQ_MASS[q] = AQ_MASS[q]; }
    CK(timed("large_prep", [&] { large_prep(C.g, pa, C.stream); return SCALE_HEVI_OK; }));
    C.launches += 2;
    CK(prepare_tables(CDZ, FDZ, RCDZ, RFDZ, FDX, RCDX, RFDX, FDY, RCDY, RFDY, wdamp_coef, CDX, CDY));
    if (*ND_COEF != 0.0) CK(prepare_nd(CDZ, CDX, CDY, FDZ, FDX, FDY, dts, *ND_COEF, *ND_ORDER, *ND_SFC_FACT));

    // With DAMP_alpha = 0 the tendencies of :606-839 equal the physics tendencies
    // *_tp on every cell the short step reads, so *_tp are passed directly.
    double *X[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    StageIn base{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                 DENS_tp, MOMZ_tp, MOMX_tp, MOMY_tp, RHOT_tp, DPRES0, RT2P, CORIOLI, num_diff, use_div ? DDIV : nullptr,
                 REF_dens, REF_rhot, use_div ? *divdmp_coef : 0.0, *J33G};
    for (int step = 1; step <= nstep; ++step) {
        if (step == 1) CK(wait_in(1));
        if (*ND_COEF == 0.0) CU(cudaMemsetAsync(num_diff, 0, 15 * N3 * sizeof(double), C.stream));
        else CK(run_numfilter(num_diff, DENS, MOMZ, MOMX, MOMY, RHOT, REF_dens, REF_pott));
        if (step == nstep) CK(done(0, 0));
        // divergence for the damping term, :860-871
        if (use_div) CK(run_divergence(DDIV, MOMZ, MOMX, MOMY, C.g.RCDZ, C.g.RCDX, C.g.RCDY, *J33G));
        if (step == 1) CK(wait_in(2));
        CK(run_short(X, mflx_hi, tflx_hi, base, dts));
        CK(timed("boundary", [&] { vertical_bc(C.g, mem(), DENS, MOMZ, MOMX, MOMY, RHOT, C.stream); return SCALE_HEVI_OK; }));
        ++C.launches;
        CK(halo(X, 5));
        CK(timed("mflx_average", [&] { mflx_accumulate(C.g, mflx_av, mflx_hi, C.stream); return SCALE_HEVI_OK; }));
        ++C.launches;
    }
    if (nstep < 1) CK(done(0, 0));
    CK(done(1, 0));
    if (qa > 0) {
        mflx_average(C.g, mflx_hi, mflx_av, nstep, C.stream);
        ++C.launches;
        double *mf[3] = {mflx_hi, mflx_hi + N3, mflx_hi + 2 * N3};
        CK(halo(mf, 3));
        CK(done(2, 0));
        CK(wait_in(3));
        for (int q = 0; q < qa; ++q) {
            double *qt = QTRC + (size_t)q * N3;
            CK(run_tracer_rk3<double>(qt, qt, RHOQ_tp + (size_t)q * N3, DENS00, DENS, mflx_hi, nullptr, dtl,
                              *FLAG_FCT_TRACER != 0, *FLAG_FCT_ALONG_STREAM != 0));
            CK(halo(&qt, 1));
            CK(done(3, q));
        }
    } else {
        CK(done(2, 0));
    }
    return SCALE_HEVI_OK;
}

// Host-array form: inputs are copied in on a second stream in the order the
// device body first needs them, and each group of outputs is copied back as
// soon as it is final, so that the copies overlap the kernels. Results are
// those of the device entry; the call returns when every copy has landed.
int ATMOS_DYN_Tstep_large_fvm_heve_b200(SCALE_HEVI_LARGE_ARGS)
{
    CK(need_single("the large step"));
    if (C.capturing) return fail(SCALE_HEVI_ERR_ARG, "the host-array large step cannot be captured");
    bool flat = false;
    CK(metrics_flat(GSQRT, J13G, J23G, MAPF, false, &flat));
    // terrain-following metrics go to the device with PHI; flat terrain needs neither
    const double *dGS = nullptr, *dJ13 = nullptr, *dJ23 = nullptr, *dMAPF = nullptr, *dPHI = PHI;
    if (!flat) {
        if (!GSQRT || !J13G || !J23G || !MAPF || !PHI)
            return fail(SCALE_HEVI_ERR_ARG, "terrain-following metrics need GSQRT, J13G, J23G, MAPF and PHI");
        double *g7, *j13, *j23, *mp, *ph;
        CK(h2d("GSQRT", GSQRT, 7 * C.N3, &g7));
        CK(h2d("J13G", J13G, 7 * C.N3, &j13));
        CK(h2d("J23G", J23G, 7 * C.N3, &j23));
        CK(h2d("MAPF", MAPF, C.N2 * 2 * 4, &mp));
        CK(h2d("PHI", PHI, C.N3, &ph));
        dGS = g7; dJ13 = j13; dJ23 = j23; dMAPF = mp; dPHI = ph;
    }
    const size_t N3 = n3(), N2 = (size_t)C.g.IA * C.g.JA;
    const int qa = *QA;
    if (qa < 0 || qa > 8) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "QA=%d (0..8 supported)", qa);
    if (!C.copy_stream) {
        CU(cudaStreamCreate(&C.copy_stream));
        for (cudaEvent_t &e : C.copy_ev) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    cudaStream_t cs = C.copy_stream;
    // the copies start after the work already queued on the library stream
    CU(cudaEventRecord(C.copy_ev[5], C.stream));
    CU(cudaStreamWaitEvent(cs, C.copy_ev[5], 0));

    double *X[5], *T[5], *q = nullptr, *rq = nullptr, *mf, *tf, *nd, *cor, *rd, *rp, *rpres;
    double *hx[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    const double *ht[5] = {DENS_tp, MOMZ_tp, MOMX_tp, MOMY_tp, RHOT_tp};
    static const char *n_x[5] = {"x0", "x1", "x2", "x3", "x4"}, *n_t[5] = {"t0", "t1", "t2", "t3", "t4"};
    LargeHooks hk;
    // group 0: DENS RHOT QTRC REF_pres
    CK(h2d(n_x[0], hx[0], N3, &X[0], cs));
    CK(h2d(n_x[4], hx[4], N3, &X[4], cs));
    if (qa > 0) CK(h2d("qtrc", QTRC, (size_t)qa * N3, &q, cs));
    CK(h2d("REF_pres", REF_pres, N3, &rpres, cs));
    CU(cudaEventRecord(C.copy_ev[0], cs));
    // group 1: MOMZ MOMX MOMY REF_dens REF_pott
    for (int v = 1; v < 4; ++v) CK(h2d(n_x[v], hx[v], N3, &X[v], cs));
    CK(h2d("REF_dens", REF_dens, N3, &rd, cs));
    CK(h2d("REF_pott", REF_pott, N3, &rp, cs));
    CU(cudaEventRecord(C.copy_ev[1], cs));
    // group 2: tendencies, CORIOLI
    for (int v = 0; v < 5; ++v) CK(h2d(n_t[v], ht[v], N3, &T[v], cs));
    CK(h2d("CORIOLI", CORIOLI, N2, &cor, cs));
    CU(cudaEventRecord(C.copy_ev[2], cs));
    // group 3: tracer tendencies
    if (qa > 0) {
        CK(h2d("rhoq_tp", RHOQ_tp, (size_t)qa * N3, &rq, cs));
        CU(cudaEventRecord(C.copy_ev[3], cs));
    }
    for (int g = 0; g < 4; ++g) hk.in[g] = (g < 3 || qa > 0) ? C.copy_ev[g] : nullptr;
    CK(stage_buf("mflx", 3 * N3, &mf));
    CK(stage_buf("tflx", 3 * N3, &tf));
    CK(stage_buf("num_diff", 15 * N3, &nd));
    hk.done = [&](int what, int iq) -> int {
        CU(cudaEventRecord(C.copy_ev[4], C.stream));
        CU(cudaStreamWaitEvent(cs, C.copy_ev[4], 0));
        switch (what) {
        case 0: return d2h(num_diff, nd, 15 * N3, cs);
        case 1:
            for (int v = 0; v < 5; ++v) CK(d2h(hx[v], X[v], N3, cs));
            return d2h(tflx_hi, tf, 3 * N3, cs);
        case 2: return d2h(mflx_hi, mf, 3 * N3, cs);
        default: return d2h(QTRC + (size_t)iq * N3, q + (size_t)iq * N3, N3, cs);
        }
    };
    C.large_hooks = &hk;
    int rc = ATMOS_DYN_Tstep_large_fvm_heve_b200_dev(
        X[0], X[1], X[2], X[3], X[4], q, QA, mf, tf, nd, T[0], T[1], T[2], T[3], T[4], rq, cor,
        CDZ, CDX, CDY, FDZ, FDX, FDY, RCDZ, RCDX, RCDY, RFDZ, RFDX, RFDY, dPHI, dGS, dJ13, dJ23, J33G, dMAPF,
        AQ_R, AQ_CV, AQ_CP, AQ_MASS, rd, rp, rpres, ND_COEF, ND_ORDER, ND_SFC_FACT, ND_USE_RS, wdamp_coef, divdmp_coef,
        FLAG_FCT_TRACER, FLAG_FCT_ALONG_STREAM, DTLS, DTSS);
    C.large_hooks = nullptr;
    // both streams drain before the host arrays are handed back, also on failure
    const cudaError_t e1 = cudaStreamSynchronize(cs), e2 = cudaStreamSynchronize(C.stream);
    if (rc) return rc;
    CU(e1);
    CU(e2);
    return scale_hevi_check();
}

int scale_hevi_boundary_dev(double *DENS, double *MOMZ, double *MOMX, double *MOMY, double *RHOT)
{
    CK(need_setup());
    CK(timed("boundary", [&] { vertical_bc(C.g, mem(), DENS, MOMZ, MOMX, MOMY, RHOT, C.stream); return SCALE_HEVI_OK; }));
    ++C.launches;
    double *X[5] = {DENS, MOMZ, MOMX, MOMY, RHOT};
    return halo(X, 5);
}

// ---- the differentiated short step ------------------------------------------------
int scale_hevi_adjoint_setup(const double *DPRES0, const double *RT2P, const double *REF_rhot, const double *REF_dens,
                             const double *REF_pott, const double *PHI, const double *CORIOLI, const double *CDZ,
                             const double *CDX, const double *CDY, const double *FDZ, const double *FDX,
                             const double *FDY, const double *RCDZ, const double *RCDX, const double *RCDY,
                             const double *RFDZ, const double *RFDX, const double *RFDY, const double *wdamp_coef,
                             const double *dt, const double *ND_COEF, const double *ND_SFC_FACT, const double *J33G)
{
    CK(need_single("the differentiated short step"));
    if (wide_scheme(C.scheme))
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the differentiated short step supports UD3, CD4, UD3KOREN1993 and CD2");
    if (C.short_type != 0) return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the differentiated short step is the HEVI step");
    if (C.tinteg_type != 0)
        return fail(SCALE_HEVI_ERR_UNSUPPORTED, "the differentiated short step is integrated with RK4");
    const double *v[12] = {CDZ, CDX, CDY, FDZ, FDX, FDY, RCDZ, RCDX, RCDY, RFDZ, RFDX, RFDY};
    const int len[12] = {C.g.KA, C.g.IA, C.g.JA, C.g.KA - 1, C.g.IA - 1, C.g.JA - 1,
                         C.g.KA, C.g.IA, C.g.JA, C.g.KA - 1, C.g.IA - 1, C.g.JA - 1};
    for (int q = 0; q < 12; ++q) {
        if (!v[q]) return fail(SCALE_HEVI_ERR_ARG, "a 1-D grid vector is NULL");
        C.ad_vec[q].assign(v[q], v[q] + len[q]);
    }
    if (!DPRES0 || !RT2P || !REF_rhot || !REF_dens || !REF_pott || !PHI || !CORIOLI || !dt || !ND_COEF || !ND_SFC_FACT || !J33G)
        return fail(SCALE_HEVI_ERR_ARG, "an argument of the differentiated short step is NULL");
    C.ad_wdamp.assign((size_t)C.g.KA, 0.0);
    if (wdamp_coef) C.ad_wdamp.assign(wdamp_coef, wdamp_coef + C.g.KA);
    C.ad_ndcoef = *ND_COEF;
    C.ad_sfc = *ND_SFC_FACT;
    const size_t N3 = C.N3;
    if (!C.ad_scratch) {
        CK(dalloc(&C.ad_scratch, ad::scratch_fields() * N3));
        CK(dalloc(&C.ad_zero, N3));
        CK(dalloc(&C.ad_nd, 15 * N3));
        CK(dalloc(&C.ad_flx, 6 * N3));
        CU(cudaMemsetAsync(C.ad_scratch, 0, ad::scratch_fields() * N3 * sizeof(double), C.stream));
        CU(cudaMemsetAsync(C.ad_zero, 0, N3 * sizeof(double), C.stream));
        CU(cudaMemsetAsync(C.ad_nd, 0, 15 * N3 * sizeof(double), C.stream));
    }
    ad::Model &M = C.adm;
    M.dt = *dt;
    M.J33G = *J33G;
    M.status = C.status;
    M.DPRES0 = DPRES0; M.RT2P = RT2P; M.REF_rhot = REF_rhot; M.REF_dens = REF_dens; M.REF_pott = REF_pott;
    M.PHI = PHI; M.CORIOLI = CORIOLI; M.zero = C.ad_zero; M.scratch = C.ad_scratch;
    M.scheme = C.scheme;
    M.stream = C.stream;
    C.ad_ready = true;
    return SCALE_HEVI_OK;
}

// tables of the differentiated model (cached: no transfer unless they changed)
static int ad_prepare()
{
    CK(need_single("the differentiated short step"));
    if (!C.ad_ready) return fail(SCALE_HEVI_ERR_NOT_SETUP, "scale_hevi_adjoint_setup() has not been called");
    C.terrain = false; // the differentiated model is the flat-terrain step
    const auto &v = C.ad_vec;
    CK(prepare_tables(v[0].data(), v[3].data(), v[6].data(), v[9].data(), v[4].data(), v[7].data(), v[10].data(),
                      v[5].data(), v[8].data(), v[11].data(), C.ad_wdamp.data(), nullptr, nullptr));
    CK(prepare_nd(v[0].data(), v[1].data(), v[2].data(), v[3].data(), v[4].data(), v[5].data(), C.adm.dt, C.ad_ndcoef, 1,
                  C.ad_sfc));
    C.adm.g = C.g;
    C.adm.nd = C.ndc;
    C.adm.wdamp = C.d_wdamp;
    return SCALE_HEVI_OK;
}

int scale_hevi_short_step_dev(double *X)
{
    CK(ad_prepare());
    const size_t N3 = C.N3;
    double *Xv[5] = {X, X + N3, X + 2 * N3, X + 3 * N3, X + 4 * N3};
    const ad::Model &M = C.adm;
    CK(run_numfilter<double>(C.ad_nd, Xv[0], Xv[1], Xv[2], Xv[3], Xv[4], M.REF_dens, M.REF_pott));
    StageIn base{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                 M.zero, M.zero, M.zero, M.zero, M.zero, M.DPRES0, M.RT2P, M.CORIOLI, C.ad_nd, nullptr, M.REF_dens,
                 M.REF_rhot, 0.0, M.J33G};
    CK(run_rk4(Xv, C.ad_flx, C.ad_flx + 3 * N3, base, M.dt));
    return scale_hevi_boundary_dev(Xv[0], Xv[1], Xv[2], Xv[3], Xv[4]);
}

int scale_hevi_short_step_passes_dev(double *X)
{
    CK(ad_prepare());
    CU(ad::step_forward(C.adm, X));
    return SCALE_HEVI_OK;
}

int scale_hevi_short_step_tlm_dev(double *X, double *dX)
{
    CK(ad_prepare());
    if (!X || !dX) return fail(SCALE_HEVI_ERR_ARG, "X or dX is NULL");
    CU(ad::step_tlm(C.adm, X, dX));
    return SCALE_HEVI_OK;
}

int scale_hevi_short_step_dd_dev(double *X_hi, double *X_lo)
{
    CK(ad_prepare());
    if (!X_hi || !X_lo) return fail(SCALE_HEVI_ERR_ARG, "X_hi or X_lo is NULL");
    CU(ad::step_dd(C.adm, X_hi, X_lo));
    return SCALE_HEVI_OK;
}

int scale_hevi_short_step_adjoint_dev(const double *X, double *lam)
{
    CK(ad_prepare());
    if (!X || !lam) return fail(SCALE_HEVI_ERR_ARG, "X or lam is NULL");
    CU(ad::step_adjoint(C.adm, X, lam));
    return SCALE_HEVI_OK;
}

int scale_hevi_boundary_adjoint_dev(double *lam)
{
    CK(ad_prepare());
    CU(ad::boundary_adjoint(C.adm, lam));
    return SCALE_HEVI_OK;
}

int scale_hevi_capture_begin(void)
{
    CK(need_setup());
    if (C.capturing) return fail(SCALE_HEVI_ERR_ARG, "a capture is already open");
    if (C.prof_on) return fail(SCALE_HEVI_ERR_ARG, "section timers are on; turn them off before a capture");
    CU(cudaStreamSynchronize(C.stream));
    CU(cudaStreamBeginCapture(C.stream, cudaStreamCaptureModeThreadLocal));
    C.capturing = true;
    C.capture_from = C.launches;
    return SCALE_HEVI_OK;
}

int scale_hevi_capture_end(void)
{
    CK(need_setup());
    if (!C.capturing) return fail(SCALE_HEVI_ERR_ARG, "no capture is open");
    C.capturing = false;
    const long long recorded = C.launches - C.capture_from;
    C.launches = C.capture_from; // recorded, not launched
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(C.stream, &graph);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(SCALE_HEVI_ERR_CUDA,
                    "the capture failed (%s): a call inside it synchronised or allocated; warm up with one eager call first",
                    cudaGetErrorString(e));
    }
    if (C.graph_exec) {
        cudaGraphExecDestroy(C.graph_exec);
        C.graph_exec = nullptr;
    }
    e = cudaGraphInstantiate(&C.graph_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(SCALE_HEVI_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    C.graph_launches = recorded;
    return SCALE_HEVI_OK;
}

int scale_hevi_replay(const int *n)
{
    CK(need_setup());
    if (!C.graph_exec) return fail(SCALE_HEVI_ERR_ARG, "nothing has been captured");
    for (int q = 0; q < (n ? *n : 1); ++q) {
        CU(cudaGraphLaunch(C.graph_exec, C.stream));
        C.launches += C.graph_launches;
    }
    return SCALE_HEVI_OK;
}

const char *scale_hevi_autotune_report(void) { return C.tune_text.c_str(); }

int scale_hevi_profile(int enable)
{
    CK(need_setup());
    CU(cudaStreamSynchronize(C.stream));
    C.prof_on = enable != 0;
    C.ev_used = 0;
    C.prof_marks.clear();
    return SCALE_HEVI_OK;
}

const char *scale_hevi_profile_report(void)
{
    C.prof_text = "{";
    if (C.ready && cudaStreamSynchronize(C.stream) == cudaSuccess) {
        std::map<std::string, std::pair<long, double>> acc;
        for (auto &m : C.prof_marks) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, C.ev_pool[m.second], C.ev_pool[m.second + 1]);
            auto &a = acc[m.first];
            a.first += 1;
            a.second += ms;
        }
        bool first = true;
        for (auto &kv : acc) {
            char buf[256];
            snprintf(buf, sizeof buf, "%s\"%s\": [%ld, %.6f]", first ? "" : ", ", kv.first.c_str(), kv.second.first, kv.second.second);
            C.prof_text += buf;
            first = false;
        }
    }
    C.prof_text += "}";
    return C.prof_text.c_str();
}

int scale_hevi_energy_sum_dev(const double *DENS, const double *MOMZ, const double *MOMX, const double *MOMY,
                              const double *RHOT, const double *CZ, const double *CDZ, const double *CDX,
                              const double *CDY, double *totals)
{
    CK(need_single("the energy budget"));
    if (!DENS || !MOMZ || !MOMX || !MOMY || !RHOT || !CZ || !CDZ || !CDX || !CDY || !totals)
        return fail(SCALE_HEVI_ERR_ARG, "scale_hevi_energy_sum_dev: a NULL argument");
    const int KA = C.g.KA, IA = C.g.IA, JA = C.g.JA;
    const size_t ncol = (size_t)C.g.IMAX * C.g.JMAX;
    if (!C.eng_part) CK(dalloc(&C.eng_part, 4 * ncol + 4));
    std::vector<double> h(2 * (size_t)KA + IA + JA);
    std::memcpy(h.data(), CDZ, KA * sizeof(double));
    std::memcpy(h.data() + KA, CDX, IA * sizeof(double));
    std::memcpy(h.data() + KA + IA, CDY, JA * sizeof(double));
    std::memcpy(h.data() + KA + IA + JA, CZ, KA * sizeof(double));
    double *d;
    CK(stage_buf("energy_grid", h.size(), &d));
    CU(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, C.stream));
    energy_sum(C.g, DENS, MOMZ, MOMX, MOMY, RHOT, d + KA + IA + JA, d + KA, d + KA + IA, d, C.eng_part,
               C.eng_part + 4 * ncol, C.stream);
    C.launches += 5;
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(totals, C.eng_part + 4 * ncol, 4 * sizeof(double), cudaMemcpyDeviceToHost, C.stream));
    CU(cudaStreamSynchronize(C.stream));
    return SCALE_HEVI_OK;
}

int scale_hevi_domain_sum_dev(const double *var, const double *CDZ, const double *CDX, const double *CDY, double *total)
{
    CK(need_single("the domain sum"));
    const int KA = C.g.KA, IA = C.g.IA, JA = C.g.JA;
    std::vector<double> h(KA + IA + JA);
    std::memcpy(h.data(), CDZ, KA * sizeof(double));
    std::memcpy(h.data() + KA, CDX, IA * sizeof(double));
    std::memcpy(h.data() + KA + IA, CDY, JA * sizeof(double));
    double *d;
    CK(stage_buf("sum_grid", h.size(), &d));
    CU(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, C.stream));
    domain_sum(C.g, var, d + KA, d + KA + IA, d, C.sum_part, C.sum_out, C.stream);
    C.launches += 2;
    CU(cudaMemcpyAsync(total, C.sum_out, sizeof(double), cudaMemcpyDeviceToHost, C.stream));
    CU(cudaStreamSynchronize(C.stream));
    return SCALE_HEVI_OK;
}

}  // extern "C"
