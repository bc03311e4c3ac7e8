// cdd_stress_noalloc: the internal-stress solve of cdd_stress for one instance, for callers that
// cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not allowed or not wanted -- a host framework
// that owns all device memory through its own allocator and forbids libraries from allocating
// behind its back, or a long-running service that must not grow its device memory after start-up
// (an allocation there can fail late, or stall every stream while the driver maps memory). Such a
// caller cannot create a cdd_plan (plan creation allocates its scratch), so this entry point
// keeps its scratch in a fixed array inside the library instead.
//
// The scratch is one file-scope device array of CDD_STRESS_NOALLOC_MAX_BYTES. Every GPU that
// loads the library holds it until the process exits. Host code may not use the array's name as a
// device address (on the host it only names a stand-in), so the first call on each device, with that
// device current, looks the address up once with cudaGetSymbolAddress and caches it; that first
// call should come before any stream capture. The cached address belongs to the device's primary
// context: after a cudaDeviceReset in the same process it is stale, as every other device pointer
// is. Nothing here calls cudaMalloc, cudaFree or any allocating library routine. Each call copies
// its small tables (FFT twiddles, k tables, launch description) from a host buffer of the call
// into the front of the scratch with one cudaMemcpyAsync.
//
// Every call shares the one array and it keeps the last call's contents; calls that overlap on
// the GPU (different streams or threads) race on it and must be serialised by the caller. Each
// call writes every scratch byte it later reads (tables, row sums, spectra) before reading it,
// so nothing has to start at zero.
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "cdd_internal.cuh"

namespace cdd {
int report_error(int code, const char* msg);   // plan.cu
}

using namespace cdd;

static __device__ __align__(256) unsigned char g_stress_scratch[CDD_STRESS_NOALLOC_MAX_BYTES];

namespace {

constexpr int MAX_DEVICES = 64;
std::mutex g_mutex;
unsigned char* g_scratch_ptr[MAX_DEVICES] = {nullptr};

int err(int code, const std::string& m) { return report_error(code, m.c_str()); }

bool na_factor(int n, int& a, int& b, int& c) {
    a = b = c = 0;
    while (n % 2 == 0) { n /= 2; ++a; }
    while (n % 3 == 0) { n /= 3; ++b; }
    while (n % 5 == 0) { n /= 5; ++c; }
    return n == 1;
}

bool na_line_plan(int n, LinePlan& lp) {
    int a, b, c;
    if (!na_factor(n, a, b, c) || a < 1) return false;
    std::memset(&lp, 0, sizeof lp);
    lp.n = n;
    std::vector<int> r;
    int q = a / 4, m = a % 4;
    if (m == 1 && q > 0) { q -= 1; m = 5; }
    for (int i = 0; i < q; ++i) r.push_back(16);
    if (m == 1) r.push_back(2);
    else if (m == 2) r.push_back(4);
    else if (m == 3) r.push_back(8);
    else if (m == 5) { r.push_back(8); r.push_back(4); }
    for (int i = 0; i < b; ++i) r.push_back(3);
    for (int i = 0; i < c; ++i) r.push_back(5);
    if ((int)r.size() > MAX_STAGES) return false;
    lp.nst = (int)r.size();
    int ns = 1;
    for (int i = 0; i < lp.nst; ++i) {
        lp.radix[i] = r[i];
        lp.nr[i] = fdiv_make(n / r[i]);
        lp.ns[i] = fdiv_make(ns);
        ns *= r[i];
    }
    return true;
}

// exp(-2 pi i k / n) from long-double cos/sin of the angle reduced to its first-octant offset.
void na_twiddle(int n, int k, double& re, double& im) {
    const long double PI = 3.141592653589793238462643383279502884L;
    const long double r2 = 0.707106781186547524400844362104849039L;
    k %= n;
    long long k8 = 8LL * k, q = k8 / n, rem8 = k8 - q * n;
    long double t = (long double)rem8 / (long double)n * (PI / 4.0L);
    long double ct = cosl(t), st = sinl(t), cr, ci;
    switch (q) {
        case 0: cr = ct; ci = st; break;
        case 1: cr = r2 * (ct - st); ci = r2 * (ct + st); break;
        case 2: cr = -st; ci = ct; break;
        case 3: cr = -r2 * (ct + st); ci = r2 * (ct - st); break;
        case 4: cr = -ct; ci = -st; break;
        case 5: cr = -r2 * (ct - st); ci = -r2 * (ct + st); break;
        case 6: cr = st; ci = -ct; break;
        default: cr = r2 * (ct + st); ci = -r2 * (ct - st); break;
    }
    re = (double)cr;
    im = (double)(-ci);
}

double na_k(int n_scale, int n_axis, int i) {
    double a = 2.0 * M_PI * (double)i / (double)n_axis;
    if (a > M_PI) a = a - 2 * M_PI;
    return (double)n_scale * a;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

extern "C" int cdd_stress_noalloc(const cdd_instance* d, int precision, const void* beta, void* sigma6,
                                  void* stream) {
    if (!d || !beta || !sigma6) return err(CDD_ERR_ARG, "cdd_stress_noalloc: null argument");
    if (precision != CDD_F64 && precision != CDD_F32)
        return err(CDD_ERR_ARG, "cdd_stress_noalloc: bad precision");
    if (d->ndim != 2 && d->ndim != 3) return err(CDD_ERR_SHAPE, "cdd_stress_noalloc: ndim must be 2 or 3");
    int sh[3] = {d->shape[0], d->shape[1], d->ndim == 3 ? d->shape[2] : 1};
    for (int a = 0; a < d->ndim; ++a) {
        int A, B, C;
        if (sh[a] < 4 || sh[a] > 1024 || sh[a] % 2 || !na_factor(sh[a], A, B, C) || (B > 0 && C > 0))
            return err(CDD_ERR_SHAPE, "cdd_stress_noalloc: axis size " + std::to_string(sh[a]) +
                                          " unsupported (even, 4..1024, 2^a 3^b or 2^a 5^c)");
    }
    if (!(d->mu > 0) || !(d->nu < 0.5) || !(d->nu > -1.0))
        return err(CDD_ERR_ARG, "cdd_stress_noalloc: need mu > 0 and -1 < nu < 0.5");
    const bool f64 = (precision == CDD_F64);
    const size_t elt = f64 ? sizeof(double) : sizeof(float), velt = 2 * elt;

    // ---------------- instance description (one instance, offsets 0) ----------------
    InstDev I;
    std::memset(&I, 0, sizeof I);
    I.nd = d->ndim;
    I.n0 = sh[0]; I.n1 = sh[1]; I.n2 = sh[2];
    I.nl = (I.nd == 3) ? I.n2 : I.n1;
    I.nh = I.nl / 2 + 1;
    I.nhp = (I.nh + 7) & ~7;
    I.fd_nl = fdiv_make(I.nl);
    I.fd_nh = fdiv_make(I.nh);
    I.cells = (long long)I.n0 * I.n1 * I.n2;
    I.rows = (int)(I.cells / I.nl);
    I.fd_rows = fdiv_make(I.rows);
    I.mu = d->mu;
    I.nu = d->nu;
    I.lamb = 2. * d->mu * d->nu / (1. - 2. * d->nu);
    I.inv_cells = 1.0 / (double)I.cells;
    std::vector<double> twre, twim, ktab;
    std::map<int, LinePlan> lp_done;
    LinePlan* lps[3] = {&I.lp_last, &I.lp_mid, &I.lp_first};
    int lens[3] = {I.nl, I.nd == 3 ? I.n1 : I.n0, I.n0};
    for (int k = 0; k < 3; ++k) {
        if (!na_line_plan(lens[k], *lps[k]))
            return err(CDD_ERR_SHAPE, "cdd_stress_noalloc: no FFT plan for length " + std::to_string(lens[k]));
        auto it = lp_done.find(lens[k]);
        if (it == lp_done.end()) {
            lps[k]->tw = (int)twre.size();
            for (int j = 0; j < lens[k]; ++j) {
                double re, im;
                na_twiddle(lens[k], j, re, im);
                twre.push_back(re);
                twim.push_back(im);
            }
            append_stage_twiddles(*lps[k], twre, twim);
            it = lp_done.emplace(lens[k], *lps[k]).first;
        }
        *lps[k] = it->second;
    }
    if (I.nd == 3) {
        I.koff0 = (int)ktab.size();
        for (int a = 0; a < I.n0; ++a) ktab.push_back(na_k(I.n0, I.n0, a));
        I.koff1 = (int)ktab.size();
        for (int a = 0; a < I.n1; ++a) ktab.push_back(na_k(I.n1, I.n1, a));
        I.koffh = (int)ktab.size();
        for (int a = 0; a < I.nh; ++a) ktab.push_back(na_k(I.n2, I.n2, a));
    } else {
        I.koff0 = (int)ktab.size();
        for (int a = 0; a < I.n0; ++a) ktab.push_back(na_k(I.n1, I.n0, a));
        I.koff1 = I.koff0;
        I.koffh = (int)ktab.size();
        for (int a = 0; a < I.nh; ++a) ktab.push_back(na_k(I.n1, I.n1, a));
    }

    // ---------------- launch shapes (same tiling as the plan path) ----------------
    PlanCore P;
    P.n_inst = 1;
    P.precision = precision;
    P.any3d = (I.nd == 3);
    size_t smem_need = 48 * 1024;
    int blocks[NUM_PASSES] = {0, 0, 0, 0, 0};
    for (int k : {PASS_R2C, PASS_C2R}) {
        const int comps = 6;
        long long npairs = ((long long)comps * I.rows + 1) / 2;
        const size_t line_bytes = (size_t)(I.nl + (I.nl >> 4) + 1) * velt;
        int Pl = (velt == 8 ? 4096 : 2048) / I.nl;
        if (Pl < 1) Pl = 1;
        if (Pl > npairs) Pl = (int)npairs;
        PassTile& t = I.tile[k];
        t.lines = Pl;
        t.threads = (velt == 8) ? 256 : 128;
        t.blocks = (int)((npairs + Pl - 1) / Pl);
        t.tiles_a = 1;
        P.pass[k].threads = t.threads;
        P.pass[k].smem = ((2 * (size_t)Pl * (line_bytes / velt) + 1) & ~(size_t)1) * velt +
                         (size_t)I.lp_last.twspan * velt + rows_table_bytes(Pl);
    }
    for (int k : {PASS_MID_F, PASS_MID_I}) {
        PassTile& t = I.tile[k];
        P.pass[k].threads = 256;
        if (I.nd != 3) continue;
        const int comps = 6;
        int W = (int)(128 / velt);
        while (W > 1 && 2 * (size_t)W * I.n1 * velt > 96 * 1024) W >>= 1;
        t.lines = W;
        while ((1 << t.lgw) < W) ++t.lgw;
        t.threads = 256;
        t.tiles_a = (I.nh + W - 1) / W;
        t.blocks = comps * I.n0 * t.tiles_a;
        P.pass[k].smem = ((line_plan_io(I.lp_mid) && I.lp_mid.nst == 2) ? 1 : 2) * (size_t)W * I.n1 * velt +
                         (size_t)I.lp_mid.twspan * velt;
    }
    {
        PassTile& t = I.tile[PASS_GREEN];
        int W = (int)(32 / velt);
        while (W > 1 && (size_t)9 * (I.n0 * W + W) * velt > 100 * 1024) W >>= 1;
        if ((size_t)9 * (I.n0 * W + W) * velt > 220 * 1024)
            return err(CDD_ERR_SHAPE, "cdd_stress_noalloc: axis-0 length too large for the k-space pass");
        t.lines = W;
        while ((1 << t.lgw) < W) ++t.lgw;
        t.threads = 256;
        t.tiles_a = (I.nh + W - 1) / W;
        t.blocks = (I.nd == 3 ? I.n1 : 1) * t.tiles_a;
        P.pass[PASS_GREEN].threads = 256;
        P.pass[PASS_GREEN].smem = ((size_t)9 * (I.n0 * W + W) + 1) / 2 * 2 * velt + (size_t)I.lp_first.twspan * velt;
    }
    for (int k = 0; k < NUM_PASSES; ++k) {
        blocks[k] = I.tile[k].blocks;
        P.pass[k].blocks = blocks[k];
        if (P.pass[k].smem > smem_need) smem_need = P.pass[k].smem;
    }

    // ---------------- scratch layout and capacity ----------------
    const size_t off_inst = 0;
    const size_t off_pre = align256(off_inst + sizeof(InstDev));
    const size_t off_tw = align256(off_pre + sizeof(int) * 2 * NUM_PASSES);
    const size_t off_k = align256(off_tw + velt * twre.size());
    const size_t off_rs = align256(off_k + elt * ktab.size());
    const size_t off_sbar = align256(off_rs + (f64 ? 0 : sizeof(double) * 9 * (size_t)I.rows));
    const size_t off_spec = align256(off_sbar + sizeof(double) * 9);
    const size_t total = off_spec + velt * 9 * (size_t)I.rows * I.nhp;
    if (total > (size_t)CDD_STRESS_NOALLOC_MAX_BYTES)
        return err(CDD_ERR_SHAPE, "cdd_stress_noalloc: grid needs " + std::to_string(total) +
                                      " bytes of scratch, the fixed scratch holds " +
                                      std::to_string((size_t)CDD_STRESS_NOALLOC_MAX_BYTES) +
                                      "; use a cdd_plan for this size");

    // ---------------- once per device: the scratch array's device address ----------------
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return err(CDD_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= MAX_DEVICES) return err(CDD_ERR_ARG, "cdd_stress_noalloc: device ordinal out of range");
    unsigned char* base;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_stress_scratch);
            if (e != cudaSuccess || !p)
                return err(CDD_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            g_scratch_ptr[dev] = (unsigned char*)p;
        }
        base = g_scratch_ptr[dev];
    }
    int optin = 0;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess)
        return err(CDD_ERR_CUDA, std::string("cudaDeviceGetAttribute(shared memory): ") + cudaGetErrorString(e));
    if (smem_need > (size_t)optin) return err(CDD_ERR_SHAPE, "cdd_stress_noalloc: shared memory need exceeds the device limit");
    // raise (never lower) the kernels' dynamic shared-memory limit: plans launch the same kernels
    e = stress_set_attributes(precision, (size_t)optin);
    if (e != cudaSuccess) return err(CDD_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));

    // ---------------- tables: one host->device copy into the scratch ----------------
    std::vector<unsigned char> host(off_spec, 0);
    std::memcpy(host.data() + off_inst, &I, sizeof(InstDev));
    int pre[NUM_PASSES][2];
    for (int k = 0; k < NUM_PASSES; ++k) { pre[k][0] = 0; pre[k][1] = blocks[k]; }
    std::memcpy(host.data() + off_pre, pre, sizeof pre);
    for (size_t j = 0; j < twre.size(); ++j) {
        if (f64) {
            double2 v = make_double2(twre[j], twim[j]);
            std::memcpy(host.data() + off_tw + j * velt, &v, velt);
        } else {
            float2 v = make_float2((float)twre[j], (float)twim[j]);
            std::memcpy(host.data() + off_tw + j * velt, &v, velt);
        }
    }
    for (size_t j = 0; j < ktab.size(); ++j) {
        if (f64) std::memcpy(host.data() + off_k + j * elt, &ktab[j], elt);
        else { float v = (float)ktab[j]; std::memcpy(host.data() + off_k + j * elt, &v, elt); }
    }
    cudaStream_t st = (cudaStream_t)stream;
    e = cudaMemcpyAsync(base, host.data(), off_spec, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return err(CDD_ERR_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));

    P.d_inst = (InstDev*)(base + off_inst);
    for (int k = 0; k < NUM_PASSES; ++k) P.pass[k].d_pre = (int*)(base + off_pre) + 2 * k;
    P.d_tw = base + off_tw;
    P.d_k = base + off_k;
    P.d_rowsum = f64 ? nullptr : (double*)(base + off_rs);
    P.d_sbar = (double*)(base + off_sbar);
    P.d_spec = base + off_spec;
    e = launch_stress(P, beta, sigma6, st);
    if (e != cudaSuccess) return err(CDD_ERR_CUDA, std::string("stress launch: ") + cudaGetErrorString(e));
    return CDD_OK;
}
