// Plan construction and the C ABI of libcdd (see include/cdd.h).
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "cdd_internal.cuh"

using namespace cdd;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CDD_CUDA(call)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(CDD_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));       \
    } while (0)

// ------------------------------------------------------------------------------------------
// FFT length plans
// ------------------------------------------------------------------------------------------
bool factor(int n, int& a, int& b, int& c) {
    a = b = c = 0;
    while (n % 2 == 0) { n /= 2; ++a; }
    while (n % 3 == 0) { n /= 3; ++b; }
    while (n % 5 == 0) { n /= 5; ++c; }
    return n == 1;
}

// Radix sequence for length n = 2^a 3^b 5^c: stages of radix maxr = 2^e (16, 8 or 4) for the
// power of two, the remainder as one smaller power-of-two stage (a radix-2 remainder after a
// larger stage is folded into a (maxr/2, 4) pair), then radix 3 and radix 5 stages.
bool make_line_plan(int n, LinePlan& lp, int maxr = 16) {
    int a, b, c;
    if (!factor(n, a, b, c) || a < 1) return false;
    std::memset(&lp, 0, sizeof lp);
    lp.n = n;
    const int e = (maxr == 4) ? 2 : (maxr == 8) ? 3 : 4;
    std::vector<int> r;
    int q = a / e, m = a % e;
    bool fold = (m == 1 && q > 0 && e >= 3);
    if (fold) q -= 1;
    for (int i = 0; i < q; ++i) r.push_back(1 << e);
    if (fold) { r.push_back(1 << (e - 1)); r.push_back(4); }
    else if (m > 0) r.push_back(1 << m);
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

// w_n^k = exp(-2 pi i k / n): cosl/sinl of the exact angle in long double, reduced to the first
// octant by the symmetries of the unit circle so that the table is exactly symmetric.
void twiddle(int n, int k, long double& re, long double& im) {
    const long double PI = 3.141592653589793238462643383279502884L;
    k %= n;
    // angle = 2 pi k / n; use the octant index of 8k/n
    long long k8 = 8LL * k;
    long long q = k8 / n;              // octant 0..7
    long long rem8 = k8 - q * n;       // 8k mod n, in [0, n)
    // angle = (q + rem8/n) * pi/4 ; t = rem8 / n * pi/4 in [0, pi/4)
    long double t = (long double)rem8 / (long double)n * (PI / 4.0L);
    long double ct = cosl(t), st = sinl(t);
    long double cr, ci;   // cos and sin of the full angle
    const long double r2 = 0.707106781186547524400844362104849039L;
    switch (q) {
        case 0: cr = ct; ci = st; break;
        case 1: cr = r2 * (ct - st); ci = r2 * (ct + st); break;   // pi/4 + t
        case 2: cr = -st; ci = ct; break;
        case 3: cr = -r2 * (ct + st); ci = r2 * (ct - st); break;  // 3pi/4 + t
        case 4: cr = -ct; ci = -st; break;
        case 5: cr = -r2 * (ct - st); ci = -r2 * (ct + st); break;
        case 6: cr = st; ci = -ct; break;
        default: cr = r2 * (ct + st); ci = -r2 * (ct - st); break;
    }
    re = cr;
    im = -ci;
}

// k_d = n_scale * identity(2 pi i / n_axis), identity wrapping angles above pi by -2 pi
// (FourierSpaceTools.py L5-7, L29-49), evaluated with the same double operations as the reference.
double k_value(int n_scale, int n_axis, int i) {
    double a = 2.0 * M_PI * (double)i / (double)n_axis;
    if (a > M_PI) a = a - 2 * M_PI;
    return (double)n_scale * a;
}

// The 'sinK' tables, FourierSpaceTools(gridShape, func=sin): n_scale * sin(2 pi i / n_axis).
double k_value_sin(int n_scale, int n_axis, int i) {
    return (double)n_scale * std::sin(2.0 * M_PI * (double)i / (double)n_axis);
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {}
};

}  // namespace

struct cdd_plan {
    PlanCore core;
    std::vector<InstDev> inst;
    std::vector<cdd_instance> desc;
    long long scratch_bytes = 0;
    std::vector<void*> allocs;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    const void* graph_beta = nullptr;
    const void* graph_vac = nullptr;
    int device = 0;
    StencilMapSet maps_f0, maps_f1, maps_user;   // tensor maps of the stage inputs
    const void* maps_user_ptr = nullptr;
    std::vector<cdd_tuning> tune;                 // requested (zeros: built-in), then effective
};

namespace {

cudaError_t dalloc(cdd_plan* p, void** ptr, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e == cudaSuccess) {
        p->allocs.push_back(*ptr);
        p->scratch_bytes += (long long)bytes;
    }
    return e;
}

void free_plan(cdd_plan* p) {
    if (!p) return;
    if (p->graph) cudaGraphExecDestroy(p->graph);
    if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
    for (void* a : p->allocs) cudaFree(a);
    delete p;
}

int build_shapes(cdd_plan* p, size_t elt) {
    PlanCore& C = p->core;
    const int n = C.n_inst;
    const size_t velt = 2 * elt;
    std::vector<int> pre[NUM_PASSES];
    std::vector<int> pre_st, pre_cw, pre_ob;
    for (int k = 0; k < NUM_PASSES; ++k) pre[k].push_back(0);
    pre_st.push_back(0);
    pre_cw.push_back(0);
    pre_ob.push_back(0);
    size_t smem_max[NUM_PASSES] = {0, 0, 0, 0, 0};
    int n_tma = 0;
    int thr_max[NUM_PASSES] = {0, 0, 0, 0, 0};
    std::vector<int> pre9[NUM_PASSES];   // the observables' launch shapes (9 components)
    for (int k = 0; k < NUM_PASSES; ++k) pre9[k].push_back(0);
    size_t smem_green12 = 0;
    // the fused plane passes of the stress solve (3-D FP32 shapes that allow them) and the separate
    // row / axis-1 passes of the other instances
    std::vector<int> pre_plane(1, 0), pre_rest[NUM_PASSES];
    for (int k = 0; k < NUM_PASSES; ++k) pre_rest[k].push_back(0);
    size_t smem_plane = 0;
    int optin_dev = 0;
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin_dev, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    }
    for (int i = 0; i < n; ++i) {
        InstDev& I = p->inst[i];
        // rows kernels (R2C: 9 components, C2R: 6); ping-pong buffers of P padded rows
        // the transforms carry the 6 components of sym(beta) (forward) or of the stress cotangent
        for (int k : {PASS_R2C, PASS_C2R}) {
            const int comps = 6;
            long long npairs = ((long long)comps * I.rows + 1) / 2;
            const size_t line_bytes = (size_t)(I.nl + (I.nl >> 4) + 1) * velt;
            const cdd_tuning& tu = p->tune[i];
            int P = (velt == 8 ? 4096 : 2048) / I.nl;   // radix-16 stages: one butterfly per thread
            if (tu.rows_lines > 0) P = tu.rows_lines;
            if (P < 1) P = 1;
            if (P > npairs) P = (int)npairs;
            PassTile& t = I.tile[k];
            t.lines = P;
            // one first-stage butterfly per thread for 16-point stages: 256 threads from 16 line pairs
            // on (FP32), 128 below (and for FP64)
            t.threads = (velt == 8 && P >= 16) ? 256 : 128;
            t.blocks = (int)((npairs + P - 1) / P);
            t.tiles_a = 1;
            size_t sm = (((size_t)rows_buffers(I.lp_last, P) * P * (line_bytes / velt) + 1) & ~(size_t)1) * velt +
                        (size_t)I.lp_last.twspan * velt + rows_table_bytes(P);   // buffers + twiddle rows + row table
            if (sm > smem_max[k]) smem_max[k] = sm;
            if (t.threads > thr_max[k]) thr_max[k] = t.threads;
        }
        // axis-1 FFT (3-D only): W columns of 128 bytes
        for (int k : {PASS_MID_F, PASS_MID_I}) {
            PassTile& t = I.tile[k];
            if (I.nd != 3) { t.blocks = 0; t.lines = t.threads = t.tiles_a = 0; continue; }
            const int comps = 6;
            int W = (int)(128 / velt);
            while (W > 1 && 2 * (size_t)W * I.n1 * velt > 96 * 1024) W >>= 1;
            if (p->tune[i].mid_cols > 0) W = p->tune[i].mid_cols;
            t.lines = W;
            t.lgw = 0;
            while ((1 << t.lgw) < W) ++t.lgw;
            t.threads = 256;
            t.tiles_a = (I.nh + W - 1) / W;
            t.blocks = comps * I.n0 * t.tiles_a;
            // one shared tile for two-stage plans run with the first and last stage in global memory
            const int bufs = (line_plan_io(I.lp_mid) && I.lp_mid.nst == 2) ? 1 : 2;
            size_t sm = bufs * (size_t)W * I.n1 * velt + (size_t)I.lp_mid.twspan * velt;
            if (sm > smem_max[k]) smem_max[k] = sm;
            if (t.threads > thr_max[k]) thr_max[k] = t.threads;
        }
        // fused Green pass along axis 0: 6 component slots + 3 scratch slots of W columns
        {
            PassTile& t = I.tile[PASS_GREEN];
            int W = (int)(32 / velt);   // 32-byte row segments
            while (W > 1 && (size_t)9 * (I.n0 * W + W) * velt > 100 * 1024) W >>= 1;
            if (p->tune[i].green_cols > 0) W = p->tune[i].green_cols;
            if ((size_t)9 * (I.n0 * W + W) * velt > 220 * 1024) {
                if (p->tune[i].green_cols > 0)
                    return fail(CDD_ERR_ARG, "instance %d: tuning green_cols %d needs too much shared memory", i, W);
                return fail(CDD_ERR_SHAPE, "axis-0 length %d too large for the fused k-space pass", I.n0);
            }
            t.lines = W;
            t.lgw = 0;
            while ((1 << t.lgw) < W) ++t.lgw;
            t.threads = 256;
            t.tiles_a = (I.nh + W - 1) / W;
            t.blocks = (I.nd == 3 ? I.n1 : 1) * t.tiles_a;
            size_t sm = ((size_t)9 * (I.n0 * W + W) + 1) / 2 * 2 * velt + (size_t)I.lp_first.twspan * velt;
            if (sm > smem_max[PASS_GREEN]) smem_max[PASS_GREEN] = sm;
            if (t.threads > thr_max[PASS_GREEN]) thr_max[PASS_GREEN] = t.threads;
        }
        for (int k = 0; k < NUM_PASSES; ++k) pre[k].push_back(pre[k].back() + I.tile[k].blocks);
        {
            // the observables carry up to 9 components through the row and axis-1 passes and keep
            // 9 + 3 component slots in the k-space pass
            const long long np9 = (9LL * I.rows + 1) / 2;
            const int P = I.tile[PASS_R2C].lines;
            const int b_rows = (int)((np9 + P - 1) / P);
            const int b_mid = (I.nd == 3) ? 9 * I.n0 * I.tile[PASS_MID_F].tiles_a : 0;
            const int b9[NUM_PASSES] = {b_rows, b_mid, I.tile[PASS_GREEN].blocks, b_mid, b_rows};
            for (int k = 0; k < NUM_PASSES; ++k) pre9[k].push_back(pre9[k].back() + b9[k]);
            const int W = I.tile[PASS_GREEN].lines;
            const size_t sm = ((size_t)12 * (I.n0 * W + W) + 1) / 2 * 2 * velt + (size_t)I.lp_first.twspan * velt;
            if (sm > smem_green12) smem_green12 = sm;
        }
        {
            const bool ok = plane_eligible(I, C.precision, (size_t)optin_dev);
            if (p->tune[i].plane_fft == 1 && !ok)
                return fail(CDD_ERR_ARG, "instance %d: tuning plane_fft 1, but the shape or precision does not allow "
                                         "the fused plane passes", i);
            I.plane = (ok && p->tune[i].plane_fft == 1) ? 1 : 0;   // built-in: the separate passes (faster)
            p->tune[i].plane_fft = (I.nd == 3 && C.precision == CDD_F32) ? (I.plane ? 1 : -1) : 0;
            pre_plane.push_back(pre_plane.back() + (I.plane ? 6 * I.n0 * PLANE_CLUSTER : 0));
            for (int k = 0; k < NUM_PASSES; ++k) pre_rest[k].push_back(pre_rest[k].back() + (I.plane ? 0 : I.tile[k].blocks));
            if (I.plane && plane_smem_bytes(I) > smem_plane) smem_plane = plane_smem_bytes(I);
        }
        stencil_geometry(I, C.precision, p->tune[i].stencil_planes);
        // effective launch shapes of this instance
        p->tune[i].rows_lines = I.tile[PASS_R2C].lines;
        p->tune[i].mid_cols = (I.nd == 3) ? I.tile[PASS_MID_F].lines : 0;
        p->tune[i].green_cols = I.tile[PASS_GREEN].lines;
        p->tune[i].stencil_planes = (I.nd == 3) ? I.st_zc : 0;
        // consecutive instances of one shape (contiguous in every field) share one 5-D tensor map
        I.tma_slot = -1;
        I.tma_sub = 0;
        if (stencil_tma_eligible(I, C.precision)) {
            const InstDev* Q = (i > 0) ? &p->inst[i - 1] : nullptr;
            if (Q && Q->tma_slot >= 0 && Q->nd == I.nd && Q->n0 == I.n0 && Q->n1 == I.n1 && Q->n2 == I.n2) {
                I.tma_slot = Q->tma_slot;
                I.tma_sub = Q->tma_sub + 1;
            } else if (n_tma < CDD_MAX_TMA_MAPS) {
                I.tma_slot = n_tma++;
            }
        }
        pre_st.push_back(pre_st.back() + I.stencil_blocks);
        pre_ob.push_back(pre_ob.back() + (int)((I.cells + 255) / 256));
        pre_cw.push_back(pre_cw.back() + (int)((9 * I.cells + 1023) / 1024));
    }
    {
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        for (int k = 0; k < NUM_PASSES; ++k)
            if (optin > 0 && smem_max[k] + 1024 > (size_t)optin)
                return fail(CDD_ERR_ARG, "launch shapes need %zu bytes of shared memory in FFT pass %d (limit %d)",
                            smem_max[k], k, optin);
    }
    size_t smem_all = 0;
    for (int k = 0; k < NUM_PASSES; ++k) {
        LaunchShape& L = C.pass[k];
        L.blocks = pre[k].back();
        L.threads = (k == PASS_R2C || k == PASS_C2R) ? thr_max[k] : 256;
        L.smem = smem_max[k];
        if (L.smem > smem_all) smem_all = L.smem;
        CDD_CUDA(dalloc(p, (void**)&L.d_pre, sizeof(int) * (n + 1)));
        CDD_CUDA(cudaMemcpy(L.d_pre, pre[k].data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
        LaunchShape& L9 = C.pass9[k];
        L9.blocks = pre9[k].back();
        L9.threads = L.threads;
        L9.smem = (k == PASS_GREEN) ? smem_green12 : L.smem;
        if (L9.smem > smem_all) smem_all = L9.smem;
        CDD_CUDA(dalloc(p, (void**)&L9.d_pre, sizeof(int) * (n + 1)));
        CDD_CUDA(cudaMemcpy(L9.d_pre, pre9[k].data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    }
    C.plane.blocks = pre_plane.back();
    C.plane.threads = 256;
    C.plane.smem = smem_plane;
    CDD_CUDA(dalloc(p, (void**)&C.plane.d_pre, sizeof(int) * (n + 1)));
    CDD_CUDA(cudaMemcpy(C.plane.d_pre, pre_plane.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    for (int k = 0; k < NUM_PASSES; ++k) {
        LaunchShape& L = C.rest[k];
        L.blocks = pre_rest[k].back();
        L.threads = C.pass[k].threads;
        L.smem = C.pass[k].smem;
        CDD_CUDA(dalloc(p, (void**)&L.d_pre, sizeof(int) * (n + 1)));
        CDD_CUDA(cudaMemcpy(L.d_pre, pre_rest[k].data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    }
    {
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        C.obs_ok = !(optin > 0 && smem_green12 + 1024 > (size_t)optin);
        if (!C.obs_ok) C.pass9[PASS_GREEN].smem = C.pass[PASS_GREEN].smem;   // never launched
        if (C.pass9[PASS_GREEN].smem > smem_all) smem_all = C.pass9[PASS_GREEN].smem;
    }
    C.stencil.blocks = pre_st.back();
    C.stencil.threads = 256;
    C.stencil.smem = stencil_smem_bytes(C.precision, C.any3d);
    CDD_CUDA(stencil_set_attributes(C.precision, SIZE_MAX));   // device limit (see set_dyn_smem_limit)
    {
        std::vector<int> pre_v(1, 0);
        for (int i = 0; i < n; ++i) pre_v.push_back(pre_v.back() + (int)((p->inst[i].cells + 127) / 128));
        C.vjp.blocks = pre_v.back();
        C.vjp.threads = 128;
        CDD_CUDA(dalloc(p, (void**)&C.vjp.d_pre, sizeof(int) * (n + 1)));
        CDD_CUDA(cudaMemcpy(C.vjp.d_pre, pre_v.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    }
    C.obs.blocks = pre_ob.back();
    C.obs.threads = 256;
    CDD_CUDA(dalloc(p, (void**)&C.obs.d_pre, sizeof(int) * (n + 1)));
    CDD_CUDA(cudaMemcpy(C.obs.d_pre, pre_ob.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    CDD_CUDA(dalloc(p, (void**)&C.stencil.d_pre, sizeof(int) * (n + 1)));
    CDD_CUDA(cudaMemcpy(C.stencil.d_pre, pre_st.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    C.cellwise.blocks = pre_cw.back();
    C.cellwise.threads = 256;
    CDD_CUDA(dalloc(p, (void**)&C.cellwise.d_pre, sizeof(int) * (n + 1)));
    CDD_CUDA(cudaMemcpy(C.cellwise.d_pre, pre_cw.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    CDD_CUDA(stress_set_attributes(C.precision, SIZE_MAX));   // device limit (see set_dyn_smem_limit)
    (void)smem_all;
    return CDD_OK;
}

int check_plan(const cdd_plan* p) {
    if (!p) return fail(CDD_ERR_ARG, "null plan");
    return CDD_OK;
}

const StencilMapSet& user_maps(cdd_plan* p, const void* beta) {
    if (p->maps_user_ptr != beta) {
        encode_stencil_maps(p->core, p->inst.data(), beta, p->maps_user);
        p->maps_user_ptr = beta;
    }
    return p->maps_user;
}

int record_step(cdd_plan* p, void* beta, cudaStream_t st, int fixed, double dt_fixed) {
    PlanCore& C = p->core;
    if (C.any_vac && !C.d_vac) return fail(CDD_ERR_ARG, "the plan has vacancy instances: call cdd_set_vacancy first");
    const StencilMapSet& mu = user_maps(p, beta);
    if (C.any_vac) CDD_CUDA(launch_vacancy_pre(C, beta, st));
    CDD_CUDA(launch_stress(C, beta, C.d_sigma, st));
    CDD_CUDA(launch_stencil(C, M_STAGE1, beta, beta, C.d_f0, nullptr, 0.0, mu, st));
    CDD_CUDA(launch_dt(C, fixed, dt_fixed, st));
    CDD_CUDA(launch_stress_f0(C, beta, C.d_f0, C.d_sigma, st));
    CDD_CUDA(launch_stencil(C, M_STAGE2, C.d_f0, beta, C.d_f1, nullptr, 0.0, p->maps_f0, st));
    CDD_CUDA(launch_stress(C, C.d_f1, C.d_sigma, st));
    CDD_CUDA(launch_stencil(C, M_STAGE3, C.d_f1, beta, beta, nullptr, 0.0, p->maps_f1, st));
    if (C.any_vac) CDD_CUDA(launch_vacancy_post(C, beta, st));
    return CDD_OK;
}

}  // namespace

namespace cdd {
// Lets other translation units report through cdd_last_error().
int report_error(int code, const char* msg) { return fail(code, "%s", msg); }
}  // namespace cdd

extern "C" {

const char* cdd_last_error(void) { return g_last_error.c_str(); }
const char* cdd_version(void) { return "cdd-b200 0.1 (sm_100a)"; }

int cdd_plan_create(const cdd_instance* inst, int n_inst, int precision, cdd_plan** out) {
    return cdd_plan_create_tuned(inst, n_inst, precision, nullptr, out);
}

int cdd_plan_tuning(const cdd_plan* p, int i, cdd_tuning* out) {
    if (!p || !out || i < 0 || i >= p->core.n_inst) return fail(CDD_ERR_ARG, "bad arguments to cdd_plan_tuning");
    *out = p->tune[i];
    return CDD_OK;
}

int cdd_plan_create_tuned(const cdd_instance* inst, int n_inst, int precision, const cdd_tuning* tune,
                          cdd_plan** out) {
    g_last_error.clear();
    if (!inst || n_inst <= 0 || !out) return fail(CDD_ERR_ARG, "bad arguments to cdd_plan_create");
    if (precision != CDD_F64 && precision != CDD_F32) return fail(CDD_ERR_ARG, "bad precision %d", precision);
    *out = nullptr;
    auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
    for (int i = 0; tune && i < n_inst; ++i) {
        const cdd_tuning& t = tune[i];
        if ((t.fft_radix && t.fft_radix != 4 && t.fft_radix != 8 && t.fft_radix != 16) ||
            (t.rows_lines && t.rows_lines > 1024) ||
            (t.mid_cols && (!pow2(t.mid_cols) || t.mid_cols > 64)) ||
            (t.green_cols && (!pow2(t.green_cols) || t.green_cols > 64)) || t.stencil_planes < 0 ||
            t.fft_radix < 0 || t.rows_lines < 0 || t.mid_cols < 0 || t.green_cols < 0 ||
            t.plane_fft < -1 || t.plane_fft > 1)
            return fail(CDD_ERR_ARG, "instance %d: bad tuning (radix 4/8/16; lines <= 1024; columns: powers of "
                                     "two <= 64; planes >= 0; plane_fft -1, 0 or 1)", i);
    }
    cdd_plan* p = new cdd_plan();
    p->tune.assign(n_inst, cdd_tuning{0, 0, 0, 0, 0, 0});
    if (tune) p->tune.assign(tune, tune + n_inst);
    for (auto& t : p->tune)
        if (!t.fft_radix) t.fft_radix = 16;
    PlanCore& C = p->core;
    C.n_inst = n_inst;
    C.precision = precision;
    const size_t elt = precision == CDD_F64 ? sizeof(double) : sizeof(float);
    p->desc.assign(inst, inst + n_inst);
    p->inst.resize(n_inst);
    std::map<int, LinePlan> lp_done;   // line plans (with twiddle offsets) by (length, largest radix)
    std::vector<double> twre, twim;
    std::vector<double> ktab, ksin;   // k tables: wrapped identity and sine ('sinK'), same layout
    long long foff = 0, soff = 0, coff = 0, spoff = 0, rsoff = 0;
    C.any3d = false;
    for (int i = 0; i < n_inst; ++i) {
        const cdd_instance& d = inst[i];
        InstDev& I = p->inst[i];
        std::memset(&I, 0, sizeof I);
        if (d.ndim != 2 && d.ndim != 3) {
            free_plan(p);
            return fail(CDD_ERR_SHAPE, "instance %d: ndim must be 2 or 3 (got %d)", i, d.ndim);
        }
        int sh[3] = {d.shape[0], d.shape[1], d.ndim == 3 ? d.shape[2] : 1};
        for (int a = 0; a < d.ndim; ++a) {
            int A, B, Cc;
            if (sh[a] < 4 || sh[a] > 1024 || sh[a] % 2 || !factor(sh[a], A, B, Cc) || (B > 0 && Cc > 0)) {
                free_plan(p);
                return fail(CDD_ERR_SHAPE,
                            "instance %d: axis %d size %d unsupported (even, 4..1024, 2^a 3^b or 2^a 5^c)",
                            i, a, sh[a]);
            }
        }
        if (!(d.mu > 0) || !(d.nu < 0.5) || !(d.nu > -1.0) || !(d.cfl > 0)) {
            free_plan(p);
            return fail(CDD_ERR_ARG, "instance %d: need mu > 0, -1 < nu < 0.5, cfl > 0", i);
        }
        if (d.dynamics != CDD_DYN_GLIDE_CLIMB && d.dynamics != CDD_DYN_GLIDE_ONLY) {
            free_plan(p);
            return fail(CDD_ERR_ARG, "instance %d: unknown dynamics %d", i, d.dynamics);
        }
        if (d.dynamics == CDD_DYN_GLIDE_ONLY && d.Lambda != 0.0) {
            free_plan(p);
            return fail(CDD_ERR_ARG, "instance %d: the glide-only dynamics takes no Lambda", i);
        }
        if (d.vacancy && (d.dynamics != CDD_DYN_GLIDE_CLIMB || !(d.vac_gamma >= 0) || !std::isfinite(d.vac_alpha) ||
                          !std::isfinite(d.vac_beta))) {
            free_plan(p);
            return fail(CDD_ERR_ARG, "instance %d: vacancy coupling needs the glide-and-climb dynamics, finite "
                        "vac_alpha, vac_beta and vac_gamma >= 0", i);
        }
        if (!(d.dt_max >= 0)) {
            free_plan(p);
            return fail(CDD_ERR_ARG, "instance %d: dt_max must be >= 0", i);
        }
        I.nd = d.ndim;
        I.n0 = sh[0]; I.n1 = sh[1]; I.n2 = sh[2];
        if (I.nd == 3) C.any3d = true;
        I.nl = (I.nd == 3) ? I.n2 : I.n1;
        I.nh = I.nl / 2 + 1;
        I.nhp = (I.nh + 7) & ~7;
        I.fd_nl = fdiv_make(I.nl);
        I.fd_nh = fdiv_make(I.nh);
        I.cells = (long long)I.n0 * I.n1 * I.n2;
        I.rows = (int)(I.cells / I.nl);
        I.fd_rows = fdiv_make(I.rows);
        I.foff = foff; foff += 9 * I.cells;
        I.soff = soff; soff += 6 * I.cells;
        I.coff = coff; coff += I.cells;
        I.spoff = spoff; spoff += 9LL * I.rows * I.nhp;
        I.rsoff = rsoff; rsoff += 9LL * I.rows;
        LinePlan* lps[3] = {&I.lp_last, &I.lp_mid, &I.lp_first};
        int lens[3] = {I.nl, I.nd == 3 ? I.n1 : I.n0, I.n0};
        for (int k = 0; k < 3; ++k) {
            if (!make_line_plan(lens[k], *lps[k], p->tune[i].fft_radix)) {
                free_plan(p);
                return fail(CDD_ERR_SHAPE, "instance %d: no FFT plan for length %d", i, lens[k]);
            }
            const int key = lens[k] * 32 + p->tune[i].fft_radix;
            auto it = lp_done.find(key);
            if (it == lp_done.end()) {
                lps[k]->tw = (int)twre.size();
                for (int kk = 0; kk < lens[k]; ++kk) {
                    long double re, im;
                    twiddle(lens[k], kk, re, im);
                    twre.push_back((double)re);
                    twim.push_back((double)im);
                }
                append_stage_twiddles(*lps[k], twre, twim);
                it = lp_done.emplace(key, *lps[k]).first;
            }
            *lps[k] = it->second;
        }
        // k tables (FourierSpaceTools.py L26-55)
        if (I.nd == 3) {
            I.koff0 = (int)ktab.size();
            for (int a = 0; a < I.n0; ++a) {
                ktab.push_back(k_value(I.n0, I.n0, a));
                ksin.push_back(k_value_sin(I.n0, I.n0, a));
            }
            I.koff1 = (int)ktab.size();
            for (int a = 0; a < I.n1; ++a) {
                ktab.push_back(k_value(I.n1, I.n1, a));
                ksin.push_back(k_value_sin(I.n1, I.n1, a));
            }
            I.koffh = (int)ktab.size();
            for (int a = 0; a < I.nh; ++a) {
                ktab.push_back(k_value(I.n2, I.n2, a));
                ksin.push_back(k_value_sin(I.n2, I.n2, a));
            }
        } else {
            I.koff0 = (int)ktab.size();
            for (int a = 0; a < I.n0; ++a) {
                ktab.push_back(k_value(I.n1, I.n0, a));
                ksin.push_back(k_value_sin(I.n1, I.n0, a));
            }
            I.koff1 = I.koff0;
            I.koffh = (int)ktab.size();
            for (int a = 0; a < I.nh; ++a) {
                ktab.push_back(k_value(I.n1, I.n1, a));
                ksin.push_back(k_value_sin(I.n1, I.n1, a));
            }
        }
        I.mu = d.mu;
        I.nu = d.nu;
        I.glide = (d.dynamics == CDD_DYN_GLIDE_ONLY) ? 1 : 0;
        if (I.glide) C.any_glide = true;
        I.vacancy = d.vacancy ? 1 : 0;
        I.vac_alpha = d.vac_alpha;
        I.vac_beta = d.vac_beta;
        I.vac_gamma = d.vac_gamma;
        I.dt_max = d.dt_max;
        if (I.vacancy) C.any_vac = true;
        I.lamb = 2. * d.mu * d.nu / (1. - 2. * d.nu);
        I.Lambda = d.Lambda;
        I.cfl = d.cfl;
        I.nmax = (double)(I.n0 > I.n1 ? (I.n0 > I.n2 ? I.n0 : I.n2) : (I.n1 > I.n2 ? I.n1 : I.n2));
        I.h = 1.0 / (double)I.nl;
        I.inv_h = (double)I.nl;
        I.inv_cells = 1.0 / (double)I.cells;
        I.has_load = d.has_load ? 1 : 0;
        for (int a = 0; a < 3; ++a) { I.load_rate[a] = d.load_rate[a]; I.load_init[a] = d.load_initial[a]; }
        I.load_t0 = d.load_t0;
        I.load_mu = d.load_mu;
        I.load_lamb = 2. * d.load_mu * d.load_nu / (1. - 2. * d.load_nu);
    }
    cudaGetDevice(&p->device);
    C.field_elems = foff;
    C.stress_elems = soff;
    C.cells = coff;
    C.spec_elems = spoff;
    C.rows_total = rsoff;

    int rc = build_shapes(p, elt);
    if (rc != CDD_OK) { free_plan(p); return rc; }

#define ALLOC_OR_FAIL(ptr, bytes)                                                               \
    do {                                                                                        \
        cudaError_t e_ = dalloc(p, (void**)&(ptr), (bytes));                                    \
        if (e_ != cudaSuccess) {                                                                \
            free_plan(p);                                                                       \
            return fail(CDD_ERR_ALLOC, "cudaMalloc of %zu bytes failed: %s", (size_t)(bytes),   \
                        cudaGetErrorString(e_));                                                \
        }                                                                                       \
    } while (0)
#define COPY_OR_FAIL(dst, src, bytes)                                                           \
    do {                                                                                        \
        cudaError_t e_ = cudaMemcpy((dst), (src), (bytes), cudaMemcpyHostToDevice);             \
        if (e_ != cudaSuccess) {                                                                \
            free_plan(p);                                                                       \
            return fail(CDD_ERR_CUDA, "cudaMemcpy failed: %s", cudaGetErrorString(e_));         \
        }                                                                                       \
    } while (0)

    ALLOC_OR_FAIL(C.d_inst, sizeof(InstDev) * n_inst);
    COPY_OR_FAIL(C.d_inst, p->inst.data(), sizeof(InstDev) * n_inst);
    ALLOC_OR_FAIL(C.d_clock, sizeof(InstClock) * n_inst);
    {
        std::vector<InstClock> clk(n_inst);
        for (auto& c : clk) { std::memset(&c, 0, sizeof c); c.t_end = 1e300; }
        COPY_OR_FAIL(C.d_clock, clk.data(), sizeof(InstClock) * n_inst);
    }
    const size_t ntw = twre.size();
    if (precision == CDD_F64) {
        std::vector<double2> tw(ntw);
        for (size_t k = 0; k < ntw; ++k) tw[k] = make_double2(twre[k], twim[k]);
        ALLOC_OR_FAIL(C.d_tw, sizeof(double2) * ntw);
        COPY_OR_FAIL(C.d_tw, tw.data(), sizeof(double2) * ntw);
        C.ksin_off = (long long)ktab.size();
        ktab.insert(ktab.end(), ksin.begin(), ksin.end());
        ALLOC_OR_FAIL(C.d_k, sizeof(double) * ktab.size());
        COPY_OR_FAIL(C.d_k, ktab.data(), sizeof(double) * ktab.size());
    } else {
        std::vector<float2> tw(ntw);
        for (size_t k = 0; k < ntw; ++k) tw[k] = make_float2((float)twre[k], (float)twim[k]);
        ALLOC_OR_FAIL(C.d_tw, sizeof(float2) * ntw);
        COPY_OR_FAIL(C.d_tw, tw.data(), sizeof(float2) * ntw);
        C.ksin_off = (long long)ktab.size();
        std::vector<float> kf(ktab.begin(), ktab.end());
        kf.insert(kf.end(), ksin.begin(), ksin.end());
        ALLOC_OR_FAIL(C.d_k, sizeof(float) * kf.size());
        COPY_OR_FAIL(C.d_k, kf.data(), sizeof(float) * kf.size());
    }
    ALLOC_OR_FAIL(C.d_spec, 2 * elt * (size_t)C.spec_elems);
    cudaMemset(C.d_spec, 0, 2 * elt * (size_t)C.spec_elems);
    ALLOC_OR_FAIL(C.d_sigma, elt * (size_t)C.stress_elems);
    ALLOC_OR_FAIL(C.d_f0, elt * (size_t)C.field_elems);
    ALLOC_OR_FAIL(C.d_f1, elt * (size_t)C.field_elems);
    if (C.any_vac) ALLOC_OR_FAIL(C.d_vtr, elt * (size_t)(C.field_elems / 9));
    if (precision == CDD_F32) ALLOC_OR_FAIL(C.d_rowsum, sizeof(double) * (size_t)C.rows_total);
    ALLOC_OR_FAIL(C.d_sbar, sizeof(double) * 9 * n_inst);
    ALLOC_OR_FAIL(C.d_bmax, sizeof(double) * (size_t)C.stencil.blocks);
    ALLOC_OR_FAIL(C.d_bsum, sizeof(double) * 2 * (size_t)(C.stencil.blocks > C.obs.blocks ? C.stencil.blocks : C.obs.blocks));
    ALLOC_OR_FAIL(C.d_obs, sizeof(double) * 2 * n_inst);
    ALLOC_OR_FAIL(C.d_status, sizeof(int));
    cudaMemset(C.d_status, 0, sizeof(int));
    encode_stencil_maps(C, p->inst.data(), C.d_f0, p->maps_f0);
    encode_stencil_maps(C, p->inst.data(), C.d_f1, p->maps_f1);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { free_plan(p); return fail(CDD_ERR_CUDA, "plan setup: %s", cudaGetErrorString(e)); }
    *out = p;
    return CDD_OK;
#undef ALLOC_OR_FAIL
#undef COPY_OR_FAIL
}

int cdd_plan_destroy(cdd_plan* plan) {
    if (!plan) return CDD_OK;
    free_plan(plan);
    return CDD_OK;
}

int cdd_plan_num_instances(const cdd_plan* p) { return p ? p->core.n_inst : 0; }
int cdd_plan_precision(const cdd_plan* p) { return p ? p->core.precision : -1; }
long long cdd_plan_field_elems(const cdd_plan* p) { return p ? p->core.field_elems : -1; }
long long cdd_plan_field_offset(const cdd_plan* p, int i) {
    return (p && i >= 0 && i < p->core.n_inst) ? p->inst[i].foff : -1;
}
long long cdd_plan_stress_elems(const cdd_plan* p) { return p ? p->core.stress_elems : -1; }
long long cdd_plan_stress_offset(const cdd_plan* p, int i) {
    return (p && i >= 0 && i < p->core.n_inst) ? p->inst[i].soff : -1;
}
long long cdd_plan_cells(const cdd_plan* p, int i) {
    if (!p) return -1;
    if (i < 0) return p->core.cells;
    return i < p->core.n_inst ? p->inst[i].cells : -1;
}
long long cdd_plan_scratch_bytes(const cdd_plan* p) { return p ? p->scratch_bytes : -1; }

int cdd_stress(cdd_plan* p, const void* beta, void* sigma6, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (!beta || !sigma6) return fail(CDD_ERR_ARG, "null buffer");
    CDD_CUDA(launch_stress(p->core, beta, sigma6, (cudaStream_t)stream));
    return CDD_OK;
}

int cdd_flux(cdd_plan* p, const void* beta, double t, void* rhs, void* speed, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (!beta || !rhs) return fail(CDD_ERR_ARG, "null buffer");
    if (p->core.any_vac && !p->core.d_vac) return fail(CDD_ERR_ARG, "the plan has vacancy instances: call cdd_set_vacancy first");
    cudaStream_t st = (cudaStream_t)stream;
    CDD_CUDA(launch_stress(p->core, beta, p->core.d_sigma, st));
    CDD_CUDA(launch_stencil(p->core, M_FLUX, beta, beta, rhs, speed, t, user_maps(p, beta), st));
    return CDD_OK;
}

int cdd_flux_with_stress(cdd_plan* p, const void* beta, const void* sigma6, double t, void* rhs, void* speed,
                         void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (!beta || !sigma6 || !rhs) return fail(CDD_ERR_ARG, "null buffer");
    if (p->core.any_vac && !p->core.d_vac) return fail(CDD_ERR_ARG, "the plan has vacancy instances: call cdd_set_vacancy first");
    PlanCore K = p->core;
    K.d_sigma = const_cast<void*>(sigma6);
    CDD_CUDA(launch_stencil(K, M_FLUX, beta, beta, rhs, speed, t, user_maps(p, beta), (cudaStream_t)stream));
    return CDD_OK;
}

// ------------------------------------------------------------------------------------------
// The reference CUDA solver's file formats (.ics, .plas)
// ------------------------------------------------------------------------------------------
namespace {

// Grid of instance i as the transpose kernel sees it (2-D (n0, n1) -> (n0, 1, n1)).
void xpose_dims(const InstDev& I, int& n0, int& n1, int& n2) {
    if (I.nd == 3) { n0 = I.n0; n1 = I.n1; n2 = I.n2; }
    else { n0 = I.n0; n1 = 1; n2 = I.n1; }
}

int check_inst_prec(const cdd_plan* p, int i, int prec) {
    if (int rc = check_plan(p)) return rc;
    if (i < 0 || i >= p->core.n_inst) return fail(CDD_ERR_ARG, "instance %d out of range", i);
    if (prec != CDD_F64 && prec != CDD_F32) return fail(CDD_ERR_ARG, "bad file precision %d", prec);
    return CDD_OK;
}

size_t prec_bytes(int prec) { return prec == CDD_F64 ? 8 : 4; }

// Device staging buffer released on scope exit.
struct StageBuf {
    void* ptr = nullptr;
    ~StageBuf() { if (ptr) cudaFree(ptr); }
};

struct File {
    FILE* f = nullptr;
    ~File() { if (f) fclose(f); }
};

int io_fail(const char* what, const char* path) {
    return fail(CDD_ERR_IO, "%s '%s': %s", what, path ? path : "(null)", strerror(errno));
}

// Export instance i to host memory in the file layout and precision.
int export_to_host(cdd_plan* p, int i, const void* beta, int prec, std::vector<char>& host, cudaStream_t st) {
    const InstDev& I = p->inst[i];
    const size_t bytes = 9 * (size_t)I.cells * prec_bytes(prec);
    StageBuf d;
    CDD_CUDA(cudaMalloc(&d.ptr, bytes));
    int n0, n1, n2;
    xpose_dims(I, n0, n1, n2);
    const size_t el = prec_bytes(p->core.precision);
    CDD_CUDA(launch_field_xpose(true, (const char*)beta + I.foff * el, p->core.precision, d.ptr, prec, n0, n1, n2, st));
    host.resize(bytes);
    CDD_CUDA(cudaMemcpyAsync(host.data(), d.ptr, bytes, cudaMemcpyDeviceToHost, st));
    CDD_CUDA(cudaStreamSynchronize(st));
    return CDD_OK;
}

// Import a host buffer in the file layout and precision into instance i.
int import_from_host(cdd_plan* p, int i, const std::vector<char>& host, int prec, void* beta, cudaStream_t st) {
    const InstDev& I = p->inst[i];
    const size_t bytes = 9 * (size_t)I.cells * prec_bytes(prec);
    StageBuf d;
    CDD_CUDA(cudaMalloc(&d.ptr, bytes));
    CDD_CUDA(cudaMemcpyAsync(d.ptr, host.data(), bytes, cudaMemcpyHostToDevice, st));
    int n0, n1, n2;
    xpose_dims(I, n0, n1, n2);
    const size_t el = prec_bytes(p->core.precision);
    CDD_CUDA(launch_field_xpose(false, d.ptr, prec, (char*)beta + I.foff * el, p->core.precision, n0, n1, n2, st));
    CDD_CUDA(cudaStreamSynchronize(st));
    return CDD_OK;
}

long long file_size(FILE* f) {
    if (fseeko(f, 0, SEEK_END) != 0) return -1;
    const long long n = (long long)ftello(f);
    fseeko(f, 0, SEEK_SET);
    return n;
}

}  // namespace

int cdd_field_import(cdd_plan* p, int i, const void* src, int src_precision, void* beta, void* stream) {
    if (int rc = check_inst_prec(p, i, src_precision)) return rc;
    if (!src || !beta) return fail(CDD_ERR_ARG, "null buffer");
    const InstDev& I = p->inst[i];
    int n0, n1, n2;
    xpose_dims(I, n0, n1, n2);
    const size_t el = prec_bytes(p->core.precision);
    CDD_CUDA(launch_field_xpose(false, src, src_precision, (char*)beta + I.foff * el, p->core.precision, n0, n1, n2,
                                (cudaStream_t)stream));
    return CDD_OK;
}

int cdd_field_export(cdd_plan* p, int i, const void* beta, void* dst, int dst_precision, void* stream) {
    if (int rc = check_inst_prec(p, i, dst_precision)) return rc;
    if (!dst || !beta) return fail(CDD_ERR_ARG, "null buffer");
    const InstDev& I = p->inst[i];
    int n0, n1, n2;
    xpose_dims(I, n0, n1, n2);
    const size_t el = prec_bytes(p->core.precision);
    CDD_CUDA(launch_field_xpose(true, (const char*)beta + I.foff * el, p->core.precision, dst, dst_precision, n0, n1,
                                n2, (cudaStream_t)stream));
    return CDD_OK;
}

int cdd_ics_read(cdd_plan* p, int i, const char* path, void* beta, void* stream) {
    if (int rc = check_inst_prec(p, i, CDD_F64)) return rc;
    if (!path || !beta) return fail(CDD_ERR_ARG, "null argument");
    File f;
    f.f = fopen(path, "rb");
    if (!f.f) return io_fail("cannot open", path);
    const size_t bytes = 9 * (size_t)p->inst[i].cells * 8;
    std::vector<char> host(bytes);
    if (fread(host.data(), 1, bytes, f.f) != bytes)
        return fail(CDD_ERR_IO, "'%s' holds fewer than the %zu bytes of a 9-component float64 field", path, bytes);
    return import_from_host(p, i, host, CDD_F64, beta, (cudaStream_t)stream);
}

int cdd_ics_write(cdd_plan* p, int i, const char* path, const void* beta, void* stream) {
    if (int rc = check_inst_prec(p, i, CDD_F64)) return rc;
    if (!path || !beta) return fail(CDD_ERR_ARG, "null argument");
    std::vector<char> host;
    if (int rc = export_to_host(p, i, beta, CDD_F64, host, (cudaStream_t)stream)) return rc;
    File f;
    f.f = fopen(path, "wb");
    if (!f.f) return io_fail("cannot create", path);
    if (fwrite(host.data(), 1, host.size(), f.f) != host.size()) return io_fail("cannot write", path);
    return CDD_OK;
}

int cdd_plas_append(cdd_plan* p, int i, const char* path, double t, const void* beta, int file_precision,
                    void* stream) {
    if (int rc = check_inst_prec(p, i, file_precision)) return rc;
    if (!path || !beta) return fail(CDD_ERR_ARG, "null argument");
    std::vector<char> host;
    if (int rc = export_to_host(p, i, beta, file_precision, host, (cudaStream_t)stream)) return rc;
    File f;
    f.f = fopen(path, "ab");
    if (!f.f) return io_fail("cannot open", path);
    const double t64 = t;
    const float t32 = (float)t;
    const void* tag = (file_precision == CDD_F64) ? (const void*)&t64 : (const void*)&t32;
    if (fwrite(tag, 1, prec_bytes(file_precision), f.f) != prec_bytes(file_precision) ||
        fwrite(host.data(), 1, host.size(), f.f) != host.size() || fflush(f.f) != 0)
        return io_fail("cannot append to", path);
    return CDD_OK;
}

int cdd_plas_frames(cdd_plan* p, int i, const char* path, int file_precision, long long* frames) {
    if (int rc = check_inst_prec(p, i, file_precision)) return rc;
    if (!path || !frames) return fail(CDD_ERR_ARG, "null argument");
    File f;
    f.f = fopen(path, "rb");
    if (!f.f) return io_fail("cannot open", path);
    const long long size = file_size(f.f);
    if (size < 0) return io_fail("cannot size", path);
    const long long frame_bytes = (9 * p->inst[i].cells + 1) * (long long)prec_bytes(file_precision);
    *frames = size / frame_bytes;
    return CDD_OK;
}

int cdd_plas_read(cdd_plan* p, int i, const char* path, int file_precision, long long frame, double* t, void* beta,
                  void* stream) {
    if (int rc = check_inst_prec(p, i, file_precision)) return rc;
    if (!path || !beta) return fail(CDD_ERR_ARG, "null argument");
    File f;
    f.f = fopen(path, "rb");
    if (!f.f) return io_fail("cannot open", path);
    const long long size = file_size(f.f);
    if (size < 0) return io_fail("cannot size", path);
    const size_t el = prec_bytes(file_precision);
    const long long frame_bytes = (9 * p->inst[i].cells + 1) * (long long)el;
    const long long count = size / frame_bytes;
    const long long k = frame < 0 ? count + frame : frame;
    if (k < 0 || k >= count)
        return fail(CDD_ERR_IO, "'%s' has %lld whole frames; frame %lld does not exist", path, count, frame);
    if (fseeko(f.f, (off_t)(k * frame_bytes), SEEK_SET) != 0) return io_fail("cannot seek in", path);
    double t64 = 0.0;
    float t32 = 0.0f;
    if (fread(file_precision == CDD_F64 ? (void*)&t64 : (void*)&t32, 1, el, f.f) != el)
        return io_fail("cannot read", path);
    std::vector<char> host((size_t)(frame_bytes - (long long)el));
    if (fread(host.data(), 1, host.size(), f.f) != host.size()) return io_fail("cannot read", path);
    if (t) *t = (file_precision == CDD_F64) ? t64 : (double)t32;
    return import_from_host(p, i, host, file_precision, beta, (cudaStream_t)stream);
}

int cdd_set_vacancy(cdd_plan* p, void* c) {
    if (int rc = check_plan(p)) return rc;
    p->core.d_vac = c;
    return CDD_OK;
}

int cdd_observe_field(cdd_plan* p, int kind, const void* beta, void* out, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (!beta || !out) return fail(CDD_ERR_ARG, "null buffer");
    const bool sin_k = (kind & CDD_OBS_SINK) != 0;
    const int base = kind & ~CDD_OBS_SINK;
    if (base < CDD_OBS_BETA_ELASTIC || base > CDD_OBS_RODRIGUES_RHO) return fail(CDD_ERR_ARG, "bad observable %d", kind);
    if (!p->core.obs_ok)
        return fail(CDD_ERR_SHAPE, "the k-space observables need more shared memory than the device has for this "
                                   "axis-0 length");
    CDD_CUDA(launch_observable(p->core, base, beta, out, (cudaStream_t)stream, sin_k));
    return CDD_OK;
}

int cdd_set_time(cdd_plan* p, const double* t, const double* t_end) {
    if (int rc = check_plan(p)) return rc;
    const int n = p->core.n_inst;
    std::vector<InstClock> clk(n);
    CDD_CUDA(cudaMemcpy(clk.data(), p->core.d_clock, sizeof(InstClock) * n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i) {
        if (t) clk[i].t = t[i];
        if (t_end) clk[i].t_end = t_end[i];
    }
    CDD_CUDA(cudaMemcpy(p->core.d_clock, clk.data(), sizeof(InstClock) * n, cudaMemcpyHostToDevice));
    return CDD_OK;
}

int cdd_get_time(cdd_plan* p, double* t, double* dt_last, int* active) {
    if (int rc = check_plan(p)) return rc;
    const int n = p->core.n_inst;
    std::vector<InstClock> clk(n);
    CDD_CUDA(cudaMemcpy(clk.data(), p->core.d_clock, sizeof(InstClock) * n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i) {
        if (t) t[i] = clk[i].t;
        if (dt_last) dt_last[i] = clk[i].dt;
        if (active) active[i] = clk[i].active;
    }
    return CDD_OK;
}

int cdd_step(cdd_plan* p, void* beta, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (!beta) return fail(CDD_ERR_ARG, "null buffer");
    return record_step(p, beta, (cudaStream_t)stream, 0, 0.0);
}

int cdd_step_fixed(cdd_plan* p, void* beta, double dt, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (!beta) return fail(CDD_ERR_ARG, "null buffer");
    if (!(dt >= 0)) return fail(CDD_ERR_ARG, "dt must be >= 0");
    return record_step(p, beta, (cudaStream_t)stream, 1, dt);
}

int cdd_run(cdd_plan* p, void* beta, int n_steps, int use_graph, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (!beta || n_steps < 0) return fail(CDD_ERR_ARG, "bad arguments to cdd_run");
    cudaStream_t st = (cudaStream_t)stream;
    if (!use_graph) {
        for (int k = 0; k < n_steps; ++k)
            if (int rc = record_step(p, beta, st, 0, 0.0)) return rc;
        return CDD_OK;
    }
    if (!p->graph || p->graph_beta != beta || p->graph_vac != p->core.d_vac) {
        if (p->graph) { cudaGraphExecDestroy(p->graph); p->graph = nullptr; }
        if (!p->cap_stream) CDD_CUDA(cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking));
        cudaGraph_t g;
        CDD_CUDA(cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal));
        int rc = record_step(p, beta, p->cap_stream, 0, 0.0);
        cudaError_t e = cudaStreamEndCapture(p->cap_stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return fail(CDD_ERR_CUDA, "stream capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&p->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(CDD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        p->graph_beta = beta;
        p->graph_vac = p->core.d_vac;
    }
    for (int k = 0; k < n_steps; ++k) CDD_CUDA(cudaGraphLaunch(p->graph, st));
    return CDD_OK;
}

int cdd_observables(cdd_plan* p, const void* beta, double* energy, double* mean_zz, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (!beta) return fail(CDD_ERR_ARG, "null buffer");
    cudaStream_t st = (cudaStream_t)stream;
    CDD_CUDA(launch_stress(p->core, beta, p->core.d_sigma, st));
    CDD_CUDA(launch_observe(p->core, beta, st));
    const int n = p->core.n_inst;
    std::vector<double> obs(2 * n);
    CDD_CUDA(cudaMemcpyAsync(obs.data(), p->core.d_obs, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, st));
    CDD_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) {
        if (energy) energy[i] = obs[2 * i];
        if (mean_zz) mean_zz[i] = obs[2 * i + 1];
    }
    return CDD_OK;
}

namespace {
int check_adjoint_supported(const cdd_plan* p) {
    for (int i = 0; i < p->core.n_inst; ++i)
        if (p->inst[i].glide) return fail(CDD_ERR_UNSUPPORTED, "instance %d: no adjoint of the glide-only dynamics", i);
        else if (p->inst[i].vacancy) return fail(CDD_ERR_UNSUPPORTED, "instance %d: no adjoint of the vacancy coupling", i);
    return CDD_OK;
}

int ensure_adjoint_scratch(cdd_plan* p) {
    PlanCore& C = p->core;
    if (C.d_ubar) return CDD_OK;
    const size_t elt = C.precision == CDD_F64 ? sizeof(double) : sizeof(float);
    cudaError_t e;
    if ((e = dalloc(p, &C.d_ubar, elt * 54 * (size_t)C.cells)) ||
        (e = dalloc(p, (void**)&C.d_flags, sizeof(uint32_t) * 4 * (size_t)C.cells)) ||
        (e = dalloc(p, (void**)&C.d_bload, sizeof(double) * 5 * (size_t)C.vjp.blocks)) ||
        (e = dalloc(p, &C.d_adj9, elt * (size_t)C.field_elems)) ||
        (e = dalloc(p, &C.d_sb6, elt * (size_t)C.stress_elems)) ||
        (e = dalloc(p, (void**)&C.d_gpart, sizeof(double) * (size_t)C.pass[PASS_GREEN].blocks)) ||
        (e = dalloc(p, &C.d_f0b, elt * (size_t)C.field_elems)) ||
        (e = dalloc(p, &C.d_f1b, elt * (size_t)C.field_elems)))
        return fail(CDD_ERR_ALLOC, "adjoint scratch: %s", cudaGetErrorString(e));
    return CDD_OK;
}

// Step record: u, F0, F1 (fields), their stresses, their phi spectra; every part starts on a
// 256-byte boundary (offsets in elements).
struct RecLayout {
    long long u, f0, f1, su, sf0, sf1, pu, pf0, pf1, total;
};

RecLayout rec_layout(const PlanCore& C) {
    const long long elt = C.precision == CDD_F64 ? 8 : 4;
    const long long a = 256 / elt;
    auto up = [a](long long n) { return (n + a - 1) / a * a; };
    const long long F = up(C.field_elems), S = up(C.stress_elems), Ph = up(2 * (C.spec_elems / 9));
    RecLayout r;
    r.u = 0;
    r.f0 = F;
    r.f1 = 2 * F;
    r.su = 3 * F;
    r.sf0 = 3 * F + S;
    r.sf1 = 3 * F + 2 * S;
    r.pu = 3 * F + 3 * S;
    r.pf0 = r.pu + Ph;
    r.pf1 = r.pu + 2 * Ph;
    r.total = r.pu + 3 * Ph;
    return r;
}
}  // namespace

int cdd_flux_vjp(cdd_plan* p, const void* beta, double t, const void* gbar, void* betabar, void* sigbar6,
                 double* load_bar, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (int rc = check_adjoint_supported(p)) return rc;
    if (!beta || !gbar || !betabar || !sigbar6) return fail(CDD_ERR_ARG, "null buffer");
    if (int rc = ensure_adjoint_scratch(p)) return rc;
    CDD_CUDA(launch_flux_vjp(p->core, beta, t, gbar, sigbar6, betabar, load_bar, (cudaStream_t)stream));
    return CDD_OK;
}

int cdd_flux_branches(cdd_plan* p, const void* beta, double t, uint32_t* flags, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (int rc = check_adjoint_supported(p)) return rc;
    if (!beta || !flags) return fail(CDD_ERR_ARG, "null buffer");
    if (int rc = ensure_adjoint_scratch(p)) return rc;
    CDD_CUDA(launch_flux_branches(p->core, beta, t, flags, (cudaStream_t)stream));
    return CDD_OK;
}

int cdd_stress_adjoint(cdd_plan* p, const void* sigbar6, void* betabar9, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (!sigbar6 || !betabar9) return fail(CDD_ERR_ARG, "null buffer");
    CDD_CUDA(launch_stress_adjoint(p->core, sigbar6, betabar9, (cudaStream_t)stream));
    return CDD_OK;
}

int cdd_stress_dnu(cdd_plan* p, const void* beta, void* out6, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (!beta || !out6) return fail(CDD_ERR_ARG, "null buffer");
    CDD_CUDA(launch_stress_dnu(p->core, beta, out6, (cudaStream_t)stream));
    return CDD_OK;
}

long long cdd_plan_record_elems(const cdd_plan* p) {
    if (!p) return -1;
    return rec_layout(p->core).total;
}

int cdd_step_record(cdd_plan* p, void* beta, double t, double dt, void* rec, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (!beta) return fail(CDD_ERR_ARG, "null buffer");
    if (!(dt >= 0)) return fail(CDD_ERR_ARG, "dt must be >= 0");
    if (rec && ((uintptr_t)rec & 255)) return fail(CDD_ERR_ARG, "record must be 256-byte aligned");
    if (rec)
        if (int rc = check_adjoint_supported(p)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    PlanCore& C = p->core;
    const size_t elt = C.precision == CDD_F64 ? sizeof(double) : sizeof(float);
    if (!rec) {
        CDD_CUDA(launch_set_clock(C, t, st));
        return record_step(p, beta, st, 1, dt);
    }
    const RecLayout L = rec_layout(C);
    char* r = (char*)rec;
    void* u = r + L.u * elt;
    void* f0 = r + L.f0 * elt;
    void* f1 = r + L.f1 * elt;
    void* s_u = r + L.su * elt;
    void* s_f0 = r + L.sf0 * elt;
    void* s_f1 = r + L.sf1 * elt;
    // the stencil reads the stress of its input from core.d_sigma: point a copy at the record's
    PlanCore K = C;
    CDD_CUDA(launch_set_clock(C, t, st));
    CDD_CUDA(cudaMemcpyAsync(u, beta, elt * (size_t)C.field_elems, cudaMemcpyDeviceToDevice, st));
    CDD_CUDA(launch_stress(C, beta, s_u, st, r + L.pu * elt));
    K.d_sigma = s_u;
    CDD_CUDA(launch_stencil(K, M_STAGE1, beta, beta, f0, nullptr, 0.0, user_maps(p, beta), st));
    CDD_CUDA(launch_dt(C, 1, dt, st));
    CDD_CUDA(launch_stress_f0(C, beta, f0, s_f0, st, r + L.pf0 * elt));
    K.d_sigma = s_f0;
    StencilMapSet m0, m1;
    encode_stencil_maps(C, p->inst.data(), f0, m0);
    CDD_CUDA(launch_stencil(K, M_STAGE2, f0, beta, f1, nullptr, 0.0, m0, st));
    CDD_CUDA(launch_stress(C, f1, s_f1, st, r + L.pf1 * elt));
    K.d_sigma = s_f1;
    encode_stencil_maps(C, p->inst.data(), f1, m1);
    CDD_CUDA(launch_stencil(K, M_STAGE3, f1, beta, beta, nullptr, 0.0, m1, st));
    return CDD_OK;
}

int cdd_step_adjoint(cdd_plan* p, const void* rec, double t, double dt, void* ubar, double* pbar, void* stream) {
    if (int rc = check_plan(p)) return rc;
    if (int rc = check_adjoint_supported(p)) return rc;
    if (!rec || !ubar) return fail(CDD_ERR_ARG, "null buffer");
    if (int rc = ensure_adjoint_scratch(p)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    PlanCore& C = p->core;
    const size_t elt = C.precision == CDD_F64 ? sizeof(double) : sizeof(float);
    const RecLayout L = rec_layout(C);
    const char* r = (const char*)rec;
    const void* u = r + L.u * elt;
    const void* f0 = r + L.f0 * elt;
    const void* f1 = r + L.f1 * elt;
    // stage 3: F2 = 1/3 u + 2/3 F1 + 2/3 dt L(F1)
    {
        const void* x[3] = {ubar, nullptr, nullptr};
        const double a[3] = {2.0 / 3.0, 0.0, 0.0};
        CDD_CUDA(launch_vjp_stage(C, f1, r + L.sf1 * elt, r + L.pf1 * elt, t, ubar, 2.0 / 3.0 * dt, x, a, C.d_f1b,
                                  pbar, st));
    }
    // stage 2: F1 = 3/4 u + 1/4 F0 + 1/4 dt L(F0)
    {
        const void* x[3] = {C.d_f1b, nullptr, nullptr};
        const double a[3] = {0.25, 0.0, 0.0};
        CDD_CUDA(launch_vjp_stage(C, f0, r + L.sf0 * elt, r + L.pf0 * elt, t, C.d_f1b, 0.25 * dt, x, a, C.d_f0b,
                                  pbar, st));
    }
    // stage 1: F0 = u + dt L(u); u also feeds F1 (3/4) and F2 (1/3) directly
    {
        const void* x[3] = {C.d_f0b, ubar, C.d_f1b};
        const double a[3] = {1.0, 1.0 / 3.0, 0.75};
        CDD_CUDA(launch_vjp_stage(C, u, r + L.su * elt, r + L.pu * elt, t, C.d_f0b, dt, x, a, ubar, pbar, st));
    }
    return CDD_OK;
}

int cdd_check_status(cdd_plan* p) {
    if (int rc = check_plan(p)) return rc;
    int s = 0;
    CDD_CUDA(cudaMemcpy(&s, p->core.d_status, sizeof(int), cudaMemcpyDeviceToHost));
    CDD_CUDA(cudaMemset(p->core.d_status, 0, sizeof(int)));
    if (s & ST_NONFINITE) return fail(CDD_ERR_NONFINITE, "non-finite wave speed: step not applied");
    if (s & ST_TIMEOUT) return fail(CDD_ERR_TIMEOUT, "device wait timed out");
    return CDD_OK;
}

}  // extern "C"
