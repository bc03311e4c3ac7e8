// Internal declarations shared by the libcdd translation units.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <vector>

#include "../../include/cdd.h"

namespace cdd {

constexpr int MAX_STAGES = 12;
#define CDD_MAX_TMA_MAPS 32   // stencil tensor maps per plan (one per run of same-shape instances)
constexpr double ME = 2.220446049250313080847263336181640625e-16;   // DBL_EPSILON

// Exact division by an invariant divisor d >= 1 for 0 <= n < 2^31 with one wide multiply and a
// shift (Granlund & Montgomery 1994, round-up multiplier): l = ceil(log2 d),
// M = ceil(2^(32 + l) / d) < 2^33, floor(n / d) = (n * M) >> (32 + l); n * M < 2^64 and
// M d - 2^(32 + l) < d <= 2^l make it exact.
struct FDiv {
    unsigned long long M;
    int l;
    int d;
};

inline FDiv fdiv_make(int d) {
    FDiv f;
    f.d = d;
    f.l = 0;
    while ((1LL << f.l) < (long long)d) ++f.l;
    const unsigned long long num = 1ULL << (32 + f.l);
    f.M = num / (unsigned long long)d + ((num % (unsigned long long)d) ? 1ULL : 0ULL);
    return f;
}

__host__ __device__ __forceinline__ int fdiv_q(const FDiv& f, int n) {
    return (int)(((unsigned long long)(unsigned)n * f.M) >> (32 + f.l));
}

// One-dimensional FFT of length n as a sequence of Stockham stages of radix 2, 3, 4, 5, 8, 16.
struct LinePlan {
    int n;
    int nst;
    int radix[MAX_STAGES];
    int tw;   // offset (complex elements) of this length's twiddle table w_n^k, k < n
    FDiv nr[MAX_STAGES];   // stage st: butterflies per line n / radix[st]
    FDiv ns[MAX_STAGES];   // stage st: span of the finished sub-transforms (product of earlier radices)
    int twst[MAX_STAGES];  // stage st: offset (even, complex elements) of its twiddle rows
    int twspan;            // elements from twst[0] to the end of the last stage's rows
};

// Radix rounded up to even: the length of one twiddle row (pairs load as one 16-byte vector).
__host__ __device__ constexpr int tw_row(int R) { return R + (R & 1); }

// Twiddle rows of every stage of lp in butterfly order: row jm of stage st holds
// w_n^(r jm n / (ns R)), r < R (then (1, 0) padding), ns = lp.ns[st].d, from the length-n table
// already at re/im[lp.tw ...]. Appends to re/im and sets lp.twst. Over all stages the rows take
// sum_st ns_st tw_row(R_st) <= 2n entries.
inline void append_stage_twiddles(LinePlan& lp, std::vector<double>& re, std::vector<double>& im) {
    const int n = lp.n;
    for (int st = 0; st < lp.nst; ++st) {
        if (re.size() & 1) { re.push_back(1.0); im.push_back(0.0); }   // even start: 16-byte rows
        lp.twst[st] = (int)re.size();
        const int R = lp.radix[st], ns = lp.ns[st].d, Rp = tw_row(R);
        const int twstep = n / (ns * R);
        for (int jm = 0; jm < ns; ++jm)
            for (int r = 0; r < Rp; ++r) {
                if (r < R) {
                    const int k = (int)(((long long)r * jm * twstep) % n);
                    const double wr = re[lp.tw + k], wi = im[lp.tw + k];
                    re.push_back(wr);
                    im.push_back(wi);
                } else {
                    re.push_back(1.0);
                    im.push_back(0.0);
                }
            }
    }
    lp.twspan = (int)re.size() - lp.twst[0];
}

// ---- asynchronous global -> shared copies (cp.async, 16 bytes, zero fill) ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Stage a column tile of complex values: rows x 2^lgw columns of a row-major array (row stride
// `stride` elements, columns w >= wv are padding: read as zero) into dst[(e << lgw) + w], with
// 16-byte asynchronous copies. Each thread keeps one 16-byte chunk column and walks the rows with
// pointer increments. Needs 2^lgw x sizeof(V) >= 16, nt a multiple of the chunks per row and
// 16-byte aligned rows in both spaces. The caller waits (cp_async_wait_all) and synchronises the
// block before use.
template <typename V>
__device__ __forceinline__ void tile_async_load(V* dst, const V* src, long long stride, int rows, int lgw, int wv,
                                                int tid, int nt) {
    constexpr int PER = 16 / (int)sizeof(V);       // complex values per copy: 2 (FP32) or 1 (FP64)
    constexpr int LPER = (PER == 2) ? 1 : 0;
    const int cl = lgw - LPER;                     // log2 chunks per row
    const int w = (tid & ((1 << cl) - 1)) * PER;
    int valid = wv - w;
    valid = valid < 0 ? 0 : (valid > PER ? PER : valid);
    const int rstep = nt >> cl;
    if (rstep <= 0) return;   // launches use 256 threads and at most 64 columns: never taken
    int e = tid >> cl;
    const V* g = valid ? src + (long long)e * stride + w : src;
    const long long gstep = valid ? (long long)rstep * stride : 0;
    V* d = dst + (e << lgw) + w;
    const int dstep = rstep << lgw;
#pragma unroll 4
    for (; e < rows; e += rstep, g += gstep, d += dstep) cp_async16(d, g, valid * (int)sizeof(V));
}

// The inverse: a column tile in shared memory (layout as above) back to the row-major array, only
// the columns w < wv, with 16-byte stores (a partial chunk of an FP32 tile stores its one valid
// value). Same requirements; the caller synchronises before.
template <typename V>
__device__ __forceinline__ void tile_store(V* dst, const V* src, long long stride, int rows, int lgw, int wv,
                                           int tid, int nt) {
    constexpr int PER = 16 / (int)sizeof(V);
    constexpr int LPER = (PER == 2) ? 1 : 0;
    const int cl = lgw - LPER;
    const int w = (tid & ((1 << cl) - 1)) * PER;
    const int valid = wv - w;
    if (valid <= 0) return;
    const int rstep = nt >> cl;
    if (rstep <= 0) return;
    int e = tid >> cl;
    V* g = dst + (long long)e * stride + w;
    const long long gstep = (long long)rstep * stride;
    const V* d = src + (e << lgw) + w;
    const int dstep = rstep << lgw;
    if (valid >= PER) {
#pragma unroll 4
        for (; e < rows; e += rstep, g += gstep, d += dstep)
            *reinterpret_cast<float4*>(g) = *reinterpret_cast<const float4*>(d);
    } else {
#pragma unroll 4
        for (; e < rows; e += rstep, g += gstep, d += dstep) *g = *d;
    }
}

// Copy the twiddle rows of lp (global table tw) into shared memory at dst (16-byte aligned);
// fft_lines then reads them with rebase = lp.twst[0]. The caller synchronises before use.
template <typename V>
__device__ __forceinline__ void stage_tw_to_smem(const LinePlan& lp, const V* __restrict__ tw, V* dst, int tid,
                                                 int nt) {
    const V* src = tw + lp.twst[0];
    for (int i = tid; i < lp.twspan; i += nt) dst[i] = __ldg(src + i);
}

// Row kernels (R2C / C2R): per-block table of the 2P rows a block reads or writes, after the
// twiddle rows in shared memory: element offsets of the two rows (p, q; -1: past the end) and the
// FP64 mean stress added to the row (C2R of FP32 plans).
struct RowPtr {
    long long p, q;
};
// (C2R also keeps a second table of epilogue source rows; the R2C pass uses the first part only.)
__host__ __device__ constexpr size_t rows_table_bytes(int P) {
    return 16 + (size_t)2 * P * (2 * sizeof(RowPtr) + sizeof(double));
}
// The table starts 16-byte aligned after the twiddle rows (tws: twspan complex values).
template <typename V> __device__ __forceinline__ RowPtr* rows_table(V* tws, int twspan) {
    return reinterpret_cast<RowPtr*>(tws + ((twspan + 1) & ~1));
}

// Row passes (R2C / C2R) of a two-stage line plan (R0, R1) in {(16,16), (16,8), (16,4), (8,4)} with
// P lines per block run their first and last stages in registers (two butterfly loops of P R0 and
// P R1 trips, whole warps each) and keep one padded buffer of P lines in shared memory; other plans
// keep two (ping-pong stages).
__host__ __device__ inline bool rows_io_plan(const LinePlan& lp, int P) {
    if (lp.nst != 2) return false;
    const int a = lp.radix[0], b = lp.radix[1];
    if ((P * a) % 32 != 0 || (P * b) % 32 != 0) return false;
    return (a == 16 && (b == 16 || b == 8 || b == 4)) || (a == 8 && b == 4);
}
__host__ __device__ inline int rows_buffers(const LinePlan& lp, int P) { return rows_io_plan(lp, P) ? 1 : 2; }

// Per-pass tiling of one instance (host-chosen, read by the kernels).
struct PassTile {
    int blocks;    // blocks this instance contributes to the launch
    int lines;     // rows kernel: line pairs per block; strided kernels: columns per block (W, a power of 2)
    int threads;   // threads this instance needs (<= launch blockDim)
    int tiles_a;   // strided kernels: number of column tiles along the row
    int lgw;       // strided kernels: log2(lines)
};

enum Pass { PASS_R2C = 0, PASS_MID_F, PASS_GREEN, PASS_MID_I, PASS_C2R, NUM_PASSES };

// Device-side description of one instance.
struct InstDev {
    int nd;                 // 2 or 3
    int n0, n1, n2;         // grid; n2 = 1 in 2-D
    int nl;                 // length of the contiguous (last) axis
    int nh;                 // nl / 2 + 1
    int nhp;                // padded spectrum row length (complex elements)
    FDiv fd_nl, fd_nh;      // division by nl and nh
    FDiv fd_rows;           // division by rows (component of a packed row index)
    int rows;               // real rows per component (cells / nl)
    long long cells;
    long long foff;         // offset of the packed 9-component field
    long long soff;         // offset of the packed 6-component stress
    long long coff;         // offset in per-cell arrays (speed)
    long long spoff;        // offset (complex elements) of the 9-component spectrum
    long long rsoff;        // offset of the per-row FP64 sums (FP32 mean path)
    LinePlan lp_last;       // complex FFT of length nl (two real rows packed)
    LinePlan lp_mid;        // axis 1 (3-D only)
    LinePlan lp_first;      // axis 0
    int koff0, koff1, koffh;    // k tables: axis 0, axis 1 (3-D), half axis (last)
    PassTile tile[NUM_PASSES];
    int stencil_blocks;
    int st_zc;              // planes per stencil block along axis 0 (3-D)
    int plane;              // 1: the stress solve runs the fused plane passes (k_plane_fwd / k_plane_inv)
    int tma_slot;           // index of this instance's tensor map, -1: threads stage the planes
    int tma_sub;            // index of this instance in its map's run of same-shape instances
    double mu, nu, lamb, Lambda, cfl, nmax;
    double h, inv_h;        // Dx = 1 / shape[-1] (CentralUpwindHJ3D.py L15-16)
    double inv_cells;
    int has_load;
    double load_rate[3], load_init[3], load_t0, load_lamb, load_mu;
    int glide;              // glide-only dynamics (projected velocity)
    int vacancy;            // vacancy coupling: sigma_ii -= vac_alpha c, c update + diffusion per step
    double vac_alpha, vac_beta, vac_gamma;
    double dt_max;          // > 0: upper bound of the adaptive step
};

// Per-instance clock and reduction results kept on the device.
struct InstClock {
    double t;          // current time
    double t_end;      // end of the current Run interval
    double t_stage;    // step-start time (used for the load in all three stages)
    double dt;         // dt of the current/last step
    double vmax;       // last wave-speed maximum
    int active;        // this step is applied
    int steps;
};

// Device status bits.
enum StatusBits { ST_NONFINITE = 1, ST_TIMEOUT = 2 };

template <typename T> struct VecOf;
template <> struct VecOf<float> { typedef float2 type; };
template <> struct VecOf<double> { typedef double2 type; };

template <typename V> __device__ __forceinline__ V vadd(V a, V b) { V r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename V> __device__ __forceinline__ V vsub(V a, V b) { V r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
// FP32 complex add / subtract as one packed instruction (each lane rounded as the scalar operation;
// a + (-1) b is a - b exactly rounded once)
template <> __device__ __forceinline__ float2 vadd<float2>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 vsub<float2>(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
template <typename V> __device__ __forceinline__ V vmul(V a, V b) {
    V r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename V> __device__ __forceinline__ V vconj(V a) { a.y = -a.y; return a; }
// a * conj(w)
template <typename V> __device__ __forceinline__ V vmulc(V a, V w) {
    V r; r.x = a.x * w.x + a.y * w.y; r.y = a.y * w.x - a.x * w.y; return r;
}

// One twiddle row (R values) of a stage: 16-byte vector loads (two float2 or one double2 each).
// Plain loads: the rows live in shared memory (copied per block) or in global memory.
template <int R>
__device__ __forceinline__ void load_tw_row(const float2* __restrict__ row, float2* w) {
    const float4* q = reinterpret_cast<const float4*>(row);
#pragma unroll
    for (int k = 0; k < tw_row(R) / 2; ++k) {
        const float4 v = q[k];
        w[2 * k] = make_float2(v.x, v.y);
        if (2 * k + 1 < R) w[2 * k + 1] = make_float2(v.z, v.w);
    }
}
template <int R>
__device__ __forceinline__ void load_tw_row(const double2* __restrict__ row, double2* w) {
#pragma unroll
    for (int k = 0; k < R; ++k) w[k] = row[k];
}
template <typename V, typename T> __device__ __forceinline__ V vscale(V a, T s) { a.x *= s; a.y *= s; return a; }
template <typename V> __device__ __forceinline__ V vmake(double x, double y) {
    V r; r.x = (decltype(r.x))x; r.y = (decltype(r.y))y; return r;
}
// multiply by -i (forward transform) or +i (inverse transform)
template <typename V, bool INV> __device__ __forceinline__ V vrot(V a) {
    V r;
    if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
    return r;
}

// ------------------------------------------------------------------------------------------
// Small DFT codelets, out[k] = sum_n in[n] exp(-+ 2 pi i n k / R), in place.
// Constants are the exact mathematical values rounded to the working precision.
// ------------------------------------------------------------------------------------------
#define CDD_SQRT1_2 0.707106781186547524400844362104849039
#define CDD_COS_PI8 0.923879532511286756128183189396788933
#define CDD_SIN_PI8 0.382683432365089771728459984030398866
#define CDD_SQRT3_2 0.866025403784438646763723170752936183
#define CDD_COS_2PI5 0.309016994374947424102293417182819059
#define CDD_COS_4PI5 (-0.809016994374947424102293417182819059)
#define CDD_SIN_2PI5 0.951056516295153572116439333379382143
#define CDD_SIN_4PI5 0.587785252292473129168705954639072769

template <typename V, bool INV> __device__ __forceinline__ void dft2(V* x) {
    V a = x[0];
    x[0] = vadd(a, x[1]);
    x[1] = vsub(a, x[1]);
}

template <typename V, bool INV> __device__ __forceinline__ void dft3(V* x) {
    typedef decltype(x[0].x) T;
    V t1 = vadd(x[1], x[2]);
    V t2 = vsub(x[1], x[2]);
    V m = x[0];
    m.x -= (T)0.5 * t1.x;
    m.y -= (T)0.5 * t1.y;
    x[0] = vadd(x[0], t1);
    V r = vrot<V, INV>(vscale(t2, (T)CDD_SQRT3_2));
    x[1] = vadd(m, r);
    x[2] = vsub(m, r);
}

template <typename V, bool INV> __device__ __forceinline__ void dft4(V* x) {
    V t0 = vadd(x[0], x[2]);
    V t1 = vsub(x[0], x[2]);
    V t2 = vadd(x[1], x[3]);
    if constexpr (std::is_same<V, float2>::value) {
        // FP32: d = x1 - x3 formed with its halves swapped, so that t1 +- (-+i) d are one packed
        // multiply-add each (by +-1: the same roundings as the scalar adds)
        const float2 ds = make_float2(x[1].y - x[3].y, x[1].x - x[3].x);
        const float2 sp = INV ? make_float2(-1.0f, 1.0f) : make_float2(1.0f, -1.0f);
        x[0] = vadd(t0, t2);
        x[2] = vsub(t0, t2);
        x[1] = __ffma2_rn(ds, sp, t1);
        x[3] = __ffma2_rn(ds, make_float2(-sp.x, -sp.y), t1);
    } else {
        V t3 = vrot<V, INV>(vsub(x[1], x[3]));
        x[0] = vadd(t0, t2);
        x[2] = vsub(t0, t2);
        x[1] = vadd(t1, t3);
        x[3] = vsub(t1, t3);
    }
}

template <typename V, bool INV> __device__ __forceinline__ void dft5(V* x) {
    typedef decltype(x[0].x) T;
    const T c1 = (T)CDD_COS_2PI5, c2 = (T)CDD_COS_4PI5, s1 = (T)CDD_SIN_2PI5, s2 = (T)CDD_SIN_4PI5;
    V a1 = vadd(x[1], x[4]), b1 = vsub(x[1], x[4]);
    V a2 = vadd(x[2], x[3]), b2 = vsub(x[2], x[3]);
    V x0 = x[0];
    V m1, m2, n1, n2;
    m1.x = x0.x + c1 * a1.x + c2 * a2.x; m1.y = x0.y + c1 * a1.y + c2 * a2.y;
    m2.x = x0.x + c2 * a1.x + c1 * a2.x; m2.y = x0.y + c2 * a1.y + c1 * a2.y;
    n1.x = s1 * b1.x + s2 * b2.x; n1.y = s1 * b1.y + s2 * b2.y;
    n2.x = s2 * b1.x - s1 * b2.x; n2.y = s2 * b1.y - s1 * b2.y;
    V r1 = vrot<V, INV>(n1), r2 = vrot<V, INV>(n2);
    x[0] = vadd(vadd(x0, a1), a2);
    x[1] = vadd(m1, r1);
    x[4] = vsub(m1, r1);
    x[2] = vadd(m2, r2);
    x[3] = vsub(m2, r2);
}

template <typename V, bool INV> __device__ __forceinline__ void dft8(V* x) {
    typedef decltype(x[0].x) T;
    V e[4] = {x[0], x[2], x[4], x[6]};
    V o[4] = {x[1], x[3], x[5], x[7]};
    dft4<V, INV>(e);
    dft4<V, INV>(o);
    const T s = (T)CDD_SQRT1_2;
    const T sg = INV ? (T)1 : (T)-1;
    o[1] = vmul(o[1], vmake<V>(s, sg * s));
    o[2] = vrot<V, INV>(o[2]);
    o[3] = vmul(o[3], vmake<V>(-s, sg * s));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        x[k] = vadd(e[k], o[k]);
        x[k + 4] = vsub(e[k], o[k]);
    }
}

template <typename V, bool INV> __device__ __forceinline__ void dft16(V* x) {
    typedef decltype(x[0].x) T;
    V e[8], o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) { e[k] = x[2 * k]; o[k] = x[2 * k + 1]; }
    dft8<V, INV>(e);
    dft8<V, INV>(o);
    const T c = (T)CDD_COS_PI8, s = (T)CDD_SIN_PI8, r = (T)CDD_SQRT1_2;
    const T sg = INV ? (T)1 : (T)-1;
    o[1] = vmul(o[1], vmake<V>(c, sg * s));
    o[2] = vmul(o[2], vmake<V>(r, sg * r));
    o[3] = vmul(o[3], vmake<V>(s, sg * c));
    o[4] = vrot<V, INV>(o[4]);
    o[5] = vmul(o[5], vmake<V>(-s, sg * c));
    o[6] = vmul(o[6], vmake<V>(-r, sg * r));
    o[7] = vmul(o[7], vmake<V>(-c, sg * s));
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = vadd(e[k], o[k]);
        x[k + 8] = vsub(e[k], o[k]);
    }
}

template <int R, typename V, bool INV> __device__ __forceinline__ void dft(V* x) {
    if (R == 2) dft2<V, INV>(x);
    else if (R == 3) dft3<V, INV>(x);
    else if (R == 4) dft4<V, INV>(x);
    else if (R == 5) dft5<V, INV>(x);
    else if (R == 8) dft8<V, INV>(x);
    else if (R == 16) dft16<V, INV>(x);
}

// ------------------------------------------------------------------------------------------
// Shared-memory line FFT engine: out-of-place Stockham autosort, mixed radix, natural order in
// and out. Each stage reads one buffer and writes the other; a thread holds one butterfly
// (R values) at a time.
//
// Lines live in shared memory through a layout functor L:
//   L.addr(line, idx)  -> element offset of element idx of line `line`
//   L.lines            -> number of lines
//   L.line_fast        -> true when consecutive butterflies should walk lines (column tiles)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ int row_pad(int a) { return a + (a >> 4); }

struct RowLayout {   // lines are rows of length n, padded every 16 elements
    int lines, ld;
    __device__ __forceinline__ int addr(int l, int i) const { return l * ld + row_pad(i); }
    // butterfly g -> (line, butterfly index within the line): consecutive g walk one line
    __device__ __forceinline__ void split(int g, const FDiv& nr, int& l, int& j) const {
        l = fdiv_q(nr, g);
        j = g - l * nr.d;
    }
    template <int NR> __device__ __forceinline__ void split_c(int g, int& l, int& j) const {
        l = g / NR;
        j = g - l * NR;
    }
    // Offsets of elements i0 + r STEP of line l, r = 0, 1, ...  LIN: the padding splits,
    // row_pad(i0 + r STEP) = row_pad(i0) + row_pad(r STEP), so each offset is the line base plus a
    // constant (the caller guarantees it: see fft_stage_c).
    template <int STEP, bool LIN> struct Walk {
        int b, i0;
        __device__ __forceinline__ int operator()(int r) const {
            if constexpr (LIN) return b + r * STEP + ((r * STEP) >> 4);
            else return b + row_pad(i0 + r * STEP);
        }
    };
    template <int STEP, bool LIN> __device__ __forceinline__ Walk<STEP, LIN> walk(int l, int i0) const {
        if constexpr (LIN) return {l * ld + row_pad(i0), 0};
        else return {l * ld, i0};
    }
};

// K groups of 2^lgw columns: element i of line l = (c, w) at c * cs + (i << lgw) + w; consecutive
// butterflies walk the lines (columns) so that neighbouring threads touch neighbouring words.
template <int K>
struct ColLayout {
    int lgw, cs;
    __device__ __forceinline__ int lines() const { return K << lgw; }
    __device__ __forceinline__ int addr(int l, int i) const {
        const int c = (K == 1) ? 0 : (l >> lgw);
        const int w = l & ((1 << lgw) - 1);
        return c * cs + (i << lgw) + w;
    }
    __device__ __forceinline__ void split(int g, const FDiv&, int& l, int& j) const {
        j = (K == 1) ? (g >> lgw) : (g >> lgw) / K;
        l = g - j * (K << lgw);
    }
    template <int NR> __device__ __forceinline__ void split_c(int g, int& l, int& j) const {
        split(g, FDiv{}, l, j);
    }
    template <int STEP, bool LIN> struct Walk {   // elements i0 + r STEP of one line: a fixed stride
        int b, stride;
        __device__ __forceinline__ int operator()(int r) const { return b + r * stride; }
    };
    template <int STEP, bool LIN> __device__ __forceinline__ Walk<STEP, LIN> walk(int l, int i0) const {
        return {addr(l, i0), STEP << lgw};
    }
};

template <typename Lay> __device__ __forceinline__ int lay_lines(const Lay& lay) { return lay.lines; }
template <int K> __device__ __forceinline__ int lay_lines(const ColLayout<K>& lay) { return lay.lines(); }

template <int R, typename V, bool INV, typename Lay>
__device__ __forceinline__ void fft_stage(const V* __restrict__ src, V* __restrict__ dst,
                                          const Lay& lay, const FDiv& fnr, const FDiv& fns,
                                          const V* __restrict__ twrows, int tid, int nt) {
    const int nr = fnr.d;
    const int ns = fns.d;
    const int total = lay_lines(lay) * nr;
#pragma unroll 1
    for (int g = tid; g < total; g += nt) {
        int l, j;
        lay.split(g, fnr, l, j);
        const int jm = j - fdiv_q(fns, j) * ns;
        V v[R];
        if (ns == 1) {   // first stage: all twiddles are 1
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = src[lay.addr(l, j + r * nr)];
        } else {
            V w[R];
            load_tw_row<R>(twrows + jm * tw_row(R), w);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const V a = src[lay.addr(l, j + r * nr)];
                v[r] = (r == 0) ? a : (INV ? vmulc(a, w[r]) : vmul(a, w[r]));
            }
        }
        dft<R, V, INV>(v);
        const int jd = (j - jm) * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[lay.addr(l, jd + r * ns)] = v[r];
    }
    __syncthreads();
}

// One stage with radix R, span NS and NR = n / R butterflies per line known at compile time: the
// butterfly split, the twiddle row index jm = j mod NS and the element strides fold to constants.
// Same codelets, twiddle rows and operation order as fft_stage (bitwise-identical results).
// Row-layout offsets split into base + constant when the padding period 16 and the stride divide
// one another: loads walk j + r NR with j < NR; stores walk jd + r NS with jd = (j - jm) R + jm, whose
// first term is a multiple of NS R (a multiple of 16 when 16 divides NS R).
template <int R, int NS, int NR, typename V, bool INV, typename Lay>
__device__ __forceinline__ void fft_stage_c(const V* __restrict__ src, V* __restrict__ dst, const Lay& lay,
                                            const V* __restrict__ twrows, int tid, int nt) {
    constexpr bool LIN_LD = (NR % 16 == 0) || (16 % NR == 0);
    constexpr bool LIN_ST = (NS % 16 == 0) || (16 % NS == 0 && (NS * R) % 16 == 0);
    const int total = lay_lines(lay) * NR;
#pragma unroll 1
    for (int g = tid; g < total; g += nt) {
        int l, j;
        lay.template split_c<NR>(g, l, j);
        const int jm = (NS == 1) ? 0 : j % NS;
        const auto ld = lay.template walk<NR, LIN_LD>(l, j);
        V v[R];
        if constexpr (NS == 1) {   // first stage: all twiddles are 1
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = src[ld(r)];
        } else {
            V w[R];
            load_tw_row<R>(twrows + jm * tw_row(R), w);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const V a = src[ld(r)];
                v[r] = (r == 0) ? a : (INV ? vmulc(a, w[r]) : vmul(a, w[r]));
            }
        }
        dft<R, V, INV>(v);
        const auto sw = lay.template walk<NS, LIN_ST>(l, (j - jm) * R + jm);
#pragma unroll
        for (int r = 0; r < R; ++r) dst[sw(r)] = v[r];
    }
    __syncthreads();
}

template <int... Rs> struct RadixProd;
template <> struct RadixProd<> { static constexpr int v = 1; };
template <int R, int... Rs> struct RadixProd<R, Rs...> { static constexpr int v = R * RadixProd<Rs...>::v; };

// Stages st, st+1, ... of a plan whose remaining radices are R, Rs... (span NS so far).
template <typename V, bool INV, typename Lay, int NS, int R, int... Rs>
__device__ __forceinline__ V* fft_lines_c(V* src, V* dst, const Lay& lay, const LinePlan& lp,
                                          const V* __restrict__ twbase, int tid, int nt, int rebase, int st) {
    constexpr int N = NS * RadixProd<R, Rs...>::v;
    fft_stage_c<R, NS, N / R, V, INV>(src, dst, lay, twbase + (lp.twst[st] - rebase), tid, nt);
    if constexpr (sizeof...(Rs) == 0) return dst;
    else return fft_lines_c<V, INV, Lay, NS * R, Rs...>(dst, src, lay, lp, twbase, tid, nt, rebase, st + 1);
}

// ---- column tiles with the first and last stage in global memory ----
// The lines are the columns of a tile: K components of 2^lgw columns, line l = (c, w) with
// c = l >> lgw. The first stage reads its butterflies straight from global memory into registers
// and the last stage writes its outputs straight back, so a tile passes through shared memory only
// between stages (one buffer for two-stage plans). Same codelets, twiddle rows and operation order
// as fft_stage.
template <int K> __device__ __forceinline__ void col_split(int g, int lgw, int& l, int& j) {
    j = (K == 1) ? (g >> lgw) : (g >> lgw) / K;
    l = g - j * (K << lgw);
}

// Shared tile: element i of line (c, w) at base[c * cs + (i << lgw) + w].
template <typename V, int K> struct SColT {
    V* base;
    int lgw, cs;
    struct Walk {
        V* p;
        int stride;
        __device__ __forceinline__ V ld(int r) const { return p[r * stride]; }
        __device__ __forceinline__ void st(int r, V v) const { p[r * stride] = v; }
    };
    __device__ __forceinline__ Walk walk(int l, int i0, int step) const {
        const int c = (K == 1) ? 0 : (l >> lgw), w = l & ((1 << lgw) - 1);
        return {base + c * cs + (i0 << lgw) + w, step << lgw};
    }
};

// Global tile: element i of line (c, w) at base[c * cstride + i * stride + w]; columns w >= wv are
// padding: they read as zero and are not written.
template <typename V, int K> struct GColT {
    V* base;
    long long stride, cstride;
    int lgw, wv;
    struct Walk {
        V* p;
        long long stride;
        bool valid;
        __device__ __forceinline__ V ld(int r) const {
            V z;
            z.x = 0;
            z.y = 0;
            return valid ? p[r * stride] : z;
        }
        __device__ __forceinline__ void st(int r, V v) const {
            if (valid) p[r * stride] = v;
        }
    };
    __device__ __forceinline__ Walk walk(int l, int i0, int step) const {
        const int c = (K == 1) ? 0 : (l >> lgw), w = l & ((1 << lgw) - 1);
        return {base + c * cstride + (long long)i0 * stride + w, (long long)step * stride, w < wv};
    }
};

template <int R, int NS, int NR, typename V, bool INV, int K, class LS, class LD>
__device__ __forceinline__ void fft_stage_io(const LS& src, const LD& dst, int lgw, const V* __restrict__ twrows,
                                             int tid, int nt) {
    const int total = (K << lgw) * NR;
#pragma unroll 1
    for (int g = tid; g < total; g += nt) {
        int l, j;
        col_split<K>(g, lgw, l, j);
        const int jm = (NS == 1) ? 0 : j % NS;
        const auto a = src.walk(l, j, NR);
        V v[R];
        if constexpr (NS == 1) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = a.ld(r);
        } else {
            V w[R];
            load_tw_row<R>(twrows + jm * tw_row(R), w);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const V x = a.ld(r);
                v[r] = (r == 0) ? x : (INV ? vmulc(x, w[r]) : vmul(x, w[r]));
            }
        }
        dft<R, V, INV>(v);
        const auto b = dst.walk(l, (j - jm) * R + jm, NS);
#pragma unroll
        for (int r = 0; r < R; ++r) b.st(r, v[r]);
    }
    __syncthreads();
}

// Stages st, st+1, ... (remaining radices R, Rs..., span NS so far) from `in` to `out`; stage k
// writes the shared tile x when k is even and y when odd, the last stage writes `out`.
template <typename V, bool INV, int K, class LIn, class LOut, int NS, int R, int... Rs>
__device__ __forceinline__ void fft_io_c(const LIn& in, const SColT<V, K>& x, const SColT<V, K>& y, const LOut& out,
                                         int lgw, const LinePlan& lp, const V* __restrict__ twbase, int tid, int nt,
                                         int rebase, int st) {
    constexpr int N = NS * RadixProd<R, Rs...>::v;
    const V* tw = twbase + (lp.twst[st] - rebase);
    if constexpr (sizeof...(Rs) == 0) {
        fft_stage_io<R, NS, N / R, V, INV, K>(in, out, lgw, tw, tid, nt);
    } else {
        fft_stage_io<R, NS, N / R, V, INV, K>(in, x, lgw, tw, tid, nt);
        fft_io_c<V, INV, K, SColT<V, K>, LOut, NS * R, Rs...>(x, y, x, out, lgw, lp, twbase, tid, nt, rebase, st + 1);
    }
}

// The compile-time radix sequences of at least two stages (make_line_plan with the default largest
// radix 16 for 32..512 and 48, 96, 192, 24).
#define CDD_IO_SEQS(X)                                  \
    X(nst == 2 && r0 == 16 && r1 == 16, 16, 16)         \
    X(nst == 2 && r0 == 16 && r1 == 8, 16, 8)           \
    X(nst == 2 && r0 == 16 && r1 == 4, 16, 4)           \
    X(nst == 2 && r0 == 8 && r1 == 4, 8, 4)             \
    X(nst == 3 && r0 == 16 && r1 == 8 && r2 == 4, 16, 8, 4) \
    X(nst == 2 && r0 == 16 && r1 == 3, 16, 3)           \
    X(nst == 2 && r0 == 8 && r1 == 3, 8, 3)             \
    X(nst == 3 && r0 == 8 && r1 == 4 && r2 == 3, 8, 4, 3)   \
    X(nst == 3 && r0 == 16 && r1 == 4 && r2 == 3, 16, 4, 3)

// True when lp runs through fft_io (the host sizes shared memory with this).
__host__ __device__ inline bool line_plan_io(const LinePlan& lp) {
    const int nst = lp.nst, r0 = lp.radix[0], r1 = lp.radix[1], r2 = lp.radix[2];
    (void)r2;
#define CDD_IO_TEST(COND, ...) if (COND) return true;
    CDD_IO_SEQS(CDD_IO_TEST)
#undef CDD_IO_TEST
    return false;
}

// All stages of lp from `in` to `out` through the shared tiles x, y (y unused by two-stage plans).
// Returns false, doing nothing, when lp has no compile-time sequence. Every thread of the block
// must call this; it ends synchronised.
template <typename V, bool INV, int K, class LIn, class LOut>
__device__ __forceinline__ bool fft_io(const LIn& in, const SColT<V, K>& x, const SColT<V, K>& y, const LOut& out,
                                       int lgw, const LinePlan& lp, const V* __restrict__ twbase, int tid, int nt,
                                       int rebase) {
    const int nst = lp.nst, r0 = lp.radix[0], r1 = lp.radix[1], r2 = lp.radix[2];
    (void)r2;
#define CDD_IO_RUN(COND, ...)                                                                               \
    if (COND) {                                                                                             \
        fft_io_c<V, INV, K, LIn, LOut, 1, __VA_ARGS__>(in, x, y, out, lgw, lp, twbase, tid, nt, rebase, 0); \
        return true;                                                                                        \
    }
    CDD_IO_SEQS(CDD_IO_RUN)
#undef CDD_IO_RUN
    return false;
}

// Run all stages of `lp` on the lines of `lay`, starting in buffer a (b is scratch of the same
// layout). Returns the buffer that holds the result. Every thread of the block must call this.
// The radix sequences that make_line_plan gives the usual lengths (16 to 512, and 24, 48, 96, 192
// with the default largest radix 16) run the compile-time stages; others the general engine.
template <typename V, bool INV, typename Lay>
__device__ __forceinline__ V* fft_lines_g(V* a, V* b, const Lay& lay, const LinePlan& lp,
                                          const V* __restrict__ twbase, int tid, int nt, int rebase);

template <typename V, bool INV, typename Lay>
__device__ __forceinline__ V* fft_lines(V* a, V* b, const Lay& lay, const LinePlan& lp, const V* __restrict__ twbase,
                                        int tid, int nt, int rebase = 0) {
    const int nst = lp.nst, r0 = lp.radix[0], r1 = lp.radix[1], r2 = lp.radix[2];
#define CDD_SEQ(COND, ...) \
    if (COND) return fft_lines_c<V, INV, Lay, 1, __VA_ARGS__>(a, b, lay, lp, twbase, tid, nt, rebase, 0);
    CDD_SEQ(nst == 2 && r0 == 16 && r1 == 16, 16, 16)
    CDD_SEQ(nst == 2 && r0 == 16 && r1 == 8, 16, 8)
    CDD_SEQ(nst == 2 && r0 == 16 && r1 == 4, 16, 4)
    CDD_SEQ(nst == 2 && r0 == 8 && r1 == 4, 8, 4)
    CDD_SEQ(nst == 3 && r0 == 16 && r1 == 8 && r2 == 4, 16, 8, 4)
    CDD_SEQ(nst == 1 && r0 == 16, 16)
    CDD_SEQ(nst == 2 && r0 == 16 && r1 == 3, 16, 3)
    CDD_SEQ(nst == 2 && r0 == 8 && r1 == 3, 8, 3)
    CDD_SEQ(nst == 3 && r0 == 8 && r1 == 4 && r2 == 3, 8, 4, 3)
    CDD_SEQ(nst == 3 && r0 == 16 && r1 == 4 && r2 == 3, 16, 4, 3)
#undef CDD_SEQ
    return fft_lines_g<V, INV>(a, b, lay, lp, twbase, tid, nt, rebase);
}

template <typename V, bool INV, typename Lay>
__device__ __forceinline__ V* fft_lines_g(V* a, V* b, const Lay& lay, const LinePlan& lp, const V* __restrict__ twbase,
                        int tid, int nt, int rebase) {
    V* src = a;
    V* dst = b;
    for (int st = 0; st < lp.nst; ++st) {
        const int R = lp.radix[st];
        const FDiv& fnr = lp.nr[st];
        const FDiv& fns = lp.ns[st];
        const V* tw = twbase + (lp.twst[st] - rebase);
        switch (R) {
            case 2: fft_stage<2, V, INV>(src, dst, lay, fnr, fns, tw, tid, nt); break;
            case 3: fft_stage<3, V, INV>(src, dst, lay, fnr, fns, tw, tid, nt); break;
            case 4: fft_stage<4, V, INV>(src, dst, lay, fnr, fns, tw, tid, nt); break;
            case 5: fft_stage<5, V, INV>(src, dst, lay, fnr, fns, tw, tid, nt); break;
            case 8: fft_stage<8, V, INV>(src, dst, lay, fnr, fns, tw, tid, nt); break;
            default: fft_stage<16, V, INV>(src, dst, lay, fnr, fns, tw, tid, nt); break;
        }
        V* t = src; src = dst; dst = t;
    }
    return src;
}

// Find the instance that owns global block b, given prefix sums pre[0..n] of blocks.
__device__ __forceinline__ int find_instance(const int* __restrict__ pre, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&pre[mid]) <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ------------------------------------------------------------------------------------------
// Host-side plan core shared by the translation units (device pointers + launch shapes).
// ------------------------------------------------------------------------------------------
struct LaunchShape {
    int blocks = 0;       // total blocks over all instances
    int threads = 0;      // blockDim.x
    size_t smem = 0;      // dynamic shared memory bytes
    int* d_pre = nullptr; // prefix sums of blocks per instance (n_inst + 1)
};

struct PlanCore {
    int n_inst = 0;
    int precision = CDD_F64;
    int max_nd = 3;
    bool any3d = false;
    bool any_glide = false;          // some instance uses the glide-only dynamics
    bool any_vac = false;            // some instance has vacancy coupling
    void* d_vac = nullptr;           // caller's vacancy concentrations (cdd_set_vacancy), field_elems / 9
    void* d_vtr = nullptr;           // trace of beta^P at the step start (vacancy instances), field_elems / 9
    long long field_elems = 0, stress_elems = 0, cells = 0, spec_elems = 0, rows_total = 0;
    InstDev* d_inst = nullptr;       // device copy of the instance table
    InstClock* d_clock = nullptr;
    void* d_tw = nullptr;            // twiddles (double2 or float2)
    void* d_k = nullptr;             // k tables (double or float): the wrapped identity ones, then the sine ones
    long long ksin_off = 0;          // offset (elements) of the sine k tables ('sinK') in d_k
    void* d_spec = nullptr;          // 9-component half spectra
    void* d_sigma = nullptr;         // 6-component internal stress
    void* d_f0 = nullptr;            // stage-1 rhs / F0
    void* d_f1 = nullptr;            // F1
    double* d_rowsum = nullptr;      // FP32 path: FP64 per-row sums
    double* d_sbar = nullptr;        // FP32 path: FP64 mean of each beta component (9 per instance)
    double* d_bmax = nullptr;        // per-block wave-speed maxima
    double* d_bsum = nullptr;        // per-block energy and mean-zz partial sums (2 per block)
    double* d_obs = nullptr;         // per-instance energy, mean zz (2 per instance)
    int* d_status = nullptr;
    LaunchShape pass[NUM_PASSES];
    LaunchShape pass9[NUM_PASSES];   // the k-space observables: 9-component row / axis-1 passes, 12-slot k-space pass
    LaunchShape plane;               // stress solve: fused plane passes of the instances with plane set
    LaunchShape rest[NUM_PASSES];    // stress solve: the row and axis-1 passes of the other instances
    bool obs_ok = false;             // pass9 fits the device (shared memory of the 12-slot k-space pass)
    LaunchShape stencil;
    LaunchShape cellwise;            // elementwise kernels over cells
    LaunchShape obs;                 // observables: one thread per cell
    LaunchShape vjp;                 // flux VJP: 128 cells per block
    void* d_ubar = nullptr;          // adjoint scratch (allocated on first use): 54 derivative cotangents per cell
    uint32_t* d_flags = nullptr;     // limiter selections, 4 words per cell
    double* d_bload = nullptr;       // per-block parameter partials of the VJP (VJP_PARTS per block)
    void* d_adj9 = nullptr;          // beta cotangent from the adjoint stress solve
    void* d_sb6 = nullptr;           // stress cotangent of one stage (6 components)
    double* d_gpart = nullptr;       // per-green-block partials of the Parseval nu sum
    void* d_f0b = nullptr;           // reverse RK3: cotangents of F0 and F1
    void* d_f1b = nullptr;
};

// Tensor maps of one stage-input buffer for the TMA-staged instances (see stencil.cu).
struct StencilMapSet {
    int enabled = 0;
    CUtensorMap m[CDD_MAX_TMA_MAPS];
};

// stress.cu
// phi (optional): per k point of the input, s1 / kSq - r / kSqSq (see k_green), for the nu gradient.
cudaError_t launch_stress(const PlanCore& P, const void* beta, void* sigma, cudaStream_t st, void* phi = nullptr);
// The second RK3 stage's stress: rhs_f0 holds the stage-1 rhs on entry and F0 = u + dt rhs on
// return (dt from the instances' clocks); sigma = stress(F0).
cudaError_t launch_stress_f0(const PlanCore& P, const void* u, void* rhs_f0, void* sigma, cudaStream_t st,
                             void* phi = nullptr);
// phi / part (optional): phi of the state, per-green-block partials of the Parseval nu sum.
cudaError_t launch_stress_adjoint(const PlanCore& P, const void* sigbar6, void* betabar9, cudaStream_t st,
                                  const void* phi = nullptr, double* part = nullptr);
cudaError_t launch_stress_dnu(const PlanCore& P, const void* beta, void* out6, cudaStream_t st);
// adjoint.cu
cudaError_t launch_flux_branches(const PlanCore& P, const void* beta, double t, uint32_t* flags, cudaStream_t st);
// One stage of the reverse sweep: out = c L_v^T g + sum a_k x_k (x_k may be null), with v's stress
// sig_v and k-space phi_v precomputed; parameter cotangents (scaled by c) added to pbar if non-null.
cudaError_t launch_vjp_stage(const PlanCore& P, const void* v, const void* sig_v, const void* phi_v, double t,
                             const void* gbar, double c, const void* const x[3], const double a[3], void* out,
                             double* pbar, cudaStream_t st);
cudaError_t launch_flux_vjp(const PlanCore& P, const void* beta, double t, const void* gbar, void* sigbar,
                            void* betabar, double* load_bar, cudaStream_t st);
// stencil.cu
enum StencilMode { M_FLUX = 0, M_STAGE1 = 1, M_STAGE2 = 2, M_STAGE3 = 3 };
cudaError_t launch_stencil(const PlanCore& P, int mode, const void* bs, const void* bn, void* out,
                           void* speed, double t_flux, const StencilMapSet& maps, cudaStream_t st);
// Encode the tensor maps of buffer `base` for every run of instances with tma_slot >= 0; returns false
// (and leaves maps disabled) if the driver entry point is missing or an address is misaligned.
bool encode_stencil_maps(const PlanCore& P, const InstDev* insts, const void* base, StencilMapSet& maps);
bool stencil_tma_eligible(const InstDev& I, int precision);
cudaError_t launch_dt(const PlanCore& P, int fixed, double dt_fixed, cudaStream_t st);
cudaError_t launch_set_clock(const PlanCore& P, double t, cudaStream_t st);
// Vacancy coupling around a step: save tr(beta^P) before it; after it, c += vac_beta d tr and the
// diffusion c^ *= exp(-vac_gamma dt k^2) (FFT passes over one component).
cudaError_t launch_vacancy_pre(const PlanCore& P, const void* beta, cudaStream_t st);
cudaError_t launch_vacancy_post(const PlanCore& P, const void* beta, cudaStream_t st);
cudaError_t launch_vacancy_diffusion(const PlanCore& P, cudaStream_t st);
// k-space observables of beta (kind: cdd_observable); out in the packed 9- or 3-component layout.
cudaError_t launch_observable(const PlanCore& P, int kind, const void* beta, void* out, cudaStream_t st,
                              bool sin_k = false);
// Convert 9 components between the plan layout (last axis contiguous) and the reference files'
// layout (axis 0 fastest) of an n0 x n1 x n2 grid (2-D: n0 x 1 x n1); to_file selects the direction.
cudaError_t launch_field_xpose(bool to_file, const void* src, int src_prec, void* dst, int dst_prec, int n0, int n1,
                               int n2, cudaStream_t st);
cudaError_t launch_axpy_f0(const PlanCore& P, const void* u, void* rhs_f0, cudaStream_t st);
cudaError_t launch_observe(const PlanCore& P, const void* beta, cudaStream_t st);
cudaError_t stencil_set_attributes(int precision, size_t smem);

// Raise a kernel's dynamic shared-memory limit to smem, clamped to what the device allows next to
// the kernel's own static shared memory. The limit is a property of the kernel function, shared by
// every plan in the process, so plans always raise it to the device limit (SIZE_MAX) rather than
// to their own need: a later plan must not lower it under an earlier plan's launches.
template <typename F>
inline cudaError_t set_dyn_smem_limit(F* fn, size_t smem) {
    int dev = 0, optin = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev))) return e;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev))) return e;
    cudaFuncAttributes fa;
    if ((e = cudaFuncGetAttributes(&fa, fn))) return e;
    const long long lim = (long long)optin - (long long)fa.sharedSizeBytes;
    const long long v = (smem < (size_t)lim) ? (long long)smem : lim;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v);
}
size_t stencil_smem_bytes(int precision, bool any3d);
void stencil_geometry(InstDev& I, int precision, int planes = 0);
cudaError_t stress_set_attributes(int precision, size_t max_smem);
// Fused plane passes of the stress solve (stress.cu): whether instance I can take them and their
// shared memory per block.
bool plane_eligible(const InstDev& I, int precision, size_t smem_limit);
size_t plane_smem_bytes(const InstDev& I);
constexpr int PLANE_CLUSTER = 8;   // blocks per (component, plane) cluster

}  // namespace cdd
