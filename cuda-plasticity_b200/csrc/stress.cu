// Internal stress sigma(beta^P) on the device: a batched real-to-complex / complex-to-real FFT
// pipeline with the isotropic Green's-function contraction fused into the k-space pass.
//
// Mathematics (PlasticityState.CalculateSigma(source='betaE') + CalculateBetaElastic,
// Plasticity/PlasticityStates/PlasticityState.py L85-127, L357-390):
//   betaE^(k)_ij = kmask * sum_mn T_ijmn(k) betaP^(k)_mn - betaP^(k)_ij,
//   T_ijmn = A k_i k_j d_mn / kSq + k_i (k_m d_jn + k_n d_jm) / kSq - B k_i k_j k_m k_n / kSqSq,
//   A = lam / (lam + 2 mu), B = 2 (lam + mu) / (lam + 2 mu), kSq += ME, kSqSq += ME,
//   sigma_ij = lam tr(betaE) d_ij + mu (betaE_ij + betaE_ji).
// Contracting T with betaP gives, per k point,
//   sum_mn T_ijmn b_mn = k_i g_j,  g_j = k_j (A s / kSq - B r / kSqSq) + (p_j + q_j) / kSq,
//   s = tr b, p_j = sum_m k_m b_mj, q_j = sum_n b_jn k_n, r = sum_m k_m q_m,
// so the six stress components are formed directly in k space and only six inverse transforms
// are needed. The k tables are the reference's (FourierSpaceTools.py L5-59), built on the host.
//
// 3-D pipeline (grid n0 x n1 x n2, last axis contiguous, spectrum rows of nhp complex):
//   R2C rows (axis 2, two real rows per complex FFT)  -> forward FFT along axis 1
//   -> [forward FFT along axis 0, Green contraction, inverse FFT along axis 0] in one kernel
//   -> inverse FFT along axis 1 -> C2R rows (axis 2).
// 2-D: R2C rows (axis 1) -> fused Green pass along axis 0 -> C2R rows.
//
// FP32 plans keep the k = 0 mode in FP64: the R2C pass records FP64 row sums of beta, a small
// kernel turns their means into the mean stress -lam tr<b> d - mu (<b> + <b>^T), and the C2R pass
// adds it after the FP32 transforms (which carry a zero k = 0 mode).
#include "cdd_internal.cuh"

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

namespace cdd {

constexpr int ROW_THREADS = 256;
constexpr int GREEN_THREADS = 256;

__host__ __device__ inline int rows_ld(int n) { return n + (n >> 4) + 1; }

// Four consecutive reals: one 16-byte access for float, two for double (16-byte aligned).
__device__ __forceinline__ void load4(const float* p, float* v) {
    float4 q = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void load4(const double* p, double* v) {
    double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
// The same through the coherent path (data the kernel also writes).
__device__ __forceinline__ void load4c(const float* p, float* v) {
    float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void load4c(const double* p, double* v) {
    double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void store4(float* p, const float* v) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void store4(double* p, const double* v) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

// Symmetric component o = (SYM_I[o], SYM_J[o]): xx xy xz yy yz zz.
__device__ __constant__ int SYM_I[6] = {0, 0, 0, 1, 1, 2};
__device__ __constant__ int SYM_J[6] = {0, 1, 2, 1, 2, 2};

// Mean stress -lam tr<s> d_ij - 2 mu <s>_ij of symmetric component o, from the means m of the six
// components of s = sym(beta) (= -lam tr<b> d - mu (<b> + <b>^T)).
__device__ __forceinline__ double mean_stress(const InstDev& I, const double* m, int o) {
    double v = -2.0 * I.mu * m[o];
    if (o == 0 || o == 3 || o == 5) v -= I.lamb * (m[0] + m[3] + m[5]);
    return v;
}

// The stress depends on beta only through its symmetric part s = (beta + beta^T) / 2 (every term of
// the Green contraction and of sigma is symmetric in beta), so the transforms carry 6 components.
// Source rows of the R2C input, row ra = component o * rows + r:
//   RS_STRESS: row ra of a 6-component stress-layout array (p == q);
//   RS_SYM:    rows of beta_ij and beta_ji (p == q on the diagonal), 6 components;
//   RS_FULL:   row ra of a 9-component field (p == q), all 9 components.
// The value is (p + q) / 2, exact when p == q.
//   RS_VAC:    row ra of the vacancy concentrations (one component; vacancy instances only).
enum RowSource { RS_STRESS = 1, RS_SYM = 2, RS_FULL = 3, RS_VAC = 4 };

template <typename T>
__device__ __forceinline__ void src_rows(const InstDev& I, const T* base, int mode, long long ra, const T*& p,
                                         const T*& q) {
    if (mode == RS_STRESS) {
        p = q = base + I.soff + ra * I.nl;
        return;
    }
    if (mode == RS_FULL) {
        p = q = base + I.foff + ra * I.nl;
        return;
    }
    if (mode == RS_VAC) {
        p = q = base + I.foff / 9 + ra * I.nl;
        return;
    }
    const int o = fdiv_q(I.fd_rows, (int)ra);
    const long long r = ra - (long long)o * I.rows;
    const int i = SYM_I[o], j = SYM_J[o];
    p = base + I.foff + (long long)(3 * i + j) * I.cells + r * I.nl;
    q = base + I.foff + (long long)(3 * j + i) * I.cells + r * I.nl;
}

// ------------------------------------------------------------------------------------------
// Row passes of two-stage FFT plans (length N = R0 R1) with the first and the last stage in
// registers: the first stage's butterflies read their inputs straight from the rows, and the last
// stage's outputs go straight to the rows, so a tile passes through shared memory once, between
// the stages. R2C: the last stage's butterfly j of a line (R0 of them, consecutive lanes of one
// warp) holds X[j + R0 r]; the partner X[N - k] of k = j + R0 r sits in lane R0 - j at register
// R1 - 1 - r (in its own register R1 - r for j = 0), so one shuffle per r brings it, and the two
// half spectra of the line's rows are formed and stored from registers. The FP64 row sums of the
// FP32 form are summed from the first stage's inputs and reduced over the line's R1 lanes.
// Requires R0 dividing 32, R1 a power of two <= 32 and both stages' butterfly counts multiples of
// 32 (the block size is too): each warp takes part in a loop trip whole, as the shuffles need
// (rows_io_plan).
// ------------------------------------------------------------------------------------------
// The half spectra of pair p's two rows go to dst + 2 (p - p0) dld and one row (dld) further:
// the plan's spectrum (p0 = 0, dld = nhp) or a block's shared tile (the plane passes).
// F0 (the second RK3 stage's stress): the rows are formed as F0 = u + dt rhs from the rows of u and
// of rhs (held in f0w, the buffer rt points into) and written back over rhs, so the stage input is
// made in the same sweep that transforms it.
template <typename T> __device__ __forceinline__ T fma_t(T a, T b, T c);
template <> __device__ __forceinline__ float fma_t<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <> __device__ __forceinline__ double fma_t<double>(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T, bool F0>
__device__ __forceinline__ T row_value(const T* __restrict__ beta, T* f0w, const T* __restrict__ u, T dt,
                                       const RowPtr& e, int i) {
    if constexpr (F0) {
        const T xp = fma_t(dt, f0w[e.p + i], u[e.p + i]);
        f0w[e.p + i] = xp;
        T xq = xp;
        if (e.q != e.p) {
            xq = fma_t(dt, f0w[e.q + i], u[e.q + i]);
            f0w[e.q + i] = xq;
        }
        return (T)0.5 * (xp + xq);
    } else {
        return (T)0.5 * (beta[e.p + i] + beta[e.q + i]);
    }
}

// Where the row pass puts the two half spectra a (row 2q) and b (row 2q + 1) at bin k of the q-th
// line pair of the block (q = p - p0): rows of dst, dld apart.
template <typename V> struct RowSink {
    V* dst;
    int dld;
    __device__ __forceinline__ void operator()(long long q, int k, const V& a, const V& b, bool hasb) const {
        V* da = dst + 2 * q * dld;
        da[k] = a;
        if (hasb) da[dld + k] = b;
    }
};

template <typename T, bool MEAN64, int R0, int R1, bool F0, class Sink>
__device__ __forceinline__ void r2c_rows_io(const InstDev& I, int lb, int P, int ld, const RowPtr* __restrict__ rt,
                                            const T* __restrict__ beta, typename VecOf<T>::type* s,
                                            const typename VecOf<T>::type* __restrict__ tw1,
                                            const Sink& out, double* __restrict__ rowsum,
                                            long long nrows, long long npairs, int tid, int nt,
                                            long long p0, T* f0w = nullptr, const T* u = nullptr, T dt = 0) {
    typedef typename VecOf<T>::type V;
    // stage 0 (span 1): butterfly (l, j) takes elements j + R1 r of pair line l
#pragma unroll 1
    for (int g = tid; g < P * R1; g += nt) {
        const int l = g / R1, j = g - l * R1;
        const RowPtr ea = rt[2 * l], eb = rt[2 * l + 1];
        V v[R0];
        double sa = 0.0, sb = 0.0;
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const int i = j + R1 * r;
            T a = 0, b = 0;
            if (ea.p >= 0) a = row_value<T, F0>(beta, f0w, u, dt, ea, i);
            if (eb.p >= 0) b = row_value<T, F0>(beta, f0w, u, dt, eb, i);
            if (MEAN64) { sa += (double)a; sb += (double)b; }
            v[r].x = a;
            v[r].y = b;
        }
        if (MEAN64) {
#pragma unroll
            for (int o = R1 / 2; o > 0; o >>= 1) {
                sa += __shfl_xor_sync(0xffffffffu, sa, o);
                sb += __shfl_xor_sync(0xffffffffu, sb, o);
            }
            const long long row = 2LL * ((long long)lb * P + l);
            if (j == 0 && row < nrows) rowsum[I.rsoff + row] = sa;
            if (j == 0 && row + 1 < nrows) rowsum[I.rsoff + row + 1] = sb;
        }
        dft<R0, V, false>(v);
        V* d = s + l * ld + row_pad(j * R0);   // outputs j R0 + r: inside one 16-element pad period
#pragma unroll
        for (int r = 0; r < R0; ++r) d[r] = v[r];
    }
    __syncthreads();
    // stage 1 (span R0): butterfly (l, j) takes elements j + R0 r, twiddle row j; outputs X[j + R0 r]
    const int nh = I.nh;
#pragma unroll 1
    for (int g = tid; g < P * R0; g += nt) {
        const int l = g / R0, j = g - l * R0;
        V w[R1], v[R1];
        load_tw_row<R1>(tw1 + j * tw_row(R1), w);
        const V* sl = s + l * ld + row_pad(j);
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const V x = sl[r * R0 + ((r * R0) >> 4)];
            v[r] = (r == 0) ? x : vmul(x, w[r]);
        }
        dft<R1, V, false>(v);
        const int lane = tid & 31;
        const int partner = lane - j + (R0 - j) % R0;
        const long long p = (long long)lb * P + l;
        const bool valid = p < npairs;
        const bool hasb = 2 * p + 1 < nrows;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            V zs;
            zs.x = __shfl_sync(0xffffffffu, v[R1 - 1 - r].x, partner);
            zs.y = __shfl_sync(0xffffffffu, v[R1 - 1 - r].y, partner);
            const V zm = (j == 0) ? v[(R1 - r) % R1] : zs;
            const V zk = v[r];
            const int k = j + R0 * r;
            if (valid && k < nh) {
                V a, b;
                a.x = (T)0.5 * (zk.x + zm.x);
                a.y = (T)0.5 * (zk.y - zm.y);
                b.x = (T)0.5 * (zk.y + zm.y);
                b.y = (T)-0.5 * (zk.x - zm.x);
                out(p - p0, k, a, b, hasb);
            }
        }
    }
}

// The two-stage plans the row passes run with register-resident first and last stages (the plans
// rows_io_plan accepts).
#define CDD_ROWIO_SEQS(X) X(16, 16) X(16, 8) X(16, 4) X(8, 4)

// ------------------------------------------------------------------------------------------
// R2C along the contiguous axis of the 6 input components (see RowSource): pairs of real rows
// (a + i b) per complex FFT. FP32 plans also record FP64 sums of the rows (the k = 0 mode).
// ------------------------------------------------------------------------------------------
template <typename T, bool MEAN64>
__global__ void __launch_bounds__(ROW_THREADS, sizeof(T) == 4 ? 4 : 1) k_r2c_rows(const InstDev* __restrict__ insts, int n_inst,
                                                  const int* __restrict__ pre,
                                                  const T* __restrict__ beta,
                                                  typename VecOf<T>::type* __restrict__ spec,
                                                  const typename VecOf<T>::type* __restrict__ tw,
                                                  double* __restrict__ rowsum, int mode, int ncomp) {
    typedef typename VecOf<T>::type V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* s = reinterpret_cast<V*>(smem_raw);
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    const int lb = blockIdx.x - pre[ii];
    const int N = I.nl, P = I.tile[PASS_R2C].lines, ld = rows_ld(N);
    const long long nrows = (long long)ncomp * I.rows;
    if (2LL * lb * P >= nrows) return;   // launch sized for more components than this pass carries
    if (mode == RS_VAC && !I.vacancy) return;
    const long long npairs = (nrows + 1) / 2;
    const int tid = threadIdx.x, nt = blockDim.x;
    const T half = (T)0.5;

    // row table: the two source rows of each of the block's 2P rows (-1: past the last row)
    const bool io = rows_io_plan(I.lp_last, P);
    V* tws = s + ((rows_buffers(I.lp_last, P) * P * ld + 1) & ~1);   // twiddle rows, 16-byte aligned after the buffers
    RowPtr* rt = rows_table(tws, I.lp_last.twspan);
    for (int r = tid; r < 2 * P; r += nt) {
        const long long ra = 2LL * lb * P + r;
        RowPtr e;
        e.p = e.q = -1;
        if (ra < nrows) {
            const T *pa, *qa;
            src_rows(I, beta, mode, ra, pa, qa);
            e.p = pa - beta;
            e.q = qa - beta;
        }
        rt[r] = e;
    }
    stage_tw_to_smem(I.lp_last, tw, tws, tid, nt);
    __syncthreads();
    {
        const LinePlan& lq = I.lp_last;
        const V* tw1 = tws + (lq.twst[1] - lq.twst[0]);
#define CDD_R2C_IO(A, B)                                                                                      \
        if (io && lq.radix[0] == A && lq.radix[1] == B) {                                                     \
            r2c_rows_io<T, MEAN64, A, B, false>(I, lb, P, ld, rt, beta, s, tw1, RowSink<V>{spec + I.spoff, I.nhp}, \
                                                 rowsum, nrows, npairs, tid, nt, 0);                          \
            return;                                                                                           \
        }
        CDD_ROWIO_SEQS(CDD_R2C_IO)
#undef CDD_R2C_IO
    }
    const bool vec = ((N & 3) == 0) && ((((uintptr_t)(beta + I.foff)) & 15) == 0) &&
                     ((((uintptr_t)(beta + I.soff)) & 15) == 0) && ((((uintptr_t)(beta + I.foff / 9)) & 15) == 0) &&
                     ((I.cells & 3) == 0);
    if (vec) {
#pragma unroll 2
        for (int i4 = tid; i4 < (P * N) >> 2; i4 += nt) {
            const int i = i4 << 2;
            const int pl = fdiv_q(I.fd_nl, i), idx = i - pl * N;
            const RowPtr ea = rt[2 * pl], eb = rt[2 * pl + 1];
            T a[4] = {0, 0, 0, 0}, b[4] = {0, 0, 0, 0};
            if (ea.p >= 0) {
                T x[4], y[4];
                load4(beta + ea.p + idx, x);
                load4(beta + ea.q + idx, y);
#pragma unroll
                for (int q = 0; q < 4; ++q) a[q] = half * (x[q] + y[q]);
            }
            if (eb.p >= 0) {
                T x[4], y[4];
                load4(beta + eb.p + idx, x);
                load4(beta + eb.q + idx, y);
#pragma unroll
                for (int q = 0; q < 4; ++q) b[q] = half * (x[q] + y[q]);
            }
            V* d = s + pl * ld + row_pad(idx);
#pragma unroll
            for (int q = 0; q < 4; ++q) { V z; z.x = a[q]; z.y = b[q]; d[q] = z; }
        }
    } else {
#pragma unroll 2
        for (int i = tid; i < P * N; i += nt) {
            const int pl = fdiv_q(I.fd_nl, i), idx = i - pl * N;
            const RowPtr ea = rt[2 * pl], eb = rt[2 * pl + 1];
            V z; z.x = 0; z.y = 0;
            if (ea.p >= 0) z.x = half * (beta[ea.p + idx] + beta[ea.q + idx]);
            if (eb.p >= 0) z.y = half * (beta[eb.p + idx] + beta[eb.q + idx]);
            s[pl * ld + row_pad(idx)] = z;
        }
    }
    __syncthreads();
    if (MEAN64) {
        const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
        for (int r = warp; r < 2 * P; r += nw) {
            int pl = r >> 1;
            long long row = ((long long)lb * P + pl) * 2 + (r & 1);
            double acc = 0.0;
            for (int idx = lane; idx < N; idx += 32) {
                V z = s[pl * ld + row_pad(idx)];
                acc += (double)((r & 1) ? z.y : z.x);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0 && row < nrows) rowsum[I.rsoff + row] = acc;
        }
    }
    RowLayout lay{P, ld};
    s = fft_lines<V, false>(s, s + P * ld, lay, I.lp_last, tws, tid, nt, I.lp_last.twst[0]);
    const int nh = I.nh;
    V* dst = spec + I.spoff;
    for (int i = tid; i < P * nh; i += nt) {
        int pl = fdiv_q(I.fd_nh, i), k = i - pl * nh;
        long long p = (long long)lb * P + pl;
        if (p >= npairs) continue;
        V zk = s[pl * ld + row_pad(k)];
        int km = (k == 0) ? 0 : N - k;
        V zm = s[pl * ld + row_pad(km)];
        V a, b;
        a.x = (T)0.5 * (zk.x + zm.x);
        a.y = (T)0.5 * (zk.y - zm.y);
        b.x = (T)0.5 * (zk.y + zm.y);
        b.y = (T)-0.5 * (zk.x - zm.x);
        long long ra = 2 * p;
        dst[ra * I.nhp + k] = a;
        if (ra + 1 < nrows) dst[(ra + 1) * I.nhp + k] = b;
    }
}

// ------------------------------------------------------------------------------------------
// C2R along the contiguous axis of 6 components (pairs of half spectra), row ra = o * rows + r:
//   RD_STRESS:    to row ra of a 6-component stress-layout array (+ the FP64 mean stress of FP32
//                 plans);
//   RD_SYM_FIELD: to rows (i, j) and (j, i) of a 9-component field (the cotangent of beta from
//                 that of its symmetric part: d/d beta_ij = d/d beta_ji = the symmetric entry).
// The imaginary parts of the k = 0 and Nyquist bins are dropped (numpy irfft semantics).
// ------------------------------------------------------------------------------------------
//   RD_FIELD9 / RD_FIELD3: row ra of a packed 9- / 3-component array (instance offsets foff and
//                 foff / 3), with an optional epilogue (RowEpilogue).
//   RD_VAC:       row ra of the vacancy concentrations (vacancy instances whose step was applied).
enum RowDest { RD_STRESS = 0, RD_SYM_FIELD = 1, RD_FIELD9 = 2, RD_FIELD3 = 3, RD_VAC = 4 };

// Real-space terms the observables subtract from the inverse transform of output component c:
// out_c -= coef (beta[EPI_P[c]] - beta[EPI_Q[c]]) (EPI_Q < 0: no second term). beta^E: -beta^P;
// rotation (xy, xz, yz) and Rodrigues vector (x, y, z): minus the antisymmetric part of beta^P
// (PlasticityState.py L357-390, L435-446, L447-475).
enum RowEpilogue { EPI_NONE = 0, EPI_BETA_E = 1, EPI_ROTATION = 2, EPI_RODRIGUES = 3 };
__device__ __constant__ int EPI_P[4][9] = {{-1, -1, -1, -1, -1, -1, -1, -1, -1},
                                           {0, 1, 2, 3, 4, 5, 6, 7, 8},
                                           {1, 2, 5, -1, -1, -1, -1, -1, -1},
                                           {5, 6, 1, -1, -1, -1, -1, -1, -1}};
__device__ __constant__ int EPI_Q[4][9] = {{-1, -1, -1, -1, -1, -1, -1, -1, -1},
                                           {-1, -1, -1, -1, -1, -1, -1, -1, -1},
                                           {3, 6, 7, -1, -1, -1, -1, -1, -1},
                                           {7, 2, 3, -1, -1, -1, -1, -1, -1}};
__device__ __constant__ double EPI_COEF[4] = {0.0, 1.0, 0.5, 0.5};

template <typename T>
__device__ __forceinline__ void dst_rows(const InstDev& I, T* base, int mode, long long ra, T*& p, T*& q) {
    if (mode == RD_STRESS) {
        p = q = base + I.soff + ra * I.nl;
        return;
    }
    if (mode == RD_FIELD9 || mode == RD_FIELD3 || mode == RD_VAC) {
        p = q = base + (mode == RD_FIELD9 ? I.foff : (mode == RD_FIELD3 ? I.foff / 3 : I.foff / 9)) + ra * I.nl;
        return;
    }
    const int o = fdiv_q(I.fd_rows, (int)ra);
    const long long r = ra - (long long)o * I.rows;
    const int i = SYM_I[o], j = SYM_J[o];
    p = base + I.foff + (long long)(3 * i + j) * I.cells + r * I.nl;
    q = base + I.foff + (long long)(3 * j + i) * I.cells + r * I.nl;
}

// out -= coef (beta[e.p + idx ..] - beta[e.q + idx ..]) for four (epilogue4) or one value.
template <typename T>
__device__ __forceinline__ void epilogue4(const T* beta, const RowPtr& e, T coef, int idx, T* v) {
    T a[4], b[4] = {0, 0, 0, 0};
    load4c(beta + e.p + idx, a);
    if (e.q >= 0) load4c(beta + e.q + idx, b);
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] -= coef * (a[q] - b[q]);
}
template <typename T>
__device__ __forceinline__ T epilogue1(const T* beta, const RowPtr& e, T coef, int idx, T v) {
    const T b = e.q >= 0 ? beta[e.q + idx] : (T)0;
    return v - coef * (beta[e.p + idx] - b);
}

// C2R counterpart: the first stage forms z[i] = A[i] + i B[i] of a pair line straight from the
// half spectra of its two rows (z[N - i] from conjugates), the last stage writes the real rows
// (plus the FP64 mean stress or the real-space epilogue) straight to global memory.
template <typename T, bool MEAN64, int R0, int R1>
__device__ __forceinline__ void c2r_rows_io(const InstDev& I, int lb, int P, int ld, const RowPtr* __restrict__ rt,
                                            const RowPtr* __restrict__ re, const double* __restrict__ rmean,
                                            const typename VecOf<T>::type* __restrict__ src,
                                            typename VecOf<T>::type* s,
                                            const typename VecOf<T>::type* __restrict__ tw1, T* __restrict__ out,
                                            const T* __restrict__ beta, int epi, long long nrows, long long npairs,
                                            int tid, int nt, long long p0, int sld) {
    typedef typename VecOf<T>::type V;
    constexpr int N = R0 * R1;
#pragma unroll 1
    for (int g = tid; g < P * R1; g += nt) {
        const int l = g / R1, j = g - l * R1;
        const long long p = (long long)lb * P + l;
        const V* sa = (p < npairs) ? src + 2 * (p - p0) * sld : nullptr;
        const V* sb = (p < npairs && 2 * p + 1 < nrows) ? sa + sld : nullptr;
        V v[R0];
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const int i = j + R1 * r;
            const int m = (2 * i <= N) ? i : N - i;
            V A, B;
            A.x = A.y = B.x = B.y = 0;
            if (sa) A = sa[m];
            if (sb) B = sb[m];
            V z;
            if (i == 0 || 2 * i == N) { z.x = A.x; z.y = B.x; }
            else if (2 * i < N) { z.x = A.x - B.y; z.y = A.y + B.x; }
            else { z.x = A.x + B.y; z.y = B.x - A.y; }
            v[r] = z;
        }
        dft<R0, V, true>(v);
        V* d = s + l * ld + row_pad(j * R0);
#pragma unroll
        for (int r = 0; r < R0; ++r) d[r] = v[r];
    }
    __syncthreads();
#pragma unroll 1
    for (int g = tid; g < P * R0; g += nt) {
        const int l = g / R0, j = g - l * R0;
        V w[R1], v[R1];
        load_tw_row<R1>(tw1 + j * tw_row(R1), w);
        const V* sl = s + l * ld + row_pad(j);
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const V x = sl[r * R0 + ((r * R0) >> 4)];
            v[r] = (r == 0) ? x : vmulc(x, w[r]);
        }
        dft<R1, V, true>(v);
        const RowPtr ea = rt[2 * l], eb = rt[2 * l + 1];
        if (ea.p < 0) continue;
        const RowPtr xa = re[2 * l], xb = re[2 * l + 1];
        const T ma = (T)rmean[2 * l], mb = (T)rmean[2 * l + 1];
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = j + R0 * r;
            T va = v[r].x, vb = v[r].y;
            if (MEAN64) { va += ma; vb += mb; }
            if (epi != EPI_NONE) {
                va = epilogue1(beta, xa, ma, k, va);
                if (eb.p >= 0) vb = epilogue1(beta, xb, mb, k, vb);
            }
            out[ea.p + k] = va;
            if (ea.q != ea.p) out[ea.q + k] = va;
            if (eb.p >= 0) {
                out[eb.p + k] = vb;
                if (eb.q != eb.p) out[eb.q + k] = vb;
            }
        }
    }
}

template <typename T, bool MEAN64>
__global__ void __launch_bounds__(ROW_THREADS, sizeof(T) == 4 ? 4 : 1) k_c2r_rows(const InstDev* __restrict__ insts, int n_inst,
                                                  const int* __restrict__ pre,
                                                  const typename VecOf<T>::type* __restrict__ spec,
                                                  T* __restrict__ out,
                                                  const typename VecOf<T>::type* __restrict__ tw,
                                                  const double* __restrict__ sbar, int mode, int ncomp,
                                                  const T* __restrict__ beta, int epi,
                                                  const InstClock* __restrict__ clk) {
    typedef typename VecOf<T>::type V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* s = reinterpret_cast<V*>(smem_raw);
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    const int lb = blockIdx.x - pre[ii];
    const int N = I.nl, P = I.tile[PASS_C2R].lines, ld = rows_ld(N), nh = I.nh;
    const long long nrows = (long long)ncomp * I.rows;
    if (2LL * lb * P >= nrows) return;   // launch sized for more components than this pass carries
    if (mode == RD_VAC && (!I.vacancy || !clk[ii].active)) return;
    const long long npairs = (nrows + 1) / 2;
    const int tid = threadIdx.x, nt = blockDim.x;
    const V* src = spec + I.spoff;
    const bool io = rows_io_plan(I.lp_last, P);
    V* tws = s + ((rows_buffers(I.lp_last, P) * P * ld + 1) & ~1);
    stage_tw_to_smem(I.lp_last, tw, tws, tid, nt);
    // row table: the destination rows of each of the block's 2P rows and their FP64 mean stress
    RowPtr* rt = rows_table(tws, I.lp_last.twspan);
    RowPtr* re = rt + 2 * P;                                        // epilogue source rows
    double* rmean = reinterpret_cast<double*>(re + 2 * P);          // mean stress or epilogue coefficient
    for (int r = tid; r < 2 * P; r += nt) {
        const long long ra = 2LL * lb * P + r;
        RowPtr e, ep;
        e.p = e.q = -1;
        ep.p = ep.q = -1;
        double m = 0.0;
        if (ra < nrows) {
            T *pd, *qd;
            dst_rows(I, out, mode, ra, pd, qd);
            e.p = pd - out;
            e.q = qd - out;
            if (MEAN64) m = mean_stress(I, sbar + 9 * ii, fdiv_q(I.fd_rows, (int)ra));
            if (epi != EPI_NONE) {
                const int o = fdiv_q(I.fd_rows, (int)ra);
                const long long rr = ra - (long long)o * I.rows;
                const int cp = EPI_P[epi][o], cq = EPI_Q[epi][o];
                ep.p = I.foff + (long long)cp * I.cells + rr * I.nl;
                ep.q = cq >= 0 ? I.foff + (long long)cq * I.cells + rr * I.nl : -1;
                m = EPI_COEF[epi];
            }
        }
        rt[r] = e;
        re[r] = ep;
        rmean[r] = m;
    }
    {
        const LinePlan& lq = I.lp_last;
        const V* tw1 = tws + (lq.twst[1] - lq.twst[0]);
#define CDD_C2R_IO(A, B)                                                                                      \
        if (io && lq.radix[0] == A && lq.radix[1] == B) {                                                     \
            c2r_rows_io<T, MEAN64, A, B>(I, lb, P, ld, rt, re, rmean, src, s, tw1, out, beta, epi, nrows, npairs, \
                                          tid, nt, 0, I.nhp);                                                 \
            return;                                                                                           \
        }
        CDD_ROWIO_SEQS(CDD_C2R_IO)
#undef CDD_C2R_IO
    }
#pragma unroll 4
    for (int i = tid; i < P * nh; i += nt) {
        int pl = fdiv_q(I.fd_nh, i), k = i - pl * nh;
        long long p = (long long)lb * P + pl;
        V A, B;
        A.x = A.y = B.x = B.y = 0;
        if (p < npairs) {
            long long ra = 2 * p;
            A = src[ra * I.nhp + k];
            if (ra + 1 < nrows) B = src[(ra + 1) * I.nhp + k];
        }
        V z;
        if (k == 0 || 2 * k == N) {
            z.x = A.x; z.y = B.x;
            s[pl * ld + row_pad(k)] = z;
        } else {
            z.x = A.x - B.y; z.y = A.y + B.x;
            s[pl * ld + row_pad(k)] = z;
            z.x = A.x + B.y; z.y = B.x - A.y;
            s[pl * ld + row_pad(N - k)] = z;
        }
    }
    __syncthreads();
    RowLayout lay{P, ld};
    s = fft_lines<V, true>(s, s + P * ld, lay, I.lp_last, tws, tid, nt, I.lp_last.twst[0]);
    const bool vec = ((N & 3) == 0) && ((((uintptr_t)(out + I.soff)) & 15) == 0) &&
                     ((((uintptr_t)(out + I.foff)) & 15) == 0) && ((((uintptr_t)(out + I.foff / 3)) & 15) == 0) &&
                     ((((uintptr_t)(out + I.foff / 9)) & 15) == 0) &&
                     (epi == EPI_NONE || ((((uintptr_t)(beta + I.foff)) & 15) == 0)) && ((I.cells & 3) == 0);
    if (vec) {
#pragma unroll 2
        for (int i4 = tid; i4 < (P * N) >> 2; i4 += nt) {
            const int i = i4 << 2;
            const int pl = fdiv_q(I.fd_nl, i), idx = i - pl * N;
            const RowPtr ea = rt[2 * pl], eb = rt[2 * pl + 1];
            if (ea.p < 0) continue;
            T va[4], vb[4];
            const V* sr = s + pl * ld + row_pad(idx);
#pragma unroll
            for (int q = 0; q < 4; ++q) { V z = sr[q]; va[q] = z.x; vb[q] = z.y; }
            if (MEAN64) {
                const T ma = (T)rmean[2 * pl], mb = (T)rmean[2 * pl + 1];
#pragma unroll
                for (int q = 0; q < 4; ++q) { va[q] += ma; vb[q] += mb; }
            }
            if (epi != EPI_NONE) {
                epilogue4(beta, re[2 * pl], (T)rmean[2 * pl], idx, va);
                if (eb.p >= 0) epilogue4(beta, re[2 * pl + 1], (T)rmean[2 * pl + 1], idx, vb);
            }
            store4(out + ea.p + idx, va);
            if (ea.q != ea.p) store4(out + ea.q + idx, va);
            if (eb.p >= 0) {
                store4(out + eb.p + idx, vb);
                if (eb.q != eb.p) store4(out + eb.q + idx, vb);
            }
        }
    } else {
        for (int i = tid; i < P * N; i += nt) {
            const int pl = fdiv_q(I.fd_nl, i), idx = i - pl * N;
            const RowPtr ea = rt[2 * pl], eb = rt[2 * pl + 1];
            if (ea.p < 0) continue;
            V z = s[pl * ld + row_pad(idx)];
            T va = z.x, vb = z.y;
            if (MEAN64) {
                va += (T)rmean[2 * pl];
                vb += (T)rmean[2 * pl + 1];
            }
            if (epi != EPI_NONE) {
                va = epilogue1(beta, re[2 * pl], (T)rmean[2 * pl], idx, va);
                if (eb.p >= 0) vb = epilogue1(beta, re[2 * pl + 1], (T)rmean[2 * pl + 1], idx, vb);
            }
            out[ea.p + idx] = va;
            if (ea.q != ea.p) out[ea.q + idx] = va;
            if (eb.p >= 0) {
                out[eb.p + idx] = vb;
                if (eb.q != eb.p) out[eb.q + idx] = vb;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// Complex FFT along axis 1 of a 3-D spectrum, in place, for `ncomp` components.
// Block = (component, i0, column tile of W).
// ------------------------------------------------------------------------------------------
// One column tile: W = 2^lgw columns of N = n1 elements from base (row pitch nhp), wv of them valid.
// The kernel calls it with lgw as a literal for the usual tile widths, so that every shared-memory
// offset of the stages folds to a constant.
template <typename T, bool INV>
__device__ __forceinline__ void fft_mid_tile(const InstDev& I, typename VecOf<T>::type* s,
                                             typename VecOf<T>::type* base,
                                             const typename VecOf<T>::type* __restrict__ tw, int lgw, int wv,
                                             int tid, int nt) {
    typedef typename VecOf<T>::type V;
    const int W = 1 << lgw;
    const int N = I.n1, nhp = I.nhp;
    if (line_plan_io(I.lp_mid)) {
        // first and last stage in global memory; one shared tile for two-stage plans
        V* tws = s + (I.lp_mid.nst == 2 ? 1 : 2) * N * W;
        stage_tw_to_smem(I.lp_mid, tw, tws, tid, nt);
        const GColT<V, 1> g{base, nhp, 0, lgw, wv};
        const SColT<V, 1> x{s, lgw, 0}, y{s + N * W, lgw, 0};
        fft_io<V, INV, 1>(g, x, y, g, lgw, I.lp_mid, tws, tid, nt, I.lp_mid.twst[0]);
        return;
    }
    if (W * (int)sizeof(V) >= 16) {
        tile_async_load(s, base, nhp, N, lgw, wv, tid, nt);
    } else {
#pragma unroll 8
        for (int i = tid; i < N * W; i += nt) {
            const int e = i >> lgw, w = i & (W - 1);
            V z; z.x = 0; z.y = 0;
            if (w < wv) z = base[(long long)e * nhp + w];
            s[i] = z;
        }
    }
    V* tws = s + 2 * N * W;
    stage_tw_to_smem(I.lp_mid, tw, tws, tid, nt);
    cp_async_wait_all();
    __syncthreads();
    ColLayout<1> lay{lgw, 0};
    s = fft_lines<V, INV>(s, s + N * W, lay, I.lp_mid, tws, tid, nt, I.lp_mid.twst[0]);
    if (W * (int)sizeof(V) >= 16) {
        tile_store(base, s, nhp, N, lgw, wv, tid, nt);
    } else {
#pragma unroll 4
        for (int i = tid; i < N * W; i += nt) {
            const int e = i >> lgw, w = i & (W - 1);
            if (w < wv) base[(long long)e * nhp + w] = s[i];
        }
    }
}

template <typename T, bool INV>
__global__ void __launch_bounds__(ROW_THREADS, sizeof(T) == 4 ? 4 : 2) k_fft_mid(const InstDev* __restrict__ insts, int n_inst,
                                                 const int* __restrict__ pre,
                                                 typename VecOf<T>::type* __restrict__ spec,
                                                 const typename VecOf<T>::type* __restrict__ tw,
                                                 int pass, int ncomp, int vac_only) {
    typedef typename VecOf<T>::type V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* s = reinterpret_cast<V*>(smem_raw);
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    int lb = blockIdx.x - pre[ii];
    const PassTile& tl = I.tile[pass];
    const int W = tl.lines, lgw = tl.lgw, ta_n = tl.tiles_a;
    const int ta = lb % ta_n; lb /= ta_n;
    const int i0 = lb % I.n0;
    const int c = lb / I.n0;
    if (c >= ncomp) return;   // launch sized for more components than this pass carries
    if (vac_only && !I.vacancy) return;
    const int N = I.n1, nhp = I.nhp, nh = I.nh;
    const int col0 = ta * W;
    const int wv = min(W, nh - col0);
    const int tid = threadIdx.x, nt = blockDim.x;
    V* base = spec + I.spoff + ((long long)c * I.n0 + i0) * (long long)N * nhp + col0;
    if (lgw == 4) fft_mid_tile<T, INV>(I, s, base, tw, 4, wv, tid, nt);
    else if (lgw == 3) fft_mid_tile<T, INV>(I, s, base, tw, 3, wv, tid, nt);
    else fft_mid_tile<T, INV>(I, s, base, tw, lgw, wv, tid, nt);
}

// ------------------------------------------------------------------------------------------
// Fused k-space pass along axis 0: forward FFT of the 9 components, Green contraction to the 6
// stress components (scaled by 1 / cells), inverse FFT of the 6. In place on the spectrum.
// ------------------------------------------------------------------------------------------
// Complex value times a real scalar (plus a complex value): one packed instruction in FP32.
template <typename V, typename T> __device__ __forceinline__ V csc(V a, T s) { a.x *= s; a.y *= s; return a; }
template <typename V, typename T> __device__ __forceinline__ V cfma(V a, T s, V c) {
    V r; r.x = a.x * s + c.x; r.y = a.y * s + c.y; return r;
}
template <> __device__ __forceinline__ float2 csc<float2, float>(float2 a, float s) {
    return __fmul2_rn(a, make_float2(s, s));
}
template <> __device__ __forceinline__ float2 cfma<float2, float>(float2 a, float s, float2 c) {
    return __ffma2_rn(a, make_float2(s, s), c);
}

template <typename T, typename V>
__device__ __forceinline__ void green_point(const V* b, V* out, T kx, T ky, T kz, bool kzero,
                                            T lam, T mu, T A, T B, T scale, bool drop_k0, V* phi_out) {
    const T k[3] = {kx, ky, kz};
    const T ksq = kx * kx + ky * ky + kz * kz;
    const T ikse = (T)1 / (ksq + (T)ME);
    const T ikqe = (T)1 / (ksq * ksq + (T)ME);
    V s1 = vadd(vadd(b[0], b[4]), b[8]);
    V p[3], q[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        p[j] = cfma(b[6 + j], k[2], cfma(b[3 + j], k[1], csc(b[j], k[0])));
        q[j] = cfma(b[3 * j + 2], k[2], cfma(b[3 * j + 1], k[1], csc(b[3 * j], k[0])));
    }
    const V r = cfma(q[2], k[2], cfma(q[1], k[1], csc(q[0], k[0])));
    const V cc = vsub(csc(s1, A * ikse), csc(r, B * ikqe));
    const T mask = kzero ? (T)0 : (T)1;
    if (phi_out) {
        // phi = s1 / kSq - r / kSqSq: g_j depends on nu only through k_j (dA s1 / kSq - dB r / kSqSq)
        // with dA = dB, so d sigma / d nu at this k point is a multiple of phi (minus the lambda term)
        *phi_out = csc(vsub(csc(s1, ikse), csc(r, ikqe)), mask);
    }
    V g[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) g[j] = csc(cfma(vadd(p[j], q[j]), ikse, csc(cc, k[j])), mask);
    const V tr = vsub(cfma(g[2], k[2], cfma(g[1], k[1], csc(g[0], k[0]))), s1);
    const int ia[6] = {0, 0, 0, 1, 1, 2};
    const int ja[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int o = 0; o < 6; ++o) {
        const int i = ia[o], j = ja[o];
        V v = csc(vsub(vsub(cfma(g[i], k[j], csc(g[j], k[i])), b[3 * i + j]), b[3 * j + i]), mu);
        if (i == j) v = cfma(tr, lam, v);
        v = csc(v, scale);
        if (drop_k0 && kzero) { v.x = 0; v.y = 0; }
        out[o] = v;
    }
}

// Transpose of green_point (a real linear map from 9 to 6 complex components per k point):
// cotangents of the 6 stress components in, cotangents of the 9 beta components out. Each line
// reverses one line of green_point.
template <typename T, typename V>
__device__ __forceinline__ void green_point_adj(const V* sb, V* bb, T kx, T ky, T kz, bool kzero,
                                                T lam, T mu, T A, T B, T scale) {
    const T k[3] = {kx, ky, kz};
    const T ksq = kx * kx + ky * ky + kz * kz;
    const T ikse = (T)1 / (ksq + (T)ME);
    const T ikqe = (T)1 / (ksq * ksq + (T)ME);
    const T mask = kzero ? (T)0 : (T)1;
    const int ia[6] = {0, 0, 0, 1, 1, 2};
    const int ja[6] = {0, 1, 2, 1, 2, 2};
    V gb[3], trb;
#pragma unroll
    for (int j = 0; j < 3; ++j) { gb[j].x = 0; gb[j].y = 0; }
    trb.x = 0; trb.y = 0;
#pragma unroll
    for (int c = 0; c < 9; ++c) { bb[c].x = 0; bb[c].y = 0; }
#pragma unroll
    for (int o = 0; o < 6; ++o) {
        const int i = ia[o], j = ja[o];
        V v = vscale(sb[o], scale);
        gb[j].x += mu * k[i] * v.x; gb[j].y += mu * k[i] * v.y;
        gb[i].x += mu * k[j] * v.x; gb[i].y += mu * k[j] * v.y;
        bb[3 * i + j].x -= mu * v.x; bb[3 * i + j].y -= mu * v.y;
        bb[3 * j + i].x -= mu * v.x; bb[3 * j + i].y -= mu * v.y;
        if (i == j) { trb.x += lam * v.x; trb.y += lam * v.y; }
    }
    V s1b;
    s1b.x = -trb.x; s1b.y = -trb.y;
#pragma unroll
    for (int i = 0; i < 3; ++i) { gb[i].x += k[i] * trb.x; gb[i].y += k[i] * trb.y; }
    V ccb, pb[3], qb[3];
    ccb.x = mask * (k[0] * gb[0].x + k[1] * gb[1].x + k[2] * gb[2].x);
    ccb.y = mask * (k[0] * gb[0].y + k[1] * gb[1].y + k[2] * gb[2].y);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        pb[j].x = mask * ikse * gb[j].x; pb[j].y = mask * ikse * gb[j].y;
        qb[j] = pb[j];
    }
    s1b.x += A * ikse * ccb.x; s1b.y += A * ikse * ccb.y;
    V rb;
    rb.x = -B * ikqe * ccb.x; rb.y = -B * ikqe * ccb.y;
#pragma unroll
    for (int m = 0; m < 3; ++m) { qb[m].x += k[m] * rb.x; qb[m].y += k[m] * rb.y; }
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            bb[3 * j + n].x += qb[j].x * k[n]; bb[3 * j + n].y += qb[j].y * k[n];   // q_j = b_jn k_n
            bb[3 * n + j].x += k[n] * pb[j].x; bb[3 * n + j].y += k[n] * pb[j].y;   // p_j = k_m b_mj
        }
#pragma unroll
    for (int m = 0; m < 3; ++m) { bb[4 * m].x += s1b.x; bb[4 * m].y += s1b.y; }
}

// d sigma / d nu at fixed mu of green_point: A = nu/(1-nu), B = 1/(1-nu) and lam = 2 mu nu/(1-2nu)
// give dA = dB = 1/(1-nu)^2 and dlam = 2 mu/(1-2nu)^2.
template <typename T, typename V>
__device__ __forceinline__ void green_point_dnu(const V* b, V* out, T kx, T ky, T kz, bool kzero,
                                                T lam, T mu, T A, T B, T scale, T nu) {
    const T k[3] = {kx, ky, kz};
    const T ksq = kx * kx + ky * ky + kz * kz;
    const T ikse = (T)1 / (ksq + (T)ME);
    const T ikqe = (T)1 / (ksq * ksq + (T)ME);
    const T dA = (T)1 / ((1 - nu) * (1 - nu)), dB = dA;
    const T dlam = (T)2 * mu / ((1 - 2 * nu) * (1 - 2 * nu));
    V s1 = vadd(vadd(b[0], b[4]), b[8]);
    V p[3], q[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        p[j].x = k[0] * b[j].x + k[1] * b[3 + j].x + k[2] * b[6 + j].x;
        p[j].y = k[0] * b[j].y + k[1] * b[3 + j].y + k[2] * b[6 + j].y;
        q[j].x = b[3 * j].x * k[0] + b[3 * j + 1].x * k[1] + b[3 * j + 2].x * k[2];
        q[j].y = b[3 * j].y * k[0] + b[3 * j + 1].y * k[1] + b[3 * j + 2].y * k[2];
    }
    V r;
    r.x = k[0] * q[0].x + k[1] * q[1].x + k[2] * q[2].x;
    r.y = k[0] * q[0].y + k[1] * q[1].y + k[2] * q[2].y;
    const T mask = kzero ? (T)0 : (T)1;
    V cc, dcc;
    cc.x = A * s1.x * ikse - B * r.x * ikqe;
    cc.y = A * s1.y * ikse - B * r.y * ikqe;
    dcc.x = dA * s1.x * ikse - dB * r.x * ikqe;
    dcc.y = dA * s1.y * ikse - dB * r.y * ikqe;
    V g[3], dg[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        g[j].x = mask * (k[j] * cc.x + (p[j].x + q[j].x) * ikse);
        g[j].y = mask * (k[j] * cc.y + (p[j].y + q[j].y) * ikse);
        dg[j].x = mask * k[j] * dcc.x;
        dg[j].y = mask * k[j] * dcc.y;
    }
    V tr, dtr;
    tr.x = k[0] * g[0].x + k[1] * g[1].x + k[2] * g[2].x - s1.x;
    tr.y = k[0] * g[0].y + k[1] * g[1].y + k[2] * g[2].y - s1.y;
    dtr.x = k[0] * dg[0].x + k[1] * dg[1].x + k[2] * dg[2].x;
    dtr.y = k[0] * dg[0].y + k[1] * dg[1].y + k[2] * dg[2].y;
    const int ia[6] = {0, 0, 0, 1, 1, 2};
    const int ja[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int o = 0; o < 6; ++o) {
        const int i = ia[o], j = ja[o];
        V v;
        v.x = mu * (k[i] * dg[j].x + k[j] * dg[i].x);
        v.y = mu * (k[i] * dg[j].y + k[j] * dg[i].y);
        if (i == j) {
            v.x += dlam * tr.x + lam * dtr.x;
            v.y += dlam * tr.y + lam * dtr.y;
        }
        out[o] = vscale(v, scale);
    }
}

// ---- k-space observables (PlasticityState.py) ----
// Component counts of the k-space pass per mode (see k_green) and its shared-memory slots (inputs
// or outputs, whichever are more, plus three scratch slots).
__host__ __device__ constexpr int green_nin(int gmode) { return (gmode == 6 || gmode == 8) ? 9 : (gmode == 7 ? 1 : 6); }
__host__ __device__ constexpr int green_nout(int gmode) {
    return (gmode == 3 || gmode == 6) ? 9 : ((gmode == 4 || gmode == 5 || gmode == 8) ? 3 : (gmode == 7 ? 1 : 6));
}
// transforms run on groups of three components, or one by one for the single-component mode
__host__ __device__ constexpr int green_group(int gmode) { return gmode == 7 ? 1 : 3; }
__host__ __device__ constexpr int green_slots(int gmode) {
    return (green_nin(gmode) > green_nout(gmode) ? green_nin(gmode) : green_nout(gmode)) + 3;
}

// One k point of an observable, scaled by 1 / cells for the inverse transform:
//  3: beta^E before the real-space -beta^P term (CalculateBetaElastic L357-390):
//     kmask sum_mn T_ijmn b_mn = kmask k_i g_j with g as in green_point and, b entering through
//     its symmetric part, p = q = sym(b) k;
//  4: its antisymmetric part (k_i g_j - k_j g_i) / 2 for (xy, xz, yz) (CalculateRotationField
//     L435-446);
//  5: the Rodrigues vector from beta^P (CalculateRotationRodrigues L447-475, source 'betaP'):
//     kmask sum_jst k_j (e_ijt k_s + e_ijs k_t) b_st / (2 kSq) = kmask (k x q)_i / kSq;
//  6: the Nye density rho_ai = -e_akl d_k b_li by Fourier derivatives (CalculateRhoFourier
//     L264-304): rho_xi = i (kz b_yi - ky b_zi), rho_yi = i (kx b_zi - kz b_xi),
//     rho_zi = i (ky b_xi - kx b_yi) (kz = 0 in 2-D), no mask;
//  8: the Rodrigues vector from the Nye density b = rho (CalculateRotationRodrigues L472-494, source
//     'rho'): kmask sum_mn D_imn b_mn, D_imn = i (2 k_n d_im - k_m d_in - k_i d_mn) / (2 kSq)
//     + i k_i k_n k_m / (2 kSqSq), i.e. i [(2 q_i - p_i - k_i s) / kSq + k_i r / kSqSq] / 2 with
//     q = b k, p = b^T k, s = tr b, r = k . b k.
// Inputs: 6 symmetric components xx xy xz yy yz zz (3-5) or all 9 (6, 8). The k values are those of
// the table the launch passes (the wrapped identity or, for 'sinK', the sine tables).
template <typename T, typename V, int GMODE>
__device__ __forceinline__ void obs_point(const V* b, V* o, T kx, T ky, T kz, bool kzero, T A, T B, T scale) {
    const T k[3] = {kx, ky, kz};
    if constexpr (GMODE == 8) {
        const T ksq = kx * kx + ky * ky + kz * kz;
        const T ikse = (T)1 / (ksq + (T)ME);
        const T ikqe = (T)1 / (ksq * ksq + (T)ME);
        const T f = (kzero ? (T)0 : (T)1) * (T)0.5 * scale;
        V q[3], p[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            q[i].x = b[3 * i].x * k[0] + b[3 * i + 1].x * k[1] + b[3 * i + 2].x * k[2];
            q[i].y = b[3 * i].y * k[0] + b[3 * i + 1].y * k[1] + b[3 * i + 2].y * k[2];
            p[i].x = k[0] * b[i].x + k[1] * b[3 + i].x + k[2] * b[6 + i].x;
            p[i].y = k[0] * b[i].y + k[1] * b[3 + i].y + k[2] * b[6 + i].y;
        }
        const V s1 = vadd(vadd(b[0], b[4]), b[8]);
        V r;
        r.x = k[0] * q[0].x + k[1] * q[1].x + k[2] * q[2].x;
        r.y = k[0] * q[0].y + k[1] * q[1].y + k[2] * q[2].y;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            V t;   // (2 q_i - p_i - k_i s) / kSq + k_i r / kSqSq, then times i f
            t.x = ((T)2 * q[i].x - p[i].x - k[i] * s1.x) * ikse + k[i] * r.x * ikqe;
            t.y = ((T)2 * q[i].y - p[i].y - k[i] * s1.y) * ikse + k[i] * r.y * ikqe;
            o[i].x = -t.y * f;
            o[i].y = t.x * f;
        }
        return;
    } else if constexpr (GMODE == 6) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const V bx = b[i], by = b[3 + i], bz = b[6 + i];
            V u[3];
            u[0].x = kz * by.x - ky * bz.x; u[0].y = kz * by.y - ky * bz.y;
            u[1].x = kx * bz.x - kz * bx.x; u[1].y = kx * bz.y - kz * bx.y;
            u[2].x = ky * bx.x - kx * by.x; u[2].y = ky * bx.y - kx * by.y;
#pragma unroll
            for (int a = 0; a < 3; ++a) {   // multiply by i
                o[3 * a + i].x = -u[a].y * scale;
                o[3 * a + i].y = u[a].x * scale;
            }
        }
        return;
    } else {
        const V b9[9] = {b[0], b[1], b[2], b[1], b[3], b[4], b[2], b[4], b[5]};
        const T ksq = kx * kx + ky * ky + kz * kz;
        const T ikse = (T)1 / (ksq + (T)ME);
        const T mask = kzero ? (T)0 : (T)1;
        V q[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            q[j].x = b9[3 * j].x * k[0] + b9[3 * j + 1].x * k[1] + b9[3 * j + 2].x * k[2];
            q[j].y = b9[3 * j].y * k[0] + b9[3 * j + 1].y * k[1] + b9[3 * j + 2].y * k[2];
        }
        if constexpr (GMODE == 5) {
            const T f = mask * ikse * scale;
            o[0].x = f * (k[1] * q[2].x - k[2] * q[1].x); o[0].y = f * (k[1] * q[2].y - k[2] * q[1].y);
            o[1].x = f * (k[2] * q[0].x - k[0] * q[2].x); o[1].y = f * (k[2] * q[0].y - k[0] * q[2].y);
            o[2].x = f * (k[0] * q[1].x - k[1] * q[0].x); o[2].y = f * (k[0] * q[1].y - k[1] * q[0].y);
            return;
        } else {
            const T ikqe = (T)1 / (ksq * ksq + (T)ME);
            V s1 = vadd(vadd(b9[0], b9[4]), b9[8]);
            V r;
            r.x = k[0] * q[0].x + k[1] * q[1].x + k[2] * q[2].x;
            r.y = k[0] * q[0].y + k[1] * q[1].y + k[2] * q[2].y;
            V cc;
            cc.x = A * s1.x * ikse - B * r.x * ikqe;
            cc.y = A * s1.y * ikse - B * r.y * ikqe;
            V g[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                g[j].x = mask * scale * (k[j] * cc.x + (q[j].x + q[j].x) * ikse);
                g[j].y = mask * scale * (k[j] * cc.y + (q[j].y + q[j].y) * ikse);
            }
            if constexpr (GMODE == 3) {
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) { o[3 * i + j].x = k[i] * g[j].x; o[3 * i + j].y = k[i] * g[j].y; }
            } else {
                const int ia[3] = {0, 0, 1}, ja[3] = {1, 2, 2};
                const T hf = (T)0.5;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int i = ia[c], j = ja[c];
                    o[c].x = hf * (k[i] * g[j].x - k[j] * g[i].x);
                    o[c].y = hf * (k[i] * g[j].y - k[j] * g[i].y);
                }
            }
        }
    }
}

// Shared memory: component slots of N x W (+W pad), the last three being the ping-pong scratch
// (slot `scr` on). The transforms run three components at a time against the scratch; when the
// stage count is odd the result is copied back to the component slots.
template <typename V, bool INV, int K>
__device__ __forceinline__ void fft_group(V* s, int g, int lgw, int cs, const LinePlan& lp,
                                          const V* __restrict__ tws, int tid, int nt, int scr) {
    V* a = s + K * g * cs;
    V* b = s + scr * cs;   // scratch slots
    ColLayout<K> lay{lgw, cs};
    V* r = fft_lines<V, INV>(a, b, lay, lp, tws, tid, nt, lp.twst[0]);
    if (r != a) {
        for (int i = tid; i < K * cs; i += nt) a[i] = b[i];
        __syncthreads();
    }
}

// phi (optional, one complex value per k point, laid out like one spectrum component with the
// instance base spoff / 9): GMODE 0 writes phi of the input; GMODE 1 reads the phi of the state
// whose stress the cotangent belongs to and writes, per block, the partial Parseval sum
// sum_k w_k Re(conj(sigbar_hat) . (2 mu k k + lam kSq I) phi) / cells (w_k = 1 on the first and
// the Nyquist half-axis column, 2 elsewhere): the A/B part of <sigbar, (d sigma / d nu) beta>
// per unit dA.
// One column tile of the k-space pass: W = 2^lgw spectrum columns from ta W of row i1 (3-D) of
// instance ii. k_green calls it with lgw as a literal for the usual tile widths, so that the
// shared-memory offsets of the transforms fold to constants.
template <typename T, bool MEAN64, int GMODE>
__device__ __forceinline__ void green_tile(const InstDev& I, int ii, int ta, int i1, int lgw,
                                           typename VecOf<T>::type* s,
                                           typename VecOf<T>::type* __restrict__ spec,
                                           const typename VecOf<T>::type* __restrict__ tw,
                                           const T* __restrict__ ktab,
                                           typename VecOf<T>::type* __restrict__ phi,
                                           double* __restrict__ part,
                                           const InstClock* __restrict__ clk) {
    typedef typename VecOf<T>::type V;
    const int W = 1 << lgw;
    const int N = I.n0, nhp = I.nhp, nh = I.nh;
    const int col0 = ta * W;
    const int wv = min(W, nh - col0);
    const int tid = threadIdx.x, nt = blockDim.x;
    const int cs = N * W + W;          // padded component slot in shared memory
    const long long estride = (I.nd == 3) ? (long long)I.n1 * nhp : (long long)nhp;
    const long long cstride = (long long)N * estride;
    V* base = spec + I.spoff + (I.nd == 3 ? (long long)i1 * nhp : 0) + col0;

    // components in / out of the k-space pass: sym(beta) -> sigma (0), sigma cotangent -> cotangent of
    // sym(beta) (1), sym(beta) -> d sigma / d nu (2), all 6 -> 6; the observables sym(beta) ->
    // beta^E (3, 6 -> 9), -> rotation (4, 6 -> 3), -> Rodrigues vector (5, 6 -> 3), beta -> Nye
    // density (6, 9 -> 9)
    constexpr int NIN = green_nin(GMODE);
    constexpr int NOUT = green_nout(GMODE);
    constexpr int SCR = green_slots(GMODE) - 3;   // first scratch slot
    constexpr int KG = green_group(GMODE);
    if (GMODE == 7 && !I.vacancy) return;
    V* tws = s + ((green_slots(GMODE) * cs + 1) & ~1);   // twiddle rows after the slots
    // forward: all six component tiles staged at once (16-byte asynchronous copies keep the whole
    // tile in flight), then the axis-0 transforms in shared memory
    if (W * (int)sizeof(V) >= 16) {
#pragma unroll 1
        for (int c = 0; c < NIN; ++c) tile_async_load(s + c * cs, base + c * cstride, estride, N, lgw, wv, tid, nt);
    } else {
#pragma unroll 1
        for (int c = 0; c < NIN; ++c) {
#pragma unroll 8
            for (int rem = tid; rem < N * W; rem += nt) {
                const int e = rem >> lgw, w = rem & (W - 1);
                V z; z.x = 0; z.y = 0;
                if (w < wv) z = base[c * cstride + e * estride + w];
                s[c * cs + rem] = z;
            }
        }
    }
    stage_tw_to_smem(I.lp_first, tw, tws, tid, nt);
    cp_async_wait_all();
    __syncthreads();
    for (int g = 0; g < NIN / KG; ++g) fft_group<V, false, KG>(s, g, lgw, cs, I.lp_first, tws, tid, nt, SCR);
    // vacancy diffusion factor exp(-gamma dt kSq) (VacancyDynamics.DiffusionEvolution L41-61), dt of
    // the step just taken
    const T vg = (GMODE == 7) ? (T)(-I.vac_gamma) : (T)0;
    const T vdt = (GMODE == 7) ? (T)clk[ii].dt : (T)0;
    // Green contraction, one k point per thread iteration
    const T lam = (T)I.lamb, mu = (T)I.mu;
    const T A = (T)(I.lamb / (I.lamb + 2.0 * I.mu));
    const T B = (T)(2.0 * (I.lamb + I.mu) / (I.lamb + 2.0 * I.mu));
    const T scale = (T)I.inv_cells;
    V* phib = phi ? phi + I.spoff / 9 + (I.nd == 3 ? (long long)i1 * nhp : 0) + col0 : nullptr;
    double pacc = 0.0;
    for (int i = tid; i < N * W; i += nt) {
        const int e = i >> lgw, w = i & (W - 1);
        int kh = col0 + w;
        if (w >= wv) continue;
        T kx, ky, kz;
        bool kzero;
        if (I.nd == 3) {
            kx = ktab[I.koff0 + e];
            ky = ktab[I.koff1 + i1];
            kz = ktab[I.koffh + kh];
            kzero = (e == 0 && i1 == 0 && kh == 0);
        } else {
            kx = ktab[I.koff0 + e];
            ky = ktab[I.koffh + kh];
            kz = (T)0;
            kzero = (e == 0 && kh == 0);
        }
        V b[NIN], o[NOUT];
#pragma unroll
        for (int c = 0; c < NIN; ++c) b[c] = s[c * cs + i];
        if constexpr (GMODE == 7) {
            const T ksq = kx * kx + ky * ky + kz * kz;
            const T f = exp(ksq * vg * vdt) * scale;
            o[0].x = b[0].x * f;
            o[0].y = b[0].y * f;
        } else if constexpr (GMODE >= 3) {
            obs_point<T, V, GMODE>(b, o, kx, ky, kz, kzero, A, B, scale);
        } else if constexpr (GMODE == 0) {
            // the symmetric 3 x 3 matrix of the six components (row-major, b9[3i + j])
            const V b9[9] = {b[0], b[1], b[2], b[1], b[3], b[4], b[2], b[4], b[5]};
            V ph;
            green_point<T, V>(b9, o, kx, ky, kz, kzero, lam, mu, A, B, scale, MEAN64, phib ? &ph : nullptr);
            if (phib) phib[e * estride + w] = ph;
        } else if constexpr (GMODE == 1) {
            if (phib) {
                const V ph = phib[e * estride + w];
                const double k3[3] = {(double)kx, (double)ky, (double)kz};
                const double ksq = k3[0] * k3[0] + k3[1] * k3[1] + k3[2] * k3[2];
                const int ia[6] = {0, 0, 0, 1, 1, 2}, ja[6] = {0, 1, 2, 1, 2, 2};
                double acc = 0.0;
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    double cf = 2.0 * (double)I.mu * k3[ia[c]] * k3[ja[c]];
                    if (ia[c] == ja[c]) cf += I.lamb * ksq;
                    acc += cf * ((double)b[c].x * (double)ph.x + (double)b[c].y * (double)ph.y);
                }
                const bool edge = (kh == 0) || (2 * kh == I.nl);
                pacc += (edge ? 1.0 : 2.0) * acc;
            }
            V bb[9];
            green_point_adj<T, V>(b, bb, kx, ky, kz, kzero, lam, mu, A, B, scale);
            // cotangent of beta_ij (= of beta_ji) through s_ij = (beta_ij + beta_ji) / 2
            const T hf = (T)0.5;
            o[0] = bb[0];
            o[1].x = hf * (bb[1].x + bb[3].x); o[1].y = hf * (bb[1].y + bb[3].y);
            o[2].x = hf * (bb[2].x + bb[6].x); o[2].y = hf * (bb[2].y + bb[6].y);
            o[3] = bb[4];
            o[4].x = hf * (bb[5].x + bb[7].x); o[4].y = hf * (bb[5].y + bb[7].y);
            o[5] = bb[8];
        } else {
            const V b9[9] = {b[0], b[1], b[2], b[1], b[3], b[4], b[2], b[4], b[5]};
            green_point_dnu<T, V>(b9, o, kx, ky, kz, kzero, lam, mu, A, B, scale, (T)I.nu);
        }
#pragma unroll
        for (int c = 0; c < NOUT; ++c) s[c * cs + i] = o[c];
    }
    if (GMODE == 1 && part) {
        // fixed-order block reduction (deterministic); the FFT below re-synchronises the block
        __shared__ double red[GREEN_THREADS / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) pacc += __shfl_xor_sync(0xffffffffu, pacc, o);
        if ((tid & 31) == 0) red[tid >> 5] = pacc;
        __syncthreads();
        if (tid == 0) {
            double sum = 0.0;
            for (int w = 0; w < nt / 32; ++w) sum += red[w];
            part[blockIdx.x] = sum * I.inv_cells;
        }
    }
    __syncthreads();
    if (line_plan_io(I.lp_first)) {
        // inverse transforms from the component slots straight to global memory
        const SColT<V, KG> scratch{s + SCR * cs, lgw, cs};
#pragma unroll 1
        for (int g = 0; g < NOUT / KG; ++g) {
            const SColT<V, KG> slots{s + KG * g * cs, lgw, cs};
            const GColT<V, KG> gout{base + KG * g * cstride, estride, cstride, lgw, wv};
            fft_io<V, true, KG>(slots, scratch, slots, gout, lgw, I.lp_first, tws, tid, nt, I.lp_first.twst[0]);
        }
        return;
    }
    for (int g = 0; g < NOUT / KG; ++g) fft_group<V, true, KG>(s, g, lgw, cs, I.lp_first, tws, tid, nt, SCR);
    if (W * (int)sizeof(V) >= 16) {
#pragma unroll 1
        for (int c = 0; c < NOUT; ++c) tile_store(base + c * cstride, s + c * cs, estride, N, lgw, wv, tid, nt);
    } else {
#pragma unroll 1
        for (int c = 0; c < NOUT; ++c) {
#pragma unroll 4
            for (int rem = tid; rem < N * W; rem += nt) {
                const int e = rem >> lgw, w = rem & (W - 1);
                if (w < wv) base[c * cstride + e * estride + w] = s[c * cs + rem];
            }
        }
    }
}

template <typename T, bool MEAN64, int GMODE>
__global__ void __launch_bounds__(GREEN_THREADS, sizeof(T) == 4 ? 3 : 2) k_green(const InstDev* __restrict__ insts, int n_inst,
                                                         const int* __restrict__ pre,
                                                         typename VecOf<T>::type* __restrict__ spec,
                                                         const typename VecOf<T>::type* __restrict__ tw,
                                                         const T* __restrict__ ktab,
                                                         typename VecOf<T>::type* __restrict__ phi,
                                                         double* __restrict__ part,
                                                         const InstClock* __restrict__ clk) {
    typedef typename VecOf<T>::type V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* s = reinterpret_cast<V*>(smem_raw);
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    int lb = blockIdx.x - pre[ii];
    const PassTile& tl = I.tile[PASS_GREEN];
    const int lgw = tl.lgw, ta_n = tl.tiles_a;
    const int ta = lb % ta_n;
    const int i1 = lb / ta_n;          // 0 in 2-D
    // the FP32 stress solve (GMODE 0) at the built-in tile width (4 columns) and 8 (measured: 1.5%
    // faster at 256^3, 3% at 96^3; FP64 kept the general form, which measured no slower)
    if constexpr (GMODE == 0 && sizeof(T) == 4) {
        if (lgw == 2) {
            green_tile<T, MEAN64, GMODE>(I, ii, ta, i1, 2, s, spec, tw, ktab, phi, part, clk);
            return;
        }
        if (lgw == 3) {
            green_tile<T, MEAN64, GMODE>(I, ii, ta, i1, 3, s, spec, tw, ktab, phi, part, clk);
            return;
        }
    }
    green_tile<T, MEAN64, GMODE>(I, ii, ta, i1, lgw, s, spec, tw, ktab, phi, part, clk);
}

// ------------------------------------------------------------------------------------------
// Plane passes (3-D FP32 instances that plane_eligible accepts): the transforms along the
// contiguous axis and along axis 1 of one z-plane of one component in one kernel each way, so the
// spectrum crosses HBM once between them instead of twice. One cluster of PLANE_C blocks per
// (component o, plane z); block r owns rows [r Rc, (r+1) Rc) of the plane (Rc = n1 / PLANE_C) and
// spectrum columns [r W, (r+1) W) (W = nl / (2 PLANE_C)). Data moves between the blocks of a
// cluster by stores into the owner's shared memory (distributed shared memory), which do not stall
// the storing thread:
//   forward: block r runs the R2C of its rows (two real rows per complex FFT, as k_r2c_rows); the
//     last FFT stage stores each half-spectrum bin straight into the shared column tile S_col of
//     the block that owns its column; after a cluster barrier every block transforms its W columns
//     along axis 1 and writes them to the plan's spectrum, which the k-space pass (k_green) reads
//     as before;
//   inverse: block r runs the inverse axis-1 transform of its W columns, the first stage reading
//     them from the spectrum and the last stage storing each value into the shared row tile S_own
//     of the block that owns its row; after a cluster barrier every block runs the C2R of its rows
//     (plus the FP64 mean stress) into sigma.
// Every kernel starts with a cluster barrier, so no block stores into a block that has not started.
// Columns 0 and nl/2 of a row's half spectrum are real (the R2C split makes their imaginary parts
// exactly zero), so block 0 carries them as one complex column X0 + i X_{nl/2}; its axis-1
// transform F = F0 + i FN is split again by Hermitian symmetry, F0(ky) = (F(ky) + conj F(-ky)) / 2,
// FN(ky) = (F(ky) - conj F(-ky)) / (2i). The inverse packs the Hermitian parts H(G)(ky) =
// (G(ky) + conj G(-ky)) / 2 of the two columns as H(G0) + i H(GN): the inverse transform of H(G) is
// the real part of that of G, which is what the C2R keeps of those bins (numpy's irfft semantics;
// the k tables' positive Nyquist values make the k-space operator's output not exactly Hermitian
// on the axis-1 Nyquist line). That keeps W columns per block, a power of two. Same codelets,
// twiddles and row tables as the separate passes; results agree with them to rounding.
// Shared memory (V = complex): forward: the row pass's line buffer (P x rows_ld(nl); then the
// axis-1 scratch tile, n1 x W) and S_col (n1 x W); inverse: S_own (Rc x ldo) and a buffer of
// max(n1 x W, P x rows_ld(nl)) (the axis-1 scratch tile, then the C2R line buffer); both: the row
// twiddles and the row tables.
// ------------------------------------------------------------------------------------------
constexpr int PLANE_C = PLANE_CLUSTER;

struct PlaneGeom {
    int Rc, P, W, lgw, ldo, ld;
    size_t a, b, tw, tab, total;   // region sizes in bytes (16-byte multiples) and the sum
};

__host__ __device__ inline PlaneGeom plane_geom(const InstDev& I, size_t velt) {
    PlaneGeom g;
    g.Rc = I.n1 / PLANE_C;
    g.P = g.Rc / 2;
    g.W = (I.nl / 2) / PLANE_C;
    g.lgw = 0;
    while ((1 << g.lgw) < g.W) ++g.lgw;
    g.ldo = (I.nh + 1) & ~1;   // even: 16-byte aligned FP32 rows
    g.ld = rows_ld(I.nl);
    auto r16 = [](size_t v) { return (v + 15) & ~(size_t)15; };
    const size_t colt = (size_t)I.n1 * g.W * velt;
    const size_t own = (size_t)g.Rc * g.ldo * velt, line = (size_t)g.P * g.ld * velt;
    // region a: forward line buffer / axis-1 scratch, inverse S_own; region b: forward S_col,
    // inverse axis-1 scratch / C2R line buffer
    const size_t fa = line > colt ? line : colt, ia = own;
    const size_t fb = colt, ib = line > colt ? line : colt;
    g.a = r16(fa > ia ? fa : ia);
    g.b = r16(fb > ib ? fb : ib);
    g.tw = r16((size_t)I.lp_last.twspan * velt);
    g.tab = r16(rows_table_bytes(g.P));
    g.total = g.a + g.b + g.tw + g.tab;
    return g;
}

// Whether instance I runs its stress transforms through the plane passes (FP32 plans): n1 and nl
// powers of two with Rc = n1 / PLANE_C an even number of rows, at least two columns per block, the
// register-resident two-stage row codelets (rows_io_plan) and a two-stage compile-time axis-1 plan.
bool plane_eligible(const InstDev& I, int precision, size_t smem_limit) {
    if (precision != CDD_F32 || I.nd != 3) return false;
    auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
    if (!pow2(I.n1) || !pow2(I.nl)) return false;
    if (I.n1 % (2 * PLANE_C) != 0 || (I.nl / 2) % (2 * PLANE_C) != 0) return false;
    const PlaneGeom g = plane_geom(I, sizeof(float2));
    if (!rows_io_plan(I.lp_last, g.P)) return false;
    if (!(line_plan_io(I.lp_mid) && I.lp_mid.nst == 2)) return false;
    return g.total + 1024 <= smem_limit;
}

size_t plane_smem_bytes(const InstDev& I) { return plane_geom(I, sizeof(float2)).total; }

// Forward: bin k of rows y0 + 2q and y0 + 2q + 1 of the plane goes to the column tile S_col of the
// block owning column k (element (y, w) at (y << lgw) + w); bins 0 and nl/2 (real) to the real and
// imaginary parts of block 0's column 0.
template <typename V> struct PlaneColSink {
    V* s_col;   // this block's S_col (the same offset in every block of the cluster)
    int y0, lgw, half;
    __device__ __forceinline__ void operator()(long long q, int k, const V& a, const V& b, bool) const {
        cg::cluster_group cl = cg::this_cluster();
        const int y = y0 + 2 * (int)q;
        if (k == 0 || k == half) {
            V* d = cl.map_shared_rank(s_col, 0);
            if (k == 0) {
                d[y << lgw].x = a.x;
                d[(y + 1) << lgw].x = b.x;
            } else {
                d[y << lgw].y = a.x;
                d[(y + 1) << lgw].y = b.x;
            }
        } else {
            const int w = k & ((1 << lgw) - 1);
            V* d = cl.map_shared_rank(s_col, k >> lgw);
            d[(y << lgw) + w] = a;
            d[((y + 1) << lgw) + w] = b;
        }
    }
};

// Inverse, first axis-1 stage: element ky of column w of this block read from the spectrum; block
// 0's column 0 is H(G0) + i H(GN) of spectrum columns 0 and nl/2.
template <typename V> struct PlaneSpecIn {
    const V* src;   // the plane's first spectrum row, at this block's first column
    long long nhp;
    int n1, half;
    bool packed;    // block 0: column 0 carries bins 0 and nl/2
    struct Walk {
        const V* p;       // element i0 of the column
        const V* base;    // row 0 of the plane at column 0 (packed column)
        long long stride, nhp;
        int i0, step, n1, half;
        bool packed;
        __device__ __forceinline__ V ld(int r) const {
            if (!packed) return p[r * stride];
            typedef decltype(V().x) T;
            const int ky = i0 + r * step, km = ky == 0 ? 0 : n1 - ky;
            const V* sr = base + (long long)ky * nhp;
            const V* sm = base + (long long)km * nhp;
            const V f0 = sr[0], f0m = sm[0], fn = sr[half], fnm = sm[half];
            const T ax = (T)0.5 * (f0.x + f0m.x), ay = (T)0.5 * (f0.y - f0m.y);
            const T bx = (T)0.5 * (fn.x + fnm.x), by = (T)0.5 * (fn.y - fnm.y);
            V v;
            v.x = ax - by;
            v.y = ay + bx;
            return v;
        }
    };
    __device__ __forceinline__ Walk walk(int l, int i0, int step) const {
        return {src + (long long)i0 * nhp + l, src, (long long)step * nhp, nhp, i0, step, n1, half, packed && l == 0};
    }
};

// Inverse, last axis-1 stage: element y of column w stored into the row tile S_own of the block
// owning row y (row ly at ly * ldo); block 0's column 0 is unpacked into bins 0 and nl/2 (real).
template <typename V> struct PlaneRowOut {
    V* s_own;
    int col0, lrc, ldo, half;
    bool packed;
    struct Walk {
        V* s_own;
        int i0, step, kx, lrc, ldo, half;
        bool packed;
        __device__ __forceinline__ void st(int r, V v) const {
            cg::cluster_group cl = cg::this_cluster();
            const int y = i0 + r * step;
            const int q = y >> lrc, ly = y & ((1 << lrc) - 1);
            V* d = cl.map_shared_rank(s_own, q) + ly * ldo;
            if (packed) {
                V a, b;
                a.x = v.x; a.y = 0;
                b.x = v.y; b.y = 0;
                d[0] = a;
                d[half] = b;
            } else {
                d[kx] = v;
            }
        }
    };
    __device__ __forceinline__ Walk walk(int l, int i0, int step) const {
        return {s_own, i0, step, col0 + l, lrc, ldo, half, packed && l == 0};
    }
};

// F0: beta holds the stage-1 rhs; the kernel forms F0 = u + dt rhs row by row (dt from the
// instance's clock), writes it back over rhs and transforms it (see r2c_rows_io).
template <typename T, bool F0>
__global__ void __cluster_dims__(PLANE_C, 1, 1) __launch_bounds__(ROW_THREADS, 3)
k_plane_fwd(const InstDev* __restrict__ insts, int n_inst, const int* __restrict__ pre, const T* beta,
            typename VecOf<T>::type* __restrict__ spec, const typename VecOf<T>::type* __restrict__ tw,
            double* __restrict__ rowsum, T* f0w, const T* __restrict__ u, const InstClock* __restrict__ clk) {
    typedef typename VecOf<T>::type V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();   // every block of the cluster runs before any stores into another
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    const int lb = blockIdx.x - pre[ii];
    const int rank = (int)cl.block_rank();
    const int q = lb / PLANE_C;              // o * n0 + z
    const int o = q / I.n0, z = q - o * I.n0;
    const PlaneGeom g = plane_geom(I, sizeof(V));
    const int N = I.nl, n1 = I.n1, W = g.W, lgw = g.lgw, P = g.P;
    V* s_line = reinterpret_cast<V*>(smem_raw);            // line buffer, then the axis-1 scratch tile
    V* s_col = reinterpret_cast<V*>(smem_raw + g.a);
    V* tws = reinterpret_cast<V*>(smem_raw + g.a + g.b);
    RowPtr* rt = reinterpret_cast<RowPtr*>(smem_raw + g.a + g.b + g.tw);
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long nrows = 6LL * I.rows, npairs = nrows / 2;
    const long long plane_row = (long long)o * I.rows + (long long)z * n1;   // first row of the plane
    const long long row0 = plane_row + (long long)rank * g.Rc;
    const long long p0 = row0 / 2;
    const int lbv = (int)(p0 / P);           // the row pass's block index of these rows
    for (int r = tid; r < 2 * P; r += nt) {
        const T *pa, *qa;
        src_rows(I, beta, RS_SYM, row0 + r, pa, qa);
        RowPtr e;
        e.p = pa - beta;
        e.q = qa - beta;
        rt[r] = e;
    }
    stage_tw_to_smem(I.lp_last, tw, tws, tid, nt);
    __syncthreads();
    {
        const LinePlan& lq = I.lp_last;
        const V* tw1 = tws + (lq.twst[1] - lq.twst[0]);
        constexpr bool MEAN64 = sizeof(T) == 4;
        const T dt = F0 ? (T)clk[ii].dt : (T)0;
        const PlaneColSink<V> sink{s_col, rank * g.Rc, lgw, N / 2};
#define CDD_PLANE_R2C(A, B)                                                                                 \
        r2c_rows_io<T, MEAN64, A, B, F0>(I, lbv, P, g.ld, rt, beta, s_line, tw1, sink, rowsum, nrows, npairs, \
                                         tid, nt, p0, f0w, u, dt)
        if (lq.radix[0] == 16 && lq.radix[1] == 16) CDD_PLANE_R2C(16, 16);
        else if (lq.radix[0] == 16 && lq.radix[1] == 8) CDD_PLANE_R2C(16, 8);
        else if (lq.radix[0] == 16 && lq.radix[1] == 4) CDD_PLANE_R2C(16, 4);
        else CDD_PLANE_R2C(8, 4);
#undef CDD_PLANE_R2C
    }
    cl.sync();   // every half-spectrum bin of the plane is in its owner's S_col
    SColT<V, 1> col{s_col, lgw, 0}, scr{s_line, lgw, 0};
    fft_io<V, false, 1>(col, scr, scr, col, lgw, I.lp_mid, tw, tid, nt, 0);
    V* dst = spec + I.spoff + plane_row * I.nhp;
    for (int e = tid; e < n1 * W; e += nt) {
        const int ky = e >> lgw, w = e & (W - 1);
        const V v = s_col[e];
        V* d = dst + (long long)ky * I.nhp;
        if (rank == 0 && w == 0) {
            const int km = (ky == 0) ? 0 : n1 - ky;
            const V zm = s_col[km << lgw];
            V a, b;
            a.x = (T)0.5 * (v.x + zm.x);
            a.y = (T)0.5 * (v.y - zm.y);
            b.x = (T)0.5 * (v.y + zm.y);
            b.y = (T)-0.5 * (v.x - zm.x);
            d[0] = a;
            d[N / 2] = b;
        } else {
            d[rank * W + w] = v;
        }
    }
}

template <typename T>
__global__ void __cluster_dims__(PLANE_C, 1, 1) __launch_bounds__(ROW_THREADS, 3)
k_plane_inv(const InstDev* __restrict__ insts, int n_inst, const int* __restrict__ pre,
            const typename VecOf<T>::type* __restrict__ spec, T* __restrict__ out,
            const typename VecOf<T>::type* __restrict__ tw, const double* __restrict__ sbar) {
    typedef typename VecOf<T>::type V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();   // every block of the cluster runs before any stores into another
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    const int lb = blockIdx.x - pre[ii];
    const int rank = (int)cl.block_rank();
    const int q = lb / PLANE_C;
    const int o = q / I.n0, z = q - o * I.n0;
    const PlaneGeom g = plane_geom(I, sizeof(V));
    const int N = I.nl, n1 = I.n1, lgw = g.lgw, ldo = g.ldo, P = g.P;
    V* s_own = reinterpret_cast<V*>(smem_raw);
    V* s_buf = reinterpret_cast<V*>(smem_raw + g.a);      // axis-1 scratch tile, then the C2R line buffer
    V* tws = reinterpret_cast<V*>(smem_raw + g.a + g.b);
    RowPtr* rt = reinterpret_cast<RowPtr*>(smem_raw + g.a + g.b + g.tw);
    RowPtr* re = rt + 2 * P;
    double* rmean = reinterpret_cast<double*>(re + 2 * P);
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long nrows = 6LL * I.rows, npairs = nrows / 2;
    const long long plane_row = (long long)o * I.rows + (long long)z * n1;
    const long long row0 = plane_row + (long long)rank * g.Rc;
    const long long p0 = row0 / 2;
    const int lbv = (int)(p0 / P);
    constexpr bool MEAN64 = sizeof(T) == 4;
    for (int r = tid; r < 2 * P; r += nt) {
        T *pd, *qd;
        dst_rows(I, out, RD_STRESS, row0 + r, pd, qd);
        RowPtr e, ep;
        e.p = pd - out;
        e.q = qd - out;
        ep.p = ep.q = -1;
        rt[r] = e;
        re[r] = ep;
        rmean[r] = MEAN64 ? mean_stress(I, sbar + 9 * ii, o) : 0.0;
    }
    stage_tw_to_smem(I.lp_last, tw, tws, tid, nt);
    {
        const PlaneSpecIn<V> in{spec + I.spoff + plane_row * I.nhp + rank * g.W, I.nhp, n1, N / 2, rank == 0};
        const PlaneRowOut<V> rows{s_own, rank * g.W, 31 - __clz(g.Rc), ldo, N / 2, rank == 0};
        SColT<V, 1> scr{s_buf, lgw, 0};
        fft_io<V, true, 1>(in, scr, scr, rows, lgw, I.lp_mid, tw, tid, nt, 0);
    }
    cl.sync();   // every row of every block's S_own is complete; no block reads the scratch tiles
    {
        const LinePlan& lq = I.lp_last;
        const V* tw1 = tws + (lq.twst[1] - lq.twst[0]);
#define CDD_PLANE_C2R(A, B)                                                                                   \
        c2r_rows_io<T, MEAN64, A, B>(I, lbv, P, g.ld, rt, re, rmean, s_own, s_buf, tw1, out, nullptr, EPI_NONE, \
                                     nrows, npairs, tid, nt, p0, ldo)
        if (lq.radix[0] == 16 && lq.radix[1] == 16) CDD_PLANE_C2R(16, 16);
        else if (lq.radix[0] == 16 && lq.radix[1] == 8) CDD_PLANE_C2R(16, 8);
        else if (lq.radix[0] == 16 && lq.radix[1] == 4) CDD_PLANE_C2R(16, 4);
        else CDD_PLANE_C2R(8, 4);
#undef CDD_PLANE_C2R
    }
}

// ------------------------------------------------------------------------------------------
// FP32 plans: FP64 mean of each beta component from the row sums. One cluster of MEAN_SPLIT blocks
// per (instance, component): each block sums a contiguous share of the rows (fixed-order strided
// sums and a fixed tree), block 0 of the cluster adds the shares from the blocks' shared memory
// (distributed shared memory) in rank order, so the result is deterministic.
// ------------------------------------------------------------------------------------------
constexpr int MEAN_SPLIT = 8;
__global__ void __cluster_dims__(1, 1, MEAN_SPLIT) __launch_bounds__(1024)
k_mean_beta(const InstDev* __restrict__ insts, const double* __restrict__ rowsum, double* __restrict__ mean9) {
    const InstDev& I = insts[blockIdx.x];
    const int c = blockIdx.y;
    cg::cluster_group cl = cg::this_cluster();
    const int part = (int)cl.block_rank();
    __shared__ double red[32];
    __shared__ double share;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int chunk = (I.rows + MEAN_SPLIT - 1) / MEAN_SPLIT;
    const int r0 = part * chunk, r1 = min(I.rows, r0 + chunk);
    const double* rs = rowsum + I.rsoff + (long long)c * I.rows;
    // four independent accumulators per thread keep several loads in flight; fixed order throughout
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    const int nt = blockDim.x;
    int r = r0 + tid;
    for (; r + 3 * nt < r1; r += 4 * nt) {
        a0 += rs[r];
        a1 += rs[r + nt];
        a2 += rs[r + 2 * nt];
        a3 += rs[r + 3 * nt];
    }
    for (; r < r1; r += nt) a0 += rs[r];
    double acc = (a0 + a1) + (a2 + a3);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int w = 0; w < (nt >> 5); ++w) s += red[w];
        share = s;
    }
    cl.sync();   // every block's share is written
    if (part == 0 && tid == 0) {
        double s = 0.0;
        for (int k = 0; k < MEAN_SPLIT; ++k) s += *cl.map_shared_rank(&share, k);
        mean9[9 * blockIdx.x + c] = s * I.inv_cells;
    }
    cl.sync();   // the shares stay in shared memory until block 0 has read them
}


// ------------------------------------------------------------------------------------------
// Host launch sequence
// ------------------------------------------------------------------------------------------
// u != null: beta holds the stage-1 rhs and the stress is that of F0 = u + dt rhs, formed in place
// first: by the plane instances' forward pass while it transforms the rows (fused), by the axpy
// kernel for the others (it skips the plane instances). A fused F0 in the separate row pass was
// measured slower: its write-back of F0 orders each row load after the previous store.
template <typename T>
static cudaError_t run_stress(const PlanCore& P, const void* beta, void* sigma, void* phi, cudaStream_t st,
                              const void* u = nullptr) {
    typedef typename VecOf<T>::type V;
    const bool f32 = (P.precision == CDD_F32);
    V* spec = (V*)P.d_spec;
    const V* tw = (const V*)P.d_tw;
    const LaunchShape* L = P.pass;
    // instances with the fused plane passes (FP32 only) skip the separate row and axis-1 passes
    const bool plane = std::is_same<T, float>::value && P.plane.blocks > 0;
    const LaunchShape* LR = plane ? P.rest : P.pass;
    if (u && LR[PASS_R2C].blocks > 0) {   // the other instances form F0 with the axpy kernel first
        cudaError_t e = launch_axpy_f0(P, u, const_cast<void*>(beta), st);
        if (e != cudaSuccess) return e;
    }
    if constexpr (std::is_same<T, float>::value) {
        if (plane && u)
            k_plane_fwd<T, true><<<P.plane.blocks, P.plane.threads, P.plane.smem, st>>>(
                P.d_inst, P.n_inst, P.plane.d_pre, (const T*)beta, spec, tw, P.d_rowsum, (T*)beta, (const T*)u,
                P.d_clock);
        else if (plane)
            k_plane_fwd<T, false><<<P.plane.blocks, P.plane.threads, P.plane.smem, st>>>(
                P.d_inst, P.n_inst, P.plane.d_pre, (const T*)beta, spec, tw, P.d_rowsum, nullptr, nullptr, nullptr);
    }
    if (f32) {
        if (LR[PASS_R2C].blocks > 0)
            k_r2c_rows<T, true><<<LR[PASS_R2C].blocks, LR[PASS_R2C].threads, LR[PASS_R2C].smem, st>>>(
                P.d_inst, P.n_inst, LR[PASS_R2C].d_pre, (const T*)beta, spec, tw, P.d_rowsum, RS_SYM, 6);
        k_mean_beta<<<dim3(P.n_inst, 6, MEAN_SPLIT), 1024, 0, st>>>(P.d_inst, P.d_rowsum, P.d_sbar);
    } else {
        k_r2c_rows<T, false><<<L[PASS_R2C].blocks, L[PASS_R2C].threads, L[PASS_R2C].smem, st>>>(
            P.d_inst, P.n_inst, L[PASS_R2C].d_pre, (const T*)beta, spec, tw, nullptr, RS_SYM, 6);
    }
    if (LR[PASS_MID_F].blocks > 0)
        k_fft_mid<T, false><<<LR[PASS_MID_F].blocks, LR[PASS_MID_F].threads, LR[PASS_MID_F].smem, st>>>(
            P.d_inst, P.n_inst, LR[PASS_MID_F].d_pre, spec, tw, PASS_MID_F, 6, 0);
    if (f32)
        k_green<T, true, 0><<<L[PASS_GREEN].blocks, L[PASS_GREEN].threads, L[PASS_GREEN].smem, st>>>(
            P.d_inst, P.n_inst, L[PASS_GREEN].d_pre, spec, tw, (const T*)P.d_k, (V*)phi, nullptr, nullptr);
    else
        k_green<T, false, 0><<<L[PASS_GREEN].blocks, L[PASS_GREEN].threads, L[PASS_GREEN].smem, st>>>(
            P.d_inst, P.n_inst, L[PASS_GREEN].d_pre, spec, tw, (const T*)P.d_k, (V*)phi, nullptr, nullptr);
    if (LR[PASS_MID_I].blocks > 0)
        k_fft_mid<T, true><<<LR[PASS_MID_I].blocks, LR[PASS_MID_I].threads, LR[PASS_MID_I].smem, st>>>(
            P.d_inst, P.n_inst, LR[PASS_MID_I].d_pre, spec, tw, PASS_MID_I, 6, 0);
    if constexpr (std::is_same<T, float>::value) {
        if (plane)
            k_plane_inv<T><<<P.plane.blocks, P.plane.threads, P.plane.smem, st>>>(
                P.d_inst, P.n_inst, P.plane.d_pre, spec, (T*)sigma, tw, P.d_sbar);
    }
    if (f32) {
        if (LR[PASS_C2R].blocks > 0)
            k_c2r_rows<T, true><<<LR[PASS_C2R].blocks, LR[PASS_C2R].threads, LR[PASS_C2R].smem, st>>>(
                P.d_inst, P.n_inst, LR[PASS_C2R].d_pre, spec, (T*)sigma, tw, P.d_sbar, RD_STRESS, 6, nullptr,
                EPI_NONE, nullptr);
    } else
        k_c2r_rows<T, false><<<L[PASS_C2R].blocks, L[PASS_C2R].threads, L[PASS_C2R].smem, st>>>(
            P.d_inst, P.n_inst, L[PASS_C2R].d_pre, spec, (T*)sigma, tw, nullptr, RD_STRESS, 6, nullptr, EPI_NONE, nullptr);
    return cudaGetLastError();
}

// Adjoint (GMODE 1: stress cotangent, 6 components in stress layout -> beta cotangent, written to all
// 9 components of a field) and the nu-derivative of the stress (GMODE 2: beta -> 6 components).
// Both keep the k = 0 mode in the transforms (no FP64 mean path).
template <typename T, int GMODE>
static cudaError_t run_stress_variant(const PlanCore& P, const void* in, void* out, const void* phi, double* part,
                                      cudaStream_t st) {
    typedef typename VecOf<T>::type V;
    V* spec = (V*)P.d_spec;
    const V* tw = (const V*)P.d_tw;
    const LaunchShape* L = P.pass;
    k_r2c_rows<T, false><<<L[PASS_R2C].blocks, L[PASS_R2C].threads, L[PASS_R2C].smem, st>>>(
        P.d_inst, P.n_inst, L[PASS_R2C].d_pre, (const T*)in, spec, tw, nullptr, GMODE == 1 ? RS_STRESS : RS_SYM, 6);
    if (L[PASS_MID_F].blocks > 0)
        k_fft_mid<T, false><<<L[PASS_MID_F].blocks, L[PASS_MID_F].threads, L[PASS_MID_F].smem, st>>>(
            P.d_inst, P.n_inst, L[PASS_MID_F].d_pre, spec, tw, PASS_MID_F, 6, 0);
    k_green<T, false, GMODE><<<L[PASS_GREEN].blocks, L[PASS_GREEN].threads, L[PASS_GREEN].smem, st>>>(
        P.d_inst, P.n_inst, L[PASS_GREEN].d_pre, spec, tw, (const T*)P.d_k, (V*)phi, part, nullptr);
    if (L[PASS_MID_I].blocks > 0)
        k_fft_mid<T, true><<<L[PASS_MID_I].blocks, L[PASS_MID_I].threads, L[PASS_MID_I].smem, st>>>(
            P.d_inst, P.n_inst, L[PASS_MID_I].d_pre, spec, tw, PASS_MID_I, 6, 0);
    k_c2r_rows<T, false><<<L[PASS_C2R].blocks, L[PASS_C2R].threads, L[PASS_C2R].smem, st>>>(
        P.d_inst, P.n_inst, L[PASS_C2R].d_pre, spec, (T*)out, tw, nullptr, GMODE == 1 ? RD_SYM_FIELD : RD_STRESS, 6, nullptr, EPI_NONE, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_stress_adjoint(const PlanCore& P, const void* sigbar6, void* betabar9, cudaStream_t st,
                                  const void* phi, double* part) {
    if (P.precision == CDD_F32) return run_stress_variant<float, 1>(P, sigbar6, betabar9, phi, part, st);
    return run_stress_variant<double, 1>(P, sigbar6, betabar9, phi, part, st);
}

cudaError_t launch_stress_dnu(const PlanCore& P, const void* beta, void* out6, cudaStream_t st) {
    if (P.precision == CDD_F32) return run_stress_variant<float, 2>(P, beta, out6, nullptr, nullptr, st);
    return run_stress_variant<double, 2>(P, beta, out6, nullptr, nullptr, st);
}

// Vacancy diffusion: the concentrations of the vacancy instances (one component) forward, times
// exp(-gamma dt kSq) in the axis-0 pass, inverse, written back for the instances whose step was
// applied. The stress passes' launch shapes carry it (blocks past one component exit).
template <typename T>
static cudaError_t run_vacancy_diffusion(const PlanCore& P, cudaStream_t st) {
    typedef typename VecOf<T>::type V;
    V* spec = (V*)P.d_spec;
    const V* tw = (const V*)P.d_tw;
    const LaunchShape* L = P.pass;
    k_r2c_rows<T, false><<<L[PASS_R2C].blocks, L[PASS_R2C].threads, L[PASS_R2C].smem, st>>>(
        P.d_inst, P.n_inst, L[PASS_R2C].d_pre, (const T*)P.d_vac, spec, tw, nullptr, RS_VAC, 1);
    if (L[PASS_MID_F].blocks > 0)
        k_fft_mid<T, false><<<L[PASS_MID_F].blocks, L[PASS_MID_F].threads, L[PASS_MID_F].smem, st>>>(
            P.d_inst, P.n_inst, L[PASS_MID_F].d_pre, spec, tw, PASS_MID_F, 1, 1);
    k_green<T, false, 7><<<L[PASS_GREEN].blocks, L[PASS_GREEN].threads, L[PASS_GREEN].smem, st>>>(
        P.d_inst, P.n_inst, L[PASS_GREEN].d_pre, spec, tw, (const T*)P.d_k, nullptr, nullptr, P.d_clock);
    if (L[PASS_MID_I].blocks > 0)
        k_fft_mid<T, true><<<L[PASS_MID_I].blocks, L[PASS_MID_I].threads, L[PASS_MID_I].smem, st>>>(
            P.d_inst, P.n_inst, L[PASS_MID_I].d_pre, spec, tw, PASS_MID_I, 1, 1);
    k_c2r_rows<T, false><<<L[PASS_C2R].blocks, L[PASS_C2R].threads, L[PASS_C2R].smem, st>>>(
        P.d_inst, P.n_inst, L[PASS_C2R].d_pre, spec, (T*)P.d_vac, tw, nullptr, RD_VAC, 1, nullptr, EPI_NONE,
        P.d_clock);
    return cudaGetLastError();
}

cudaError_t launch_vacancy_diffusion(const PlanCore& P, cudaStream_t st) {
    if (P.precision == CDD_F32) return run_vacancy_diffusion<float>(P, st);
    return run_vacancy_diffusion<double>(P, st);
}

// k-space observables: forward transforms of sym(beta) (6 components, the stress passes' launch
// shapes) or of all 9 components (the 9-component shapes), the observable's k-space operator in the
// fused axis-0 pass, inverse transforms of its 9 or 3 components with the real-space epilogue.
// No FP64 mean path: every operator's k = 0 mode is zero (kmask, or a factor k).
template <typename T, int GMODE>
static cudaError_t run_observable(const PlanCore& P, const void* beta, void* out, cudaStream_t st, bool sin_k) {
    typedef typename VecOf<T>::type V;
    V* spec = (V*)P.d_spec;
    const V* tw = (const V*)P.d_tw;
    constexpr int NIN = green_nin(GMODE), NOUT = green_nout(GMODE);
    constexpr int EPI = GMODE == 3 ? EPI_BETA_E : (GMODE == 4 ? EPI_ROTATION : (GMODE == 5 ? EPI_RODRIGUES : EPI_NONE));
    const LaunchShape* LI = (NIN == 9) ? P.pass9 : P.pass;
    const LaunchShape* LO = (NOUT == 9) ? P.pass9 : P.pass;
    const LaunchShape& LG = P.pass9[PASS_GREEN];
    k_r2c_rows<T, false><<<LI[PASS_R2C].blocks, LI[PASS_R2C].threads, LI[PASS_R2C].smem, st>>>(
        P.d_inst, P.n_inst, LI[PASS_R2C].d_pre, (const T*)beta, spec, tw, nullptr, NIN == 9 ? RS_FULL : RS_SYM, NIN);
    if (LI[PASS_MID_F].blocks > 0)
        k_fft_mid<T, false><<<LI[PASS_MID_F].blocks, LI[PASS_MID_F].threads, LI[PASS_MID_F].smem, st>>>(
            P.d_inst, P.n_inst, LI[PASS_MID_F].d_pre, spec, tw, PASS_MID_F, NIN, 0);
    const T* ktab = (const T*)P.d_k + (sin_k ? P.ksin_off : 0);
    k_green<T, false, GMODE><<<LG.blocks, LG.threads, LG.smem, st>>>(P.d_inst, P.n_inst, LG.d_pre, spec, tw, ktab,
                                                                      nullptr, nullptr, nullptr);
    if (LO[PASS_MID_I].blocks > 0)
        k_fft_mid<T, true><<<LO[PASS_MID_I].blocks, LO[PASS_MID_I].threads, LO[PASS_MID_I].smem, st>>>(
            P.d_inst, P.n_inst, LO[PASS_MID_I].d_pre, spec, tw, PASS_MID_I, NOUT, 0);
    k_c2r_rows<T, false><<<LO[PASS_C2R].blocks, LO[PASS_C2R].threads, LO[PASS_C2R].smem, st>>>(
        P.d_inst, P.n_inst, LO[PASS_C2R].d_pre, spec, (T*)out, tw, nullptr, NOUT == 9 ? RD_FIELD9 : RD_FIELD3, NOUT,
        (const T*)beta, EPI, nullptr);
    return cudaGetLastError();
}

template <typename T>
static cudaError_t run_observable_t(const PlanCore& P, int kind, const void* beta, void* out, cudaStream_t st,
                                    bool sin_k) {
    switch (kind) {
        case CDD_OBS_BETA_ELASTIC: return run_observable<T, 3>(P, beta, out, st, sin_k);
        case CDD_OBS_ROTATION: return run_observable<T, 4>(P, beta, out, st, sin_k);
        case CDD_OBS_RODRIGUES: return run_observable<T, 5>(P, beta, out, st, sin_k);
        case CDD_OBS_RHO: return run_observable<T, 6>(P, beta, out, st, sin_k);
        case CDD_OBS_RODRIGUES_RHO: return run_observable<T, 8>(P, beta, out, st, sin_k);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_observable(const PlanCore& P, int kind, const void* beta, void* out, cudaStream_t st,
                              bool sin_k) {
    if (P.precision == CDD_F32) return run_observable_t<float>(P, kind, beta, out, st, sin_k);
    return run_observable_t<double>(P, kind, beta, out, st, sin_k);
}

cudaError_t launch_stress(const PlanCore& P, const void* beta, void* sigma, cudaStream_t st, void* phi) {
    if (P.precision == CDD_F32) return run_stress<float>(P, beta, sigma, phi, st);
    return run_stress<double>(P, beta, sigma, phi, st);
}

cudaError_t launch_stress_f0(const PlanCore& P, const void* u, void* rhs_f0, void* sigma, cudaStream_t st,
                             void* phi) {
    if (P.precision == CDD_F32) return run_stress<float>(P, rhs_f0, sigma, phi, st, u);
    return run_stress<double>(P, rhs_f0, sigma, phi, st, u);
}

template <typename T>
static cudaError_t set_attr_t(size_t smem) {
    cudaError_t e;
    if constexpr (std::is_same<T, float>::value) {
        if ((e = set_dyn_smem_limit(k_plane_fwd<T, false>, smem))) return e;
        if ((e = set_dyn_smem_limit(k_plane_fwd<T, true>, smem))) return e;
        if ((e = set_dyn_smem_limit(k_plane_inv<T>, smem))) return e;
    }
    if ((e = set_dyn_smem_limit(k_r2c_rows<T, true>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_r2c_rows<T, false>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_c2r_rows<T, true>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_c2r_rows<T, false>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_fft_mid<T, true>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_fft_mid<T, false>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_green<T, true, 0>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_green<T, false, 0>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_green<T, false, 1>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_green<T, false, 2>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_green<T, false, 3>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_green<T, false, 4>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_green<T, false, 5>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_green<T, false, 6>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_green<T, false, 7>, smem))) return e;
    if ((e = set_dyn_smem_limit(k_green<T, false, 8>, smem))) return e;
    return cudaSuccess;
}

cudaError_t stress_set_attributes(int precision, size_t max_smem) {
    if (precision == CDD_F32) return set_attr_t<float>(max_smem);
    return set_attr_t<double>(max_smem);
}

}  // namespace cdd
