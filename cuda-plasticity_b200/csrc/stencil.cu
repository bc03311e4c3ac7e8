// Central-upwind Hamilton-Jacobi flux of the plastic distortion and the TVD-RK3 stage update,
// one thread per cell, plus the per-instance CFL time step.
//
// Reference semantics (Plasticity/FieldDynamics/CentralUpwindHJ3D.py L11-34, L99-271 and
// Plasticity/FieldDynamics/CentralUpwindHJBetaPDynamics3D.py L34-221):
//  * limited one-sided derivatives along each axis (FindDerivatives, theta = 1, Dx = 1/shape[-1]):
//      d_i = u_{i+1} - u_i, D1_i = (d_{i+1} - d_i)/h^2, D2_i = (d_{i+1} - d_{i-1})/(2 h^2),
//      dd_i = minmod(D1_i, D2_i, D1_{i-1}),
//      u+ = d_0/h - h dd_0 / 2,  u- = d_{-1}/h + h dd_{-1} / 2;
//  * at each of the 2^nd corners s (a choice of u+ or u- per axis) the dislocation velocity
//      V_l = [sum_n sum_d (u_d)_ln sigma_dn - sum_mn (u_l)_mn sigma_mn (+ Lambda terms)] / |rho|,
//      |rho|^2 = ME + sum_d |u_d|^2 - sum_d sum_j (u_d)_dj^2 - 2 sum_{d<e} sum_j (u_d)_ej (u_e)_dj,
//    and the Hamiltonian H_ij = sum_d V_d (u_d)_ij - sum_l V_l (u_i)_lj (+ Lambda trace term);
//  * directional speeds a+ = max(0, V_x over corners), a- = |min(0, V_x over corners)|, ...,
//    a_tot = a+ + a- + ME; rhs = -sum_s w_s H_s / (a_tot b_tot c_tot)
//    + sum_d (u_d+ - u_d-) a_d- a_d+ / a_d,tot, with w_s the product over axes of a_d- for a '+'
//    choice and a_d+ for a '-' choice; CFL speed = a_tot + b_tot + c_tot.
//
// Evaluation. V is linear in each axis' derivative tensor, so per axis and sign the kernel forms
// the 3-vector A[d][s] once; V at a corner is the sum of three of them over |rho|. |rho|^2 splits
// into per-axis terms P[d][s] and pair terms C_de[s_d][s_e]. The corner-weighted sum of H
// contracts to 6 scalars G[d][s] and 18 scalars Q[i][s][l] (sums of w V over the corners with a
// given sign on one axis). No per-corner H or derivative tensor is formed. The derivatives are
// computed one tensor column (j) at a time, twice: pass 1 accumulates A, P, C; pass 2 forms rhs.
#include <cudaTypedefs.h>

#include "cdd_internal.cuh"

namespace cdd {

// The limiter of FindDerivatives is MinMod3(D1_i, D2_i, D1_{i-1}) (NumericalMethods.py L367-378)
// with D2_i = (D1_i + D1_{i-1}) / 2: the middle argument is the mean of the outer two. It has the
// sign of both when they agree and its magnitude is never below the smaller of theirs (also after
// rounding: fl(a + c) / 2 >= min(a, c) for a, c > 0), so the 3-way minmod equals the 2-way one:
// min(|a|, |c|) with their common sign, 0 when the signs differ or one is zero. That is the median
// of (a, c, 0); FP32 forms it with four min/max operations and no compares or selects:
// max(min(a, c), min(max(a, c), 0)) (both positive: min(a, c); both negative: max(a, c); else 0).
// FP64 keeps the compare-and-select form.
__device__ __forceinline__ float minmod2(float a, float c) {
    return fmaxf(fminf(a, c), fminf(fmaxf(a, c), 0.0f));
}
__device__ __forceinline__ double minmod2(double a, double c) {
    const double m = fmin(fabs(a), fabs(c));
    const bool pos = (a > 0.0) & (c > 0.0);
    const bool neg = (a < 0.0) & (c < 0.0);
    return pos ? m : (neg ? -m : 0.0);
}

// 1/sqrt and division: FP32 uses the hardware approximations (<= 2 ulp), FP64 exact ones.
__device__ __forceinline__ float inv_sqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double inv_sqrt(double x) { return 1.0 / sqrt(x); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }

// Shared-memory tiles of the 2.5-D march: a block owns TXS x TYS cells of a plane (last axis x
// contiguous) and walks along axis 0 (3-D). Each staged plane holds all 9 components of a box of
// RY rows (2-row halo in y) by RX columns starting OX cells left of the tile: RX/OX keep the box's
// x origin on a 16-byte boundary (TMA), i.e. 40/4 for FP32 and 36/2 for FP64.
constexpr int TXS = 32;
template <typename T> struct TileGeom;
template <> struct TileGeom<float> { static constexpr int RX = 40, OX = 4, NS = 6, TY = 8; };
template <> struct TileGeom<double> { static constexpr int RX = 36, OX = 2, NS = 5, TY = 4; };
template <typename T> __host__ __device__ constexpr int tile_ry() { return TileGeom<T>::TY + 4; }
template <typename T> __host__ __device__ constexpr int st_threads() { return TXS * TileGeom<T>::TY; }
template <typename T> __host__ __device__ constexpr int tile_pp() { return tile_ry<T>() * TileGeom<T>::RX; }   // per component

template <typename T, int ND>
struct TileView {
    static constexpr int RX = TileGeom<T>::RX, PP = tile_pp<T>();
    const T* sm;       // shared memory base
    int so[5];         // element offsets of the ring planes z-2 .. z+2 (3-D); so[2] = current plane
    int idx;           // in-plane offset of this thread's cell (halo included)
    __device__ __forceinline__ T center(int c) const { return sm[so[2] + c * PP + idx]; }
    __device__ __forceinline__ void load5(int c, int d, T* v) const {
        if (ND == 3 && d == 0) {
#pragma unroll
            for (int q = 0; q < 5; ++q) v[q] = sm[so[q] + c * PP + idx];
        } else {
            const int st = (d == ND - 1) ? 1 : RX;
            const T* p = sm + so[2] + c * PP + idx;
            v[0] = p[-2 * st]; v[1] = p[-st]; v[2] = p[0]; v[3] = p[st]; v[4] = p[2 * st];
        }
    }
};

// ---- TMA and mbarrier primitives (inline PTX, sm_100a) ----
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after ~2^22 polls (well above any TMA latency) and reports false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (int i = 0; i < (1 << 22); ++i) {
        if (mbar_test(bar, parity)) return true;
        if (i > 64) __nanosleep(64);
    }
    return false;
}
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y,
                                            int z, int c, int n) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(c), "r"(n), "r"(smem_addr(bar))
        : "memory");
}

// One element (4 or 8 bytes) global -> shared without a register round trip; each thread waits for
// its own copies only (cp.async.wait_all), so no block barrier is needed when a thread reads back
// what it copied.
__device__ __forceinline__ void cp_async_elem(float* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_elem(double* dst, const double* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_own() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// Hint: bring the 128-byte line at p into L2 (no register result, no completion to wait for).
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p)); }

// u+ and u- from the five values u_{-2} .. u_{+2} along one axis. The limiter arguments D1, D2
// of FindDerivatives all carry 1/h^2; minmod is positively homogeneous, so the kernel limits the
// undivided second differences and applies 1/h once: u+ = (d_0 - mm/2) / h, u- = (d_-1 + mm_-1/2) / h.
// The two limiters of one axis share their middle argument em1: minmod(a, em1) is the median of
// (a, em1, 0), i.e. a clamped to [min(em1, 0), max(em1, 0)], so FP32 forms those bounds once.
__device__ __forceinline__ void minmod_pair(float e0, float em1, float em2, float& dd0, float& ddm) {
    const float lo = fminf(em1, 0.0f), hi = fmaxf(em1, 0.0f);
    dd0 = fminf(fmaxf(e0, lo), hi);
    ddm = fminf(fmaxf(em2, lo), hi);
}
__device__ __forceinline__ void minmod_pair(double e0, double em1, double em2, double& dd0, double& ddm) {
    dd0 = minmod2(e0, em1);
    ddm = minmod2(em1, em2);
}

template <typename T>
__device__ __forceinline__ void derivs5(const T* v, T ih, T& up, T& um) {
    const T dm2 = v[1] - v[0], dm1 = v[2] - v[1], d0 = v[3] - v[2], d1 = v[4] - v[3];
    const T e0 = d1 - d0, em1 = d0 - dm1, em2 = dm1 - dm2;
    T dd0, ddm;
    minmod_pair(e0, em1, em2, dd0, ddm);
    up = (d0 - (T)0.5 * dd0) * ih;
    um = (dm1 + (T)0.5 * ddm) * ih;
}

// ---- FP32 flux with paired arithmetic ----
// Every quantity of the central-upwind flux that comes in a forward / backward pair (one-sided
// derivatives u+ / u-, the A, S_d, P, trace and Q sums, the final per-axis coefficients) is kept
// as one float2 (x: forward, y: backward) and updated with the packed FP32 instructions
// (__ffma2_rn, __fadd2_rn, __fmul2_rn: two lanes per instruction, each rounded as the scalar
// operation). The corners pair up along the last axis: corners 2m and 2m + 1 differ only in
// its sign. Same formulas as the scalar path; the rhs sums are regrouped per one-sided
// derivative: rhs_ij = sum_d [(c_d - Q+_dd) (u+_d)_ij + (-c_d - Q-_dd) (u-_d)_ij]
//                      + [i < ND] sum_{s,l} Q^s_il (u^s_i)_lj,
// with c_d = a+_d a-_d / tot_d, i.e. -H / (a_tot b_tot c_tot) + the viscous term of the scalar form.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
// The differences in packed form around the centre c = u_0: P = (u_1, u_-1) - (c, c) = (d0, -dm1),
// Q = (u_2, u_-2) - (c, c), and the limiter's outer arguments (e0, em2) = Q - 2 P in one packed
// multiply-add (e0 = d1 - d0 and em2 = dm1 - dm2 up to rounding); the middle one em1 = d0 - dm1 =
// P.x + P.y and the one-sided derivatives (d0 - dd0 / 2, dm1 + ddm / 2) / h are formed as the
// scalar form does.
__device__ __forceinline__ float2 derivs5_f2(const float* v, float ih) {
    const float2 c2 = f2(v[2], v[2]);
    const float2 m1 = f2(-1.0f, -1.0f);
    const float2 P = __ffma2_rn(c2, m1, f2(v[3], v[1]));
    const float2 Q = __ffma2_rn(c2, m1, f2(v[4], v[0]));
    const float2 E = __ffma2_rn(P, f2(-2.0f, -2.0f), Q);
    float dd0, ddm;
    minmod_pair(E.x, P.x + P.y, E.y, dd0, ddm);
    return __fmul2_rn(__ffma2_rn(f2(dd0, ddm), f2(-0.5f, -0.5f), P), f2(ih, -ih));
}
__device__ __forceinline__ float lane(const float2& v, int s) { return s ? v.y : v.x; }
// Maximum / minimum that return NaN when either argument is NaN (fmaxf / fminf drop it).
__device__ __forceinline__ float fmax_nan(float a, float b) {
    float d;
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float fmin_nan(float a, float b) {
    float d;
    asm("min.NaN.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
// The same over three arguments in one instruction (three-input min / max, sm_100).
__device__ __forceinline__ float fmax3_nan(float a, float b, float c) {
    float d;
    asm("max.NaN.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float fmin3_nan(float a, float b, float c) {
    float d;
    asm("min.NaN.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

template <int ND, bool GLIDE>
__device__ __forceinline__ void flux_f32(const TileView<float, ND>& tv, float ih, const float (&S)[3][3],
                                         bool lam_on, bool glide, float Lambda, float (&rhs)[9], float& spd) {
    constexpr int NC = 1 << ND;
    constexpr int NP = (ND == 3) ? 3 : 1;
    const float2 z2 = f2(0.0f, 0.0f);
    float2 U[ND][9];   // (u+_d, u-_d) of component c = 3 l + j (row l, column j)
#pragma unroll
    for (int c = 0; c < 9; ++c)
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            float v5[5];
            tv.load5(c, d, v5);
            U[d][c] = derivs5_f2(v5, ih);
        }
    const float str = lam_on ? (S[0][0] + S[1][1] + S[2][2]) / 3.0f * Lambda : 0.0f;

    // pass 1: A_d l = sum_j (u_d)_lj S_dj, S_d = sum_{l,j} (u_d)_lj S_lj, P_d = sum_{l != d, j} (u_d)_lj^2,
    // tr(u_d), C_de[s_d][s_e] = sum_j (u_d)_ej (u_e)_dj
    float2 A[ND][3], Sd[ND], Pq[ND], trU[ND];
    float Cp[NP][2][2];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        Sd[d] = z2; Pq[d] = z2; trU[d] = z2;
#pragma unroll
        for (int l = 0; l < 3; ++l) A[d][l] = z2;
    }
#pragma unroll
    for (int p = 0; p < NP; ++p)
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) Cp[p][a][b] = 0.0f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            const float2 sdj = f2(S[d][j], S[d][j]);
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                const float2 u = U[d][3 * l + j];
                A[d][l] = __ffma2_rn(u, sdj, A[d][l]);
                Sd[d] = __ffma2_rn(u, f2(S[l][j], S[l][j]), Sd[d]);
                if (l != d) Pq[d] = __ffma2_rn(u, u, Pq[d]);
            }
            if (lam_on || glide) trU[d] = __fadd2_rn(trU[d], U[d][4 * j]);
            if (lam_on && j == d) {
#pragma unroll
                for (int l = 0; l < 3; ++l) A[d][l] = __ffma2_rn(f2(-str, -str), U[d][3 * l + j], A[d][l]);
            }
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                Cp[0][a][b] += lane(U[0][3 + j], a) * lane(U[1 % ND][j], b);
                if (ND == 3) {
                    Cp[1 % NP][a][b] += lane(U[1 % ND][6 + j], a) * lane(U[2 % ND][3 + j], b);
                    Cp[2 % NP][a][b] += lane(U[2 % ND][j], a) * lane(U[0][6 + j], b);
                }
            }
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        A[d][d] = __fadd2_rn(A[d][d], f2(-Sd[d].x, -Sd[d].y));
        if (lam_on) A[d][d] = __ffma2_rn(f2(str, str), trU[d], A[d][d]);
    }

    // corners: V = (A_x[sx] + A_y[sy] (+ A_z[sz])) / |rho|, paired along the last axis
    float2 V[NC / 2][3];
    if constexpr (ND == 3 && !GLIDE) {
        // pair m = 2 sx + sy, lanes sz = 0, 1: the x and y parts of |rho|^2 and of A are common to
        // the pair, the z parts come as pairs
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int sx = m >> 1, sy = m & 1;
            const float cr = (float)ME + lane(Pq[0], sx) + lane(Pq[1 % ND], sy) - 2.0f * Cp[0][sx][sy];
            const float2 cz = f2(Cp[1 % NP][sy][0] + Cp[2 % NP][0][sx], Cp[1 % NP][sy][1] + Cp[2 % NP][1][sx]);
            const float2 r2 = __ffma2_rn(cz, f2(-2.0f, -2.0f), __fadd2_rn(f2(cr, cr), Pq[2 % ND]));
            const float2 inv2 = f2(inv_sqrt(r2.x), inv_sqrt(r2.y));
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                const float ca = lane(A[0][l], sx) + lane(A[1 % ND][l], sy);
                V[m][l] = __fmul2_rn(__fadd2_rn(f2(ca, ca), A[2 % ND][l]), inv2);
            }
        }
    } else {
#pragma unroll
    for (int m = 0; m < NC / 2; ++m) {
        float av[2][3], inv[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int c = 2 * m + h;
            const int sx = (c >> (ND - 1)) & 1, sy = (c >> (ND - 2)) & 1;
            const int sz = (ND == 3) ? (c & 1) : 0;
            float rho2;
            if (ND == 3)
                rho2 = (float)ME + lane(Pq[0], sx) + lane(Pq[1 % ND], sy) + lane(Pq[2 % ND], sz)
                       - 2.0f * (Cp[0][sx][sy] + Cp[1 % NP][sy][sz] + Cp[2 % NP][sz][sx]);
            else
                rho2 = (float)ME + lane(Pq[0], sx) + lane(Pq[1 % ND], sy) - 2.0f * Cp[0][sx][sy];
            inv[h] = inv_sqrt(rho2);
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                float a = lane(A[0][l], sx) + lane(A[1 % ND][l], sy);
                if (ND == 3) a += lane(A[2 % ND][l], sz);
                av[h][l] = a;
            }
            if (GLIDE && glide) {
                // glide-only projection (CentralUpwindHJBetaPGlideOnlyDynamics.py L152-201, 2-D L96-129):
                // g_d = tr(u_d) - sum_e (u_e)_{d e}, v += g (ME + v.g) / (ME + g.g), then v / |rho|
                const int sgc[3] = {sx, sy, sz};
                float gv[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    float Dd = 0.0f;
#pragma unroll
                    for (int e = 0; e < ND; ++e) Dd += lane(U[e][3 * d + e], sgc[e]);
                    const float tr = (d < ND) ? lane(trU[d % ND], sgc[d]) : 0.0f;
                    gv[d] = tr - Dd;
                }
                const float rr = (float)ME + gv[0] * gv[0] + gv[1] * gv[1] + gv[2] * gv[2];
                const float rv = (float)ME + av[h][0] * gv[0] + av[h][1] * gv[1] + av[h][2] * gv[2];
                const float f = fdiv(rv, rr);
#pragma unroll
                for (int l = 0; l < 3; ++l) av[h][l] += gv[l] * f;
            }
        }
#pragma unroll
        for (int l = 0; l < 3; ++l) V[m][l] = __fmul2_rn(f2(av[0][l], av[1][l]), f2(inv[0], inv[1]));
    }
    }
    // one-sided speeds a+_d = max(0, max V_d), a-_d = -min(0, min V_d); weights normalised by
    // tot_d = a+_d + a-_d + ME first (the product of the three totals can underflow FP32). The
    // maxima and minima propagate NaN, so that a NaN anywhere in V reaches the CFL speed.
    float pp[ND], pm[ND], wm[ND], wp[ND];
    spd = 0.0f;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        float mx = 0.0f, mn = 0.0f;
        if constexpr (ND == 3) {
            // the 8 corners and 0 in four three-input operations each way
            mx = fmax3_nan(fmax3_nan(V[0][d].x, V[0][d].y, V[1][d].x), fmax3_nan(V[1][d].y, V[2][d].x, V[2][d].y),
                           fmax3_nan(V[3][d].x, V[3][d].y, 0.0f));
            mn = fmin3_nan(fmin3_nan(V[0][d].x, V[0][d].y, V[1][d].x), fmin3_nan(V[1][d].y, V[2][d].x, V[2][d].y),
                           fmin3_nan(V[3][d].x, V[3][d].y, 0.0f));
        } else {
#pragma unroll
            for (int m = 0; m < NC / 2; ++m) {
                mx = fmax_nan(mx, fmax_nan(V[m][d].x, V[m][d].y));
                mn = fmin_nan(mn, fmin_nan(V[m][d].x, V[m][d].y));
            }
        }
        pp[d] = mx;
        pm[d] = -mn;
        const float tot = pp[d] + pm[d] + (float)ME;
        spd += tot;
        const float it = fdiv(1.0f, tot);
        wm[d] = pm[d] * it;
        wp[d] = pp[d] * it;
    }

    // Q^s_dl = sum over corners with s_d = s of w_c V_cl (w_c: product of the weights a-_d / tot_d
    // or a+_d / tot_d of the corner's signs)
    float2 Q[ND][3];
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int l = 0; l < 3; ++l) Q[d][l] = z2;
    if constexpr (ND == 3) {
        // pair m = 2 sx + sy; T_m = w V over its two corners (lanes: sz). Q_z = sum_m T_m lane-wise,
        // Q_x = lane sums of (T_0 + T_1, T_2 + T_3), Q_y = lane sums of (T_0 + T_2, T_1 + T_3)
        float2 w2[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const float wb = ((m >> 1) ? wp[0] : wm[0]) * ((m & 1) ? wp[1] : wm[1]);
            w2[m] = f2(wb * wm[2], wb * wp[2]);
        }
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            float2 T4[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) T4[m] = __fmul2_rn(w2[m], V[m][l]);
            const float2 a01 = __fadd2_rn(T4[0], T4[1]), a23 = __fadd2_rn(T4[2], T4[3]);
            const float2 b02 = __fadd2_rn(T4[0], T4[2]), b13 = __fadd2_rn(T4[1], T4[3]);
            Q[0][l] = f2(a01.x + a01.y, a23.x + a23.y);
            Q[1 % ND][l] = f2(b02.x + b02.y, b13.x + b13.y);
            Q[2 % ND][l] = __fadd2_rn(a01, a23);
        }
    } else {
#pragma unroll
        for (int m = 0; m < NC / 2; ++m) {
            const int c = 2 * m;
            int sg[2];
            sg[0] = (c >> (ND - 1)) & 1;
            sg[1] = (ND == 3) ? ((c >> 1) & 1) : 0;
            float wb = 1.0f;
#pragma unroll
            for (int d = 0; d < ND - 1; ++d) wb *= (sg[d] == 0) ? wm[d] : wp[d];
            const float2 w2 = f2(wb * wm[ND - 1], wb * wp[ND - 1]);
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                const float2 wv = __fmul2_rn(w2, V[m][l]);
                const float sum = wv.x + wv.y;
#pragma unroll
                for (int d = 0; d < ND - 1; ++d) {
                    if (sg[d] == 0) Q[d][l].x += sum;
                    else Q[d][l].y += sum;
                }
                Q[ND - 1][l] = __fadd2_rn(Q[ND - 1][l], wv);
            }
        }
    }

    // pass 2: rhs
    float2 G[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        const float coef = pm[d] * wp[d];
        const float2 qdd = (d == 0) ? Q[d][0] : ((d == 1) ? Q[d][1] : Q[d][2]);
        G[d] = f2(coef - qdd.x, -coef - qdd.y);
    }
    float2 Jp2 = z2;   // Lambda trace term, J = -Lambda/3 (Jp2.x + Jp2.y)
    if (lam_on) {
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            const float2 qdd = (d == 0) ? Q[d][0] : ((d == 1) ? Q[d][1] : Q[d][2]);
            Jp2 = __ffma2_rn(qdd, trU[d], Jp2);
        }
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            float2 acc = __fmul2_rn(G[0], U[0][3 * i + j]);
#pragma unroll
            for (int d = 1; d < ND; ++d) acc = __ffma2_rn(G[d], U[d][3 * i + j], acc);
            if (i < ND) {
#pragma unroll
                for (int l = 0; l < 3; ++l) acc = __ffma2_rn(Q[i % ND][l], U[i % ND][3 * l + j], acc);
            }
            rhs[3 * i + j] = acc.x + acc.y;
        }
        if (lam_on && j < ND) {
#pragma unroll
            for (int l = 0; l < 3; ++l)
                Jp2 = __ffma2_rn(f2(-Q[j % ND][l].x, -Q[j % ND][l].y), U[j % ND][3 * l + j], Jp2);
        }
    }
    if (lam_on) {
        // the trace term enters H_ii, so rhs_ii gets -J / (a_tot b_tot c_tot) (weights normalised)
        const float J = -Lambda / 3.0f * (Jp2.x + Jp2.y);
        rhs[0] -= J;
        rhs[4] -= J;
        rhs[8] -= J;
    }
}

template <typename T>
__device__ __forceinline__ T block_reduce_max(T v, T* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    T r = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, red[w]);
    return r;
}

__device__ __forceinline__ double block_reduce_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double r = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r += red[w];
    return r;
}

__device__ __forceinline__ void applied_load(const InstDev& I, double t, double* add) {
    if (!I.has_load) { add[0] = add[1] = add[2] = 0.0; return; }
    double eps[3];
    for (int i = 0; i < 3; ++i) eps[i] = I.load_init[i] + I.load_rate[i] * (t - I.load_t0);
    double tr = eps[0] + eps[1] + eps[2];
    for (int i = 0; i < 3; ++i) add[i] = I.load_lamb * tr + 2.0 * I.load_mu * eps[i];
}

// Per block constants of one stage: the applied-load stress (FP64) and, for the stage updates,
// dt and whether the instance is still active.
struct StageConst {
    double ld[3];
    double dt;
    double cnu;   // nu / (1 + nu) of the elastic energy density (|sigma|^2 - cnu tr^2) / (4 mu)
    float cnu_f;  // the same rounded to FP32 (the FP32 form's per-cell density)
    bool active;
};

template <int MODE>
__device__ __forceinline__ StageConst stage_const(const InstDev& I, const InstClock& ck, double t_flux) {
    StageConst k;
    // load time: the step-start time in all three stages (FieldMover.py L62, L123, L133); stage 1
    // runs before the dt kernel advances t, stages 2 and 3 after it (t_stage holds the start).
    const double tload = (MODE == M_FLUX) ? t_flux : ((MODE == M_STAGE1) ? ck.t : ck.t_stage);
    applied_load(I, tload, k.ld);
    k.dt = ck.dt;
    k.cnu = I.nu / (1.0 + I.nu);
    k.cnu_f = (float)k.cnu;
    k.active = ck.active != 0;
    return k;
}

// Per-thread pointers to the current cell (component 0; components are `cells` apart) and the
// instance scalars the cell update needs, formed once per block before the march: the march only
// advances the pointers by one plane, and nothing per cell re-reads the instance table (global
// stores through `out` would otherwise force those reloads).
template <typename T> struct CellCtx {
    const T* sig;   // internal stress (6 components)
    const T* bn;    // beta_n of the stage updates
    T* out;         // rhs (flux, stage 1) or the updated state (stages 2, 3)
    T* spd;         // CFL speed (flux mode, optional)
    long long cells;
    T ih;           // 1 / Dx
    bool has_load, lam_on, glide;
};

// Stage-1 observables of a thread's cells: the CFL speed maximum (NaN and Inf map to +Inf) and
// the FP64 sums of the elastic energy density and of b_zz. FP64 keeps all three in registers.
// FP32 (its 256-thread tiles run at most 128 registers per thread) keeps the maximum as a float (a
// maximum of floats is exact) and the two FP64 sums in this thread's two shared-memory slots
// (`acc`, `acc + ST_THREADS`), so that nothing of them stays in registers across the march.
template <typename T> struct Stage1Acc {
    double vmax = 0.0, esum = 0.0, zsum = 0.0;
    __device__ __forceinline__ void start(double*, int) {}
    __device__ __forceinline__ void speed(T s) {
        double v = (double)s;
        if (!(v <= 1.0e300)) v = __longlong_as_double(0x7ff0000000000000LL);   // NaN/Inf -> +Inf
        vmax = fmax(vmax, v);
    }
    __device__ __forceinline__ void energy(double e, double*, int) { esum += e; }
    __device__ __forceinline__ void bzz(double z, double*, int) { zsum += z; }
    __device__ __forceinline__ double max_speed() const { return vmax; }
    __device__ __forceinline__ double energy_sum(const double*) const { return esum; }
    __device__ __forceinline__ double bzz_sum(const double*, int) const { return zsum; }
};
template <> struct Stage1Acc<float> {
    float vmax = 0.0f;
    __device__ __forceinline__ void start(double* acc, int nt) { acc[0] = 0.0; acc[nt] = 0.0; }
    __device__ __forceinline__ void speed(float s) {
        if (!(s <= 3.402823466e38f)) s = __int_as_float(0x7f800000);   // NaN/Inf -> +Inf
        vmax = fmaxf(vmax, s);
    }
    __device__ __forceinline__ void energy(double e, double* acc, int) { acc[0] += e; }
    __device__ __forceinline__ void bzz(double z, double* acc, int nt) { acc[nt] += z; }
    __device__ __forceinline__ double max_speed() const { return (double)vmax; }
    __device__ __forceinline__ double energy_sum(const double* acc) const { return acc[0]; }
    __device__ __forceinline__ double bzz_sum(const double* acc, int nt) const { return acc[nt]; }
};

// ssm: this thread's 6 shared-memory stress slots (component c at ssm[c * ST_THREADS]), filled by
// asynchronous copies issued one cell earlier; sig_next: the stress of the thread's cell in the
// next plane (its copies are issued as soon as this cell's values are read), or null; acc: this
// thread's FP64 sum slots (FP32 stage 1).
template <typename T, int ND, int MODE, int VAR>
__device__ __forceinline__ void stencil_cell(const InstDev& I, const CellCtx<T>& cx, bool valid,
                                             const TileView<T, ND>& tv,
                                             const StageConst& kc_block, const InstClock& ck, double t_flux,
                                             Stage1Acc<T>& sums, double* acc,
                                             const T* __restrict__ sig0, const T* __restrict__ vac,
                                             T* ssm, const T* sig_next) {
    // compile-time variant: bit 0 carries the glide-only projection, bit 1 the vacancy term
    constexpr bool GLIDE = (VAR & 1) != 0;
    constexpr bool VAC = (VAR & 2) != 0;
    const T ih = cx.ih;
    const long long cells = cx.cells;
    // FP32 reads the block's stage constants from shared memory; FP64 (no registers to spare across
    // the march) re-derives them per cell
    StageConst kc_cell;
    if constexpr (sizeof(T) == 8) kc_cell = stage_const<MODE>(I, ck, t_flux);
    const StageConst& kc = (sizeof(T) == 8) ? kc_cell : kc_block;
    // beta_n of the stage update is loaded after the flux (no registers to hold it across; FP32
    // requested its rows into L2 one plane ahead)
    constexpr bool UPD = (MODE == M_STAGE2 || MODE == M_STAGE3);
    const double* ld = kc.ld;
    // total stress at the cell: internal + applied load (FP64), symmetric
    T S[3][3];
    {
        T s6[6];
        cp_async_wait_own();
#pragma unroll
        for (int c = 0; c < 6; ++c) s6[c] = ssm[c * st_threads<T>()];
        if (sig_next) {
#pragma unroll
            for (int c = 0; c < 6; ++c) cp_async_elem(ssm + c * st_threads<T>(), sig_next + c * cells);
            cp_async_commit();
        }
        if (MODE == M_STAGE1 && valid) {
            // observables of the step-start state: elastic energy of the internal stress (k_dt
            // applies 1 / (4 mu) to the instance sum). FP32 forms the cell's density in FP32 (its
            // stress is FP32; sq >= tr^2 / 3 > cnu tr^2, so nothing cancels) and adds it to the FP64
            // sum; FP64 in FP64.
            if constexpr (sizeof(T) == 4) {
                const float d = fmaf(s6[0], s6[0], fmaf(s6[3], s6[3], s6[5] * s6[5]));
                const float o = fmaf(s6[1], s6[1], fmaf(s6[2], s6[2], s6[4] * s6[4]));
                const float tr = s6[0] + s6[3] + s6[5];
                sums.energy((double)fmaf(-kc.cnu_f, tr * tr, fmaf(2.0f, o, d)), acc, st_threads<T>());
            } else {
                const double s0 = (double)s6[0], s1 = (double)s6[1], s2 = (double)s6[2];
                const double s3 = (double)s6[3], s4 = (double)s6[4], s5 = (double)s6[5];
                const double sq = s0 * s0 + s3 * s3 + s5 * s5 + 2.0 * (s1 * s1 + s2 * s2 + s4 * s4);
                const double tr = s0 + s3 + s5;
                sums.energy(sq - kc.cnu * tr * tr, acc, st_threads<T>());
            }
        }
        S[0][0] = (T)((double)s6[0] + ld[0]);
        S[1][1] = (T)((double)s6[3] + ld[1]);
        S[2][2] = (T)((double)s6[5] + ld[2]);
        if (!cx.has_load) { S[0][0] = s6[0]; S[1][1] = s6[3]; S[2][2] = s6[5]; }
        S[0][1] = S[1][0] = s6[1];
        S[0][2] = S[2][0] = s6[2];
        S[1][2] = S[2][1] = s6[4];
        if (VAC && vac && I.vacancy) {   // BetaP_VacancyDynamics.GetSigma (VacancyDynamics.py L23-29): sigma_ii -= alpha c
            // the cell's concentration, addressed on use from the kernel arguments (the stress
            // pointer's offset is the cell index) so that nothing stays live across the march
            const long long cl = cx.sig - (sig0 + I.soff);
            const T ac = (T)I.vac_alpha * vac[I.foff / 9 + cl];
            S[0][0] -= ac;
            S[1][1] -= ac;
            S[2][2] -= ac;
        }
    }
    T rhs[9];
    T spd;
    if constexpr (sizeof(T) == 4) {
        flux_f32<ND, GLIDE>(tv, ih, S, cx.lam_on, GLIDE && cx.glide, (float)I.Lambda, rhs, spd);
    } else {
        const bool lam_on = cx.lam_on;
        const bool glide = GLIDE && cx.glide;   // glide-only dynamics (Lambda is 0 then)
        const T str = lam_on ? (S[0][0] + S[1][1] + S[2][2]) / (T)3 * (T)I.Lambda : (T)0;

        // ---------------- pass 1: A, P, C, trace ----------------
        T A[ND][2][3], Sd[ND][2], Pq[ND][2], trU[ND][2];
        constexpr int NP = (ND == 3) ? 3 : 1;
        T Cp[NP][2][2];
#pragma unroll
        for (int d = 0; d < ND; ++d)
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                Sd[d][s] = 0; Pq[d][s] = 0; trU[d][s] = 0;
#pragma unroll
                for (int l = 0; l < 3; ++l) A[d][s][l] = 0;
            }
#pragma unroll
        for (int p = 0; p < NP; ++p)
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) Cp[p][a][b] = 0;

        // the 54 one-sided derivatives are recomputed from shared memory in each pass (register
        // budget)
        T Dv[GLIDE ? ND : 1][2][3];   // glide-only: (u_e)_{d e} per axis e and sign
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T U[ND][2][3];
#pragma unroll
            for (int l = 0; l < 3; ++l) {
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    T v5[5];
                    tv.load5(3 * l + j, d, v5);
                    derivs5(v5, ih, U[d][0][l], U[d][1][l]);
                }
            }
            T Sj[3], Sdj[3];
#pragma unroll
            for (int l = 0; l < 3; ++l) { Sj[l] = (j == 0) ? S[l][0] : ((j == 1) ? S[l][1] : S[l][2]); }
#pragma unroll
            for (int d = 0; d < ND; ++d) Sdj[d] = (j == 0) ? S[d][0] : ((j == 1) ? S[d][1] : S[d][2]);
#pragma unroll
            for (int d = 0; d < ND; ++d)
#pragma unroll
                for (int s = 0; s < 2; ++s) {
#pragma unroll
                    for (int l = 0; l < 3; ++l) {
                        T v = U[d][s][l];
                        A[d][s][l] += v * Sdj[d];
                        Sd[d][s] += v * Sj[l];
                        if (l != d) Pq[d][s] += v * v;
                    }
                    if (lam_on || glide) {
                        // trace of u_d (components (j, j))
                        T dj = (j == 0) ? U[d][s][0] : ((j == 1) ? U[d][s][1] : U[d][s][2]);
                        trU[d][s] += dj;
                    }
                    if (lam_on && j == d) {
                        // the -str (u_d)_{l d} terms
#pragma unroll
                        for (int l = 0; l < 3; ++l) A[d][s][l] -= str * U[d][s][l];
                    }
                }
            if constexpr (GLIDE) {
                if (glide && j < ND) {
#pragma unroll
                    for (int s = 0; s < 2; ++s)
#pragma unroll
                        for (int l = 0; l < 3; ++l) Dv[j % ND][s][l] = U[j % ND][s][l];
                }
            }
            // pair terms C_de[s_d][s_e] = sum_j (u_d)_ej (u_e)_dj
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    Cp[0][a][b] += U[0][a][1] * U[1][b][0];
                    if (ND == 3) {
                        Cp[1 % NP][a][b] += U[1 % ND][a][2] * U[2 % ND][b][1];
                        Cp[2 % NP][a][b] += U[2 % ND][a][0] * U[0][b][2];
                    }
                }
        }
#pragma unroll
        for (int d = 0; d < ND; ++d)
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                T ad = (d == 0) ? A[d][s][0] : ((d == 1) ? A[d][s][1] : A[d][s][2]);
                ad -= Sd[d][s];
                if (lam_on) ad += str * trU[d][s];
                if (d == 0) A[d][s][0] = ad; else if (d == 1) A[d][s][1] = ad; else A[d][s][2] = ad;
            }

        // ---------------- corners: V, speeds, weights, Q ----------------
        constexpr int NC = 1 << ND;
        T V[NC][3];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int sx = (c >> (ND - 1)) & 1, sy = (c >> (ND - 2)) & 1;
            const int sz = (ND == 3) ? (c & 1) : 0;
            T rho2;
            if (ND == 3)
                rho2 = (T)ME + Pq[0][sx] + Pq[1][sy] + Pq[2 % ND][sz]
                       - (T)2 * (Cp[0][sx][sy] + Cp[1 % NP][sy][sz] + Cp[2 % NP][sz][sx]);
            else
                rho2 = (T)ME + Pq[0][sx] + Pq[1][sy] - (T)2 * Cp[0][sx][sy];
            T inv = inv_sqrt(rho2);
            T av[3];
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                T a = A[0][sx][l] + A[1][sy][l];
                if (ND == 3) a += A[2 % ND][sz][l];
                av[l] = a;
            }
            if (glide) {
                // glide-only projection (CentralUpwindHJBetaPGlideOnlyDynamics.py L152-201, 2-D L96-129):
                // g_d = tr(u_d) - sum_e (u_e)_{d e}, v += g (ME + v.g) / (ME + g.g), then v / |rho|
                const int sgc[3] = {sx, sy, sz};
                T gv[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    T Dd = (T)0;
#pragma unroll
                    for (int e = 0; e < ND; ++e) {
                        if constexpr (GLIDE) Dd += Dv[e][sgc[e]][d];
                    }
                    const T tr = (d < ND) ? trU[d % ND][sgc[d]] : (T)0;
                    gv[d] = tr - Dd;
                }
                const T rr = (T)ME + gv[0] * gv[0] + gv[1] * gv[1] + gv[2] * gv[2];
                const T rv = (T)ME + av[0] * gv[0] + av[1] * gv[1] + av[2] * gv[2];
                const T f = fdiv(rv, rr);
#pragma unroll
                for (int l = 0; l < 3; ++l) av[l] += gv[l] * f;
            }
#pragma unroll
            for (int l = 0; l < 3; ++l) V[c][l] = av[l] * inv;
        }
        T pp[ND], pm[ND], tot[ND];
        T vsum = 0;   // NaN anywhere in V (fmax/fmin would drop it) must reach the CFL maximum
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            T mx = (T)0, mn = (T)0;
#pragma unroll
            for (int c = 0; c < NC; ++c) { mx = fmax(mx, V[c][d]); mn = fmin(mn, V[c][d]); vsum += V[c][d]; }
            pp[d] = mx;
            pm[d] = -mn;
            tot[d] = pp[d] + pm[d] + (T)ME;
        }
        // the reference's order: the upwind weights a-_d, a+_d are divided by a_tot b_tot c_tot at
        // the end (the FP32 form, flux_f32, normalises each axis first)
        T wm[ND], wp[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            wm[d] = pm[d];
            wp[d] = pp[d];
        }
        T Q[ND][2][3];
#pragma unroll
        for (int d = 0; d < ND; ++d)
#pragma unroll
            for (int s = 0; s < 2; ++s)
#pragma unroll
                for (int l = 0; l < 3; ++l) Q[d][s][l] = 0;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            int sg[3];
            sg[0] = (c >> (ND - 1)) & 1;
            sg[1] = (c >> (ND - 2)) & 1;
            sg[2] = (ND == 3) ? (c & 1) : 0;
            T w = (T)1;
#pragma unroll
            for (int d = 0; d < ND; ++d) w *= (sg[d] == 0) ? wm[d] : wp[d];
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                T wv = w * V[c][l];
#pragma unroll
                for (int d = 0; d < ND; ++d) Q[d][sg[d]][l] += wv;
            }
        }
        const T inv_abc = fdiv((T)1, ND == 3 ? tot[0] * tot[1] * tot[2 % ND] : tot[0] * tot[1]);
        T coef[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) coef[d] = fdiv(pm[d] * pp[d], tot[d]);
        spd = tot[0] + tot[1];
        if (ND == 3) spd += tot[2 % ND];
        if (vsum != vsum) spd = vsum;

        // ---------------- pass 2: rhs ----------------
        T Jp = 0;   // Lambda trace term, J = -Lambda/3 * Jp
        if (lam_on) {
#pragma unroll
            for (int d = 0; d < ND; ++d)
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    T qdd = (d == 0) ? Q[d][s][0] : ((d == 1) ? Q[d][s][1] : Q[d][s][2]);
                    Jp += qdd * trU[d][s];
                }
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T U[ND][2][3];
#pragma unroll
            for (int l = 0; l < 3; ++l) {
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    T v5[5];
                    tv.load5(3 * l + j, d, v5);
                    derivs5(v5, ih, U[d][0][l], U[d][1][l]);
                }
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                T hs = 0, vis = 0;
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    T gp = (d == 0) ? Q[d][0][0] : ((d == 1) ? Q[d][0][1] : Q[d][0][2]);
                    T gm = (d == 0) ? Q[d][1][0] : ((d == 1) ? Q[d][1][1] : Q[d][1][2]);
                    hs += gp * U[d][0][i] + gm * U[d][1][i];
                    vis += (U[d][0][i] - U[d][1][i]) * coef[d];
                }
                if (i < ND) {
#pragma unroll
                    for (int s = 0; s < 2; ++s)
#pragma unroll
                        for (int l = 0; l < 3; ++l) hs -= Q[i % ND][s][l] * U[i % ND][s][l];
                }
                T r = -hs * inv_abc + vis;
                if (j == 0) { if (i == 0) rhs[0] = r; else if (i == 1) rhs[3] = r; else rhs[6] = r; }
                else if (j == 1) { if (i == 0) rhs[1] = r; else if (i == 1) rhs[4] = r; else rhs[7] = r; }
                else { if (i == 0) rhs[2] = r; else if (i == 1) rhs[5] = r; else rhs[8] = r; }
            }
            if (lam_on) {
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    if (d != j) continue;
#pragma unroll
                    for (int s = 0; s < 2; ++s)
#pragma unroll
                        for (int l = 0; l < 3; ++l) Jp -= Q[d][s][l] * U[d][s][l];
                }
            }
        }
        if (lam_on) {
            // the trace term enters H_ii, so rhs_ii gets -J / (a_tot b_tot c_tot)
            T J = -(T)I.Lambda / (T)3 * Jp;
            rhs[0] -= J * inv_abc;
            rhs[4] -= J * inv_abc;
            rhs[8] -= J * inv_abc;
        }
    }

    // ---------------- outputs ----------------
    if (MODE == M_FLUX) {
        if (valid) {
            T* o = cx.out;
#pragma unroll
            for (int c = 0; c < 9; ++c) o[c * cells] = rhs[c];
            if (cx.spd) *cx.spd = spd;
        }
    } else if (MODE == M_STAGE1) {
        if (valid) {
            T* o = cx.out;
#pragma unroll
            for (int c = 0; c < 9; ++c) o[c * cells] = rhs[c];
            sums.speed(spd);
            sums.bzz((double)tv.center(8), acc, st_threads<T>());   // mean b_zz of the step-start state
        }
    } else if constexpr (UPD) {
        if (valid && kc.active) {
            const T dt = (T)kc.dt;
            T* o = cx.out;
            T vn[9];
            const T* un = cx.bn;
#pragma unroll
            for (int c = 0; c < 9; ++c) vn[c] = un[c * cells];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                T vs = tv.center(c);
                T L = dt * rhs[c];
                T r;
                if (MODE == M_STAGE2) r = (T)0.75 * vn[c] + (T)0.25 * vs + (T)0.25 * L;
                else r = (T)(1.0 / 3.0) * vn[c] + (T)(2.0 / 3.0) * vs + (T)(2.0 / 3.0) * L;
                o[c * cells] = r;
            }
        }
    }
}

// The plane box of a stencil tile: RX x RY cells from (x0 - OX, y0 - 2) of the instance's field
// (component c at src + c * cells), wrapped periodically.
template <typename T> struct BoxGeomT {
    const T* src;
    long long cells;
    int x0, y0, nX, nY;
};
template <typename T>
__device__ __forceinline__ void stage_box(T* dst, const BoxGeomT<T>& g, int zp, bool all) {
    constexpr int RX = TileGeom<T>::RX, OX = TileGeom<T>::OX, PP = tile_pp<T>(), ST_THREADS = st_threads<T>();
    const T* sp0 = g.src + (long long)zp * g.nY * g.nX;
    for (int e = threadIdx.x; e < 9 * PP; e += ST_THREADS) {
        const int c = e / PP;
        const int r = e - c * PP;
        const int iy = r / RX, ix = r - iy * RX;
        int yy = g.y0 - 2 + iy, xx = g.x0 - OX + ix;
        if (!all && yy >= 0 && yy < g.nY && xx >= 0 && xx < g.nX) continue;
        while (yy < 0) yy += g.nY;
        while (yy >= g.nY) yy -= g.nY;
        while (xx < 0) xx += g.nX;
        while (xx >= g.nX) xx -= g.nX;
        dst[e] = __ldg(sp0 + c * g.cells + (long long)yy * g.nX + xx);
    }
}
// Patch after a TMA copy: only the box's out-of-grid cells, i.e. its columns outside [xl, xr) (all
// rows) and its rows outside [yl, yr) (the in-grid columns). Tiles with more than 8 such columns or
// 4 such rows (grids narrower than a tile) scan the whole box.
template <typename T>
__device__ __forceinline__ void patch_box_edges(T* dst, const BoxGeomT<T>& g, int zp) {
    constexpr int RX = TileGeom<T>::RX, OX = TileGeom<T>::OX, PP = tile_pp<T>(), RY = tile_ry<T>();
    constexpr int ST_THREADS = st_threads<T>();
    const int x0 = g.x0, y0 = g.y0, nX = g.nX, nY = g.nY, tid = threadIdx.x;
    const int xl = max(0, OX - x0), xr = max(xl, min(RX, nX - x0 + OX));
    const int yl = max(0, 2 - y0), yr = max(yl, min(RY, nY - y0 + 2));
    const int nxo = xl + (RX - xr), nyo = yl + (RY - yr);
    if (nxo > 8 || nyo > 4) { stage_box<T>(dst, g, zp, false); return; }
    const T* sp0 = g.src + (long long)zp * nY * nX;
    auto put = [&](int c, int iy, int ix) {
        int yy = y0 - 2 + iy, xx = x0 - OX + ix;
        if (yy < 0) yy += nY;
        if (yy >= nY) yy -= nY;
        if (xx < 0) xx += nX;
        if (xx >= nX) xx -= nX;
        dst[c * PP + iy * RX + ix] = __ldg(sp0 + c * g.cells + (long long)yy * nX + xx);
    };
    if (nxo > 0) {
        for (int e = tid; e < 9 * RY * 8; e += ST_THREADS) {
            const int c = e / (RY * 8), r = e - c * (RY * 8), iy = r >> 3, j = r & 7;
            if (j < nxo) put(c, iy, j < xl ? j : xr + (j - xl));
        }
    }
    if (nyo > 0) {
        for (int e = tid; e < 9 * 4 * RX; e += ST_THREADS) {
            const int c = e / (4 * RX), r = e - c * (4 * RX), q = r / RX, ix = r - q * RX;
            if (q < nyo && ix >= xl && ix < xr) put(c, q < yl ? q : yr + (q - yl), ix);
        }
    }
}

// Out-of-line copies: FP64 calls these (its march is at the 255-register limit, and keeping the
// rarely run staging code out of it removes most of its spills: 22.3 -> 21.7 ms per 256^3 step);
// FP32 inlines them (out of line measured 3% slower there).
template <typename T> __device__ __noinline__ void stage_box_ool(T* dst, BoxGeomT<T> g, int zp, bool all) {
    stage_box<T>(dst, g, zp, all);
}
template <typename T> __device__ __noinline__ void patch_box_edges_ool(T* dst, BoxGeomT<T> g, int zp) {
    patch_box_edges<T>(dst, g, zp);
}

// One block: a TXS x TYS tile of planes [z0, z0 + zc) (3-D) or of the single plane (2-D).
// The 3-D ring holds planes z-2 .. z+2 of all 9 components of beta_s (NS slots). With TMA
// (I.tma_slot >= 0) one 5-D bulk-tensor copy stages a whole plane box (2-D: the one plane) from
// the tensor map of the instance's run of same-shape instances; coordinates outside the
// grid read zeros, and tiles whose box crosses the periodic boundary patch those cells with
// wrapped loads after the copy lands. FP32 (6 slots) prefetches plane z+3 while computing z;
// FP64 (5 slots) refills the slot of z-2 after computing z. Otherwise threads load the box.
template <typename T, int ND, int MODE, int VAR>
__device__ __forceinline__ void march(const InstDev& I, int ii, int lb, T* sm, double* red, uint64_t* bars,
                                      const StencilMapSet& maps,
                                      const T* __restrict__ bs, const T* bn, T* out,
                                      const T* __restrict__ sig, T* __restrict__ speed_out,
                                      const InstClock* __restrict__ clk, double t_flux,
                                      double* __restrict__ bmax, double* __restrict__ bsum,
                                      int* __restrict__ status, const T* __restrict__ vac) {
    constexpr int RX = TileGeom<T>::RX, OX = TileGeom<T>::OX, PP = tile_pp<T>();
    constexpr int TYS = TileGeom<T>::TY, RY = tile_ry<T>(), ST_THREADS = st_threads<T>();
    constexpr int NS = (ND == 3) ? TileGeom<T>::NS : 1;
    constexpr uint32_t PLANE_BYTES = 9u * PP * sizeof(T);
    const int nZ = (ND == 3) ? I.n0 : 1;
    const int nY = (ND == 3) ? I.n1 : I.n0;
    const int nX = (ND == 3) ? I.n2 : I.n1;
    const int tXn = (nX + TXS - 1) / TXS, tYn = (nY + TYS - 1) / TYS;
    int b = lb;
    const int bx = b % tXn; b /= tXn;
    const int by = b % tYn; b /= tYn;
    const int z0 = b * I.st_zc;
    const int z1 = min(z0 + I.st_zc, nZ);
    const int tid = threadIdx.x, tx = tid % TXS, ty = tid / TXS;
    // the tile's own cells start at (x0n, y0n); a last, partial tile is shifted back inside the
    // grid (it recomputes cells of its neighbour without storing them), so that its box leaves the
    // grid by the halo only (x0 stays a multiple of 4 when nX is: the TMA origin x0 - OX is aligned)
    const int x0n = bx * TXS, y0n = by * TYS;
    const int x0 = (x0n + TXS > nX && nX >= TXS) ? nX - TXS : x0n;
    const int y0 = (y0n + TYS > nY && nY >= TYS) ? nY - TYS : y0n;
    const int x = x0 + tx, y = y0 + ty;
    const bool vxy = (x < nX) && (y < nY);
    const bool own = vxy && x >= x0n && y >= y0n;
    const long long cells = I.cells;
    const long long plane = (long long)nY * nX;
    const T* src = bs + I.foff;
    const bool use_tma = maps.enabled && (I.tma_slot >= 0);
    const bool edge = (x0 - OX < 0) || (x0 - OX + RX > nX) || (y0 - 2 < 0) || (y0 - 2 + RY > nY);

    auto wrapz = [&](int z) { while (z < 0) z += nZ; while (z >= nZ) z -= nZ; return z; };
    // Fill (all = true) or patch the out-of-grid cells (all = false) of the box of plane zp; the
    // patch after a TMA copy visits only the box's out-of-grid cells (edge tiles).
    const BoxGeomT<T> bg{src, cells, x0, y0, nX, nY};
    auto load_box = [&](int slot, int zp, bool all) {
        if constexpr (sizeof(T) == 8) stage_box_ool<T>(sm + slot * 9 * PP, bg, zp, all);
        else stage_box<T>(sm + slot * 9 * PP, bg, zp, all);
    };
    auto patch_box = [&](int slot, int zp) {
        if constexpr (sizeof(T) == 8) patch_box_edges_ool<T>(sm + slot * 9 * PP, bg, zp);
        else patch_box_edges<T>(sm + slot * 9 * PP, bg, zp);
    };
    // plane with relative index pr (= z - (z0 - 2)) lives in slot pr % NS
    auto issue = [&](int pr) {
        const int slot = pr % NS;
        mbar_expect_tx(&bars[slot], PLANE_BYTES);
        tma_load_5d(sm + slot * 9 * PP, &maps.m[I.tma_slot], &bars[slot], x0 - OX, y0 - 2,
                    wrapz(z0 - 2 + pr), 0, I.tma_sub);
    };
    int ok = 1;
    auto arrive = [&](int pr) {   // wait for plane pr and patch it; block-uniform result in ok
        if (!ok) return;
        const int slot = pr % NS;
        bool got = mbar_wait(&bars[slot], (uint32_t)((pr / NS) & 1));
        if (__syncthreads_or(!got)) {
            ok = 0;
            if (tid == 0) atomicOr(status, (int)ST_TIMEOUT);
            return;
        }
        if (edge) patch_box(slot, wrapz(z0 - 2 + pr));
    };

    int issued = -1;   // highest plane index handed to TMA
    if (use_tma) {
        if (tid == 0) {
#pragma unroll 1
            for (int s = 0; s < NS; ++s) mbar_init(&bars[s], 1);
            fence_mbar_init();
        }
        __syncthreads();
        constexpr int NPL = (ND == 3) ? 5 : 1;   // planes z0-2 .. z0+2 (3-D), the plane (2-D)
        if (tid == 0)
            for (int pr = 0; pr < NPL; ++pr) issue(pr);
        issued = NPL - 1;
#pragma unroll 1
        for (int pr = 0; pr < NPL; ++pr) arrive(pr);
    } else if (ND == 3) {
#pragma unroll 1
        for (int q = 0; q < 5; ++q) load_box(q, wrapz(z0 - 2 + q), true);
    } else {
        load_box(0, 0, true);
    }
    __shared__ StageConst kc;   // FP32: read per cell from shared memory (keeps registers free)
    if (sizeof(T) == 4 && tid == 0) kc = stage_const<MODE>(I, clk[ii], t_flux);
    __syncthreads();
    Stage1Acc<T> sums;
    // FP32: this thread's FP64 sum slots after the stress slots
    double* acc = reinterpret_cast<double*>(sm + NS * 9 * PP + 6 * ST_THREADS) + tid;
    if (MODE == M_STAGE1) sums.start(acc, ST_THREADS);
    // this thread's cell in plane z0 (cell (z0, 0, 0) for threads outside the grid: in-bounds
    // loads, no stores)
    CellCtx<T> cx;
    {
        const long long cl0 = vxy ? ((long long)z0 * nY + y) * nX + x : (long long)z0 * plane;
        cx.sig = sig + I.soff + cl0;
        cx.bn = bn ? bn + I.foff + cl0 : nullptr;   // stage updates only
        cx.out = out + I.foff + cl0;
        cx.spd = speed_out ? speed_out + I.coff + cl0 : nullptr;
        cx.cells = cells;
        cx.ih = (T)I.inv_h;
        cx.has_load = I.has_load != 0;
        cx.lam_on = (I.Lambda != 0.0);
        cx.glide = (I.glide != 0);
    }
    TileView<T, ND> tv;
    tv.sm = sm;
    tv.idx = (ty + 2) * RX + tx + OX;
    // the stress of the thread's cell, one plane ahead, in shared memory after the ring
    T* ssm = sm + NS * 9 * PP + tid;
#pragma unroll
    for (int c = 0; c < 6; ++c) cp_async_elem(ssm + c * ST_THREADS, cx.sig + c * cells);
    cp_async_commit();
#pragma unroll 1
    for (int z = z0, k = 0; ok && z < z1; ++z, ++k) {
        const bool more = (z + 1 < z1);
        if (use_tma && NS == 6 && more && tid == 0) {
            fence_proxy_async();
            issue(k + 5);
        }
        if (use_tma && NS == 6 && more) issued = k + 5;
        if (ND == 3) {
            // ring planes z-2 .. z+2 live in slots (k + q) mod NS: FP32 rotates them by one plane
            // per step; FP64 (no registers to spare across the march) recomputes them
            if (NS != 6) {
#pragma unroll
                for (int q = 0; q < 5; ++q) tv.so[q] = ((k + q) % NS) * 9 * PP;
            } else if (k == 0) {
#pragma unroll
                for (int q = 0; q < 5; ++q) tv.so[q] = q * 9 * PP;
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) tv.so[q] = tv.so[q + 1];
                tv.so[4] = (tv.so[3] + 9 * PP == NS * 9 * PP) ? 0 : tv.so[3] + 9 * PP;
            }
        } else {
            tv.so[2] = 0;
        }
        // FP32 stage updates read beta_n of their cell after the flux (no registers to hold it
        // across): its rows of the next plane are requested into L2 now, one 128-byte row of 32
        // cells per thread for the first 9 TYS threads (TMA-staged tiles lie inside the grid)
        if constexpr (sizeof(T) == 4 && (MODE == M_STAGE2 || MODE == M_STAGE3)) {
            if (use_tma && more && tid < 9 * TYS) {
                const int c = tid / TYS, r = tid - c * TYS;
                prefetch_l2(cx.bn + c * cells + plane + (long long)(r - ty) * nX - tx);
            }
        }
        stencil_cell<T, ND, MODE, VAR>(I, cx, own, tv, kc, clk[ii], t_flux, sums, acc, sig, vac, ssm,
                                       more ? cx.sig + plane : nullptr);
        cx.sig += plane;
        if (cx.bn) cx.bn += plane;
        cx.out += plane;
        if (cx.spd) cx.spd += plane;
        if (ND == 3 && more) {
            if (use_tma) {
                if (NS == 5) {
                    __syncthreads();
                    if (tid == 0) {
                        fence_proxy_async();
                        issue(k + 5);
                    }
                    issued = k + 5;
                }
                arrive(k + 5);
            } else {
                __syncthreads();
                load_box((k + 5) % NS, wrapz(z + 3), true);   // plane pr = k + 5 lives in slot pr % NS
            }
            // arrive's block-wide vote already orders this cell's reads before the next copy into
            // the ring; a barrier is left only for plain shared-memory stores (edge patches, thread
            // staging) to become visible
            if (!use_tma || edge) __syncthreads();
        }
    }
    cp_async_wait_own();   // no stress copy in flight past here
    if (!ok) {
        // a copy did not land in time: let every copy this block issued finish (bounded), then leave
        for (int pr = max(0, issued - NS + 1); pr <= issued; ++pr)
            mbar_wait(&bars[pr % NS], (uint32_t)((pr / NS) & 1));
        return;
    }
    if (MODE == M_STAGE1) {
        double m = block_reduce_max(sums.max_speed(), red);
        double es = block_reduce_sum(sums.energy_sum(acc), red);
        double zs = block_reduce_sum(sums.bzz_sum(acc, ST_THREADS), red);
        if (tid == 0) {
            bmax[blockIdx.x] = m;
            bsum[2 * blockIdx.x] = es;
            bsum[2 * blockIdx.x + 1] = zs;
        }
    }
}

template <typename T, int MODE, int VAR>
__global__ void __launch_bounds__(st_threads<T>(), 2)
k_stencil(const InstDev* __restrict__ insts, int n_inst, const int* __restrict__ pre,
          const T* __restrict__ bs, const T* bn, T* out, const T* __restrict__ sig,
          T* __restrict__ speed_out, const InstClock* __restrict__ clk, double t_flux,
          double* __restrict__ bmax, double* __restrict__ bsum, int* __restrict__ status,
          const T* __restrict__ vac, const __grid_constant__ StencilMapSet maps) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    __shared__ double red[st_threads<T>() / 32];
    __shared__ __align__(8) uint64_t bars[6];
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    const int lb = blockIdx.x - pre[ii];
    if (I.nd == 3)
        march<T, 3, MODE, VAR>(I, ii, lb, sm, red, bars, maps, bs, bn, out, sig, speed_out, clk, t_flux, bmax, bsum,
                          status, vac);
    else
        march<T, 2, MODE, VAR>(I, ii, lb, sm, red, bars, maps, bs, bn, out, sig, speed_out, clk, t_flux, bmax, bsum,
                          status, vac);
}

// ------------------------------------------------------------------------------------------
// Per-instance time step: dt = cfl / (max(shape) * max speed), clamped to t_end
// (FieldMover.py L94-111). Non-finite maxima raise ST_NONFINITE and skip the step.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_dt(const InstDev* __restrict__ insts,
                                           const int* __restrict__ pre,
                                           const double* __restrict__ bmax,
                                           const double* __restrict__ bsum,
                                           InstClock* __restrict__ clk, double* __restrict__ obs,
                                           int* __restrict__ status, int fixed, double dt_fixed) {
    __shared__ double red[32];
    const int ii = blockIdx.x;
    const InstDev& I = insts[ii];
    const int b0 = pre[ii], b1 = pre[ii + 1];
    double m = 0.0, es = 0.0, zs = 0.0;
    // one pass over the block partials, unrolled so that several loads are in flight; observable
    // sums: fixed-order strided partial sums, then a fixed tree (deterministic)
#pragma unroll 8
    for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x) {
        m = fmax(m, bmax[b]);
        es += bsum[2 * b];
        zs += bsum[2 * b + 1];
    }
    m = block_reduce_max(m, red);
    es = block_reduce_sum(es, red);
    zs = block_reduce_sum(zs, red);
    if (threadIdx.x == 0) {
        obs[2 * ii] = es / (4.0 * I.mu);
        obs[2 * ii + 1] = zs * I.inv_cells;
        InstClock c = clk[ii];
        c.vmax = m;
        c.t_stage = c.t;
        bool finite = (m <= 1.0e300);
        if (!fixed && !finite) atomicOr(status, (int)ST_NONFINITE);
        bool act = (c.t < c.t_end) && (fixed || finite);
        double dt;
        if (fixed) dt = dt_fixed;
        else dt = act ? I.cfl / (I.nmax * m) : 0.0;
        if (!fixed && I.dt_max > 0.0 && dt > I.dt_max) dt = I.dt_max;   // dtBound (FieldMover.py L359-360)
        if (act && c.t + dt > c.t_end) dt = c.t_end - c.t;
        if (!act) dt = 0.0;
        c.dt = dt;
        c.active = act ? 1 : 0;
        if (act) { c.t = c.t + dt; c.steps += 1; }
        clk[ii] = c;
    }
}

// F0 = u + dt * rhs, in place on the rhs buffer, for active instances (one fused multiply-add per
// value). Instances with the fused plane passes form F0 in their forward pass instead.
template <typename T>
__global__ void __launch_bounds__(256) k_axpy_f0(const InstDev* __restrict__ insts, int n_inst,
                                                 const int* __restrict__ pre, const T* __restrict__ u,
                                                 T* __restrict__ f0, const InstClock* __restrict__ clk) {
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    if (!clk[ii].active || I.plane) return;
    const T dt = (T)clk[ii].dt;
    const long long n = 9 * I.cells;
    const long long b0 = (long long)(blockIdx.x - pre[ii]) * blockDim.x * 4;   // 4 elements per thread
    const T* uu = u + I.foff;
    T* ff = f0 + I.foff;
    if (blockDim.x == 256 && b0 + 1024 <= n && ((((uintptr_t)uu) | ((uintptr_t)ff)) & 15) == 0) {
        // 16-byte vectors: one float4 (FP32) or two double2 (FP64) per thread
        if constexpr (sizeof(T) == 4) {
            const long long i = b0 + 4 * threadIdx.x;
            const float4 a = *reinterpret_cast<const float4*>(uu + i);
            float4 r = *reinterpret_cast<const float4*>(ff + i);
            r.x = __fmaf_rn(dt, r.x, a.x);
            r.y = __fmaf_rn(dt, r.y, a.y);
            r.z = __fmaf_rn(dt, r.z, a.z);
            r.w = __fmaf_rn(dt, r.w, a.w);
            *reinterpret_cast<float4*>(ff + i) = r;
        } else {
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const long long i = b0 + 512 * k + 2 * threadIdx.x;
                const double2 a = *reinterpret_cast<const double2*>(uu + i);
                double2 r = *reinterpret_cast<const double2*>(ff + i);
                r.x = __fma_rn(dt, r.x, a.x);
                r.y = __fma_rn(dt, r.y, a.y);
                *reinterpret_cast<double2*>(ff + i) = r;
            }
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        long long i = b0 + threadIdx.x + (long long)k * blockDim.x;
        if (i < n) ff[i] = fma(dt, ff[i], uu[i]);
    }
}

// Vacancy coupling, one thread per cell of the vacancy instances (OperatorSplittingTVDRK_FieldMover,
// FieldMover.py L339-380): tr(beta^P) at the step start (prevTrBetaP), and after the step
// c += vac_beta (TrBetaP - prevTrBetaP) for the instances whose step was applied; traces summed
// xx + yy, then zz, as the reference does.
template <typename T>
__global__ void __launch_bounds__(256) k_vac_trace(const InstDev* __restrict__ insts, int n_inst,
                                                   const int* __restrict__ pre, const T* __restrict__ beta,
                                                   T* __restrict__ tr) {
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    if (!I.vacancy) return;
    const long long cell = (long long)(blockIdx.x - pre[ii]) * blockDim.x + threadIdx.x;
    if (cell >= I.cells) return;
    const T* b = beta + I.foff + cell;
    tr[I.foff / 9 + cell] = (b[0] + b[4 * I.cells]) + b[8 * I.cells];
}

template <typename T>
__global__ void __launch_bounds__(256) k_vac_update(const InstDev* __restrict__ insts, int n_inst,
                                                    const int* __restrict__ pre, const T* __restrict__ beta,
                                                    const T* __restrict__ tr, T* __restrict__ c,
                                                    const InstClock* __restrict__ clk) {
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    if (!I.vacancy || !clk[ii].active) return;
    const long long cell = (long long)(blockIdx.x - pre[ii]) * blockDim.x + threadIdx.x;
    if (cell >= I.cells) return;
    const T* b = beta + I.foff + cell;
    const T trn = (b[0] + b[4 * I.cells]) + b[8 * I.cells];
    T& cv = c[I.foff / 9 + cell];
    cv = cv + (T)I.vac_beta * (trn - tr[I.foff / 9 + cell]);
}

// Energy and mean b_zz partials of a state whose internal stress is in sig (observables).
template <typename T>
__global__ void __launch_bounds__(256) k_observe(const InstDev* __restrict__ insts, int n_inst,
                                                        const int* __restrict__ pre,
                                                        const T* __restrict__ beta,
                                                        const T* __restrict__ sig,
                                                        double* __restrict__ bsum) {
    __shared__ double red[8];
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    const long long cell = (long long)(blockIdx.x - pre[ii]) * blockDim.x + threadIdx.x;
    double e = 0.0, z = 0.0;
    if (cell < I.cells) {
        const T* sp = sig + I.soff + cell;
        const long long cells = I.cells;
        double s0 = (double)sp[0], s1 = (double)sp[cells], s2 = (double)sp[2 * cells];
        double s3 = (double)sp[3 * cells], s4 = (double)sp[4 * cells], s5 = (double)sp[5 * cells];
        double sq = s0 * s0 + s3 * s3 + s5 * s5 + 2.0 * (s1 * s1 + s2 * s2 + s4 * s4);
        double tr = s0 + s3 + s5;
        e = (sq - I.nu / (1.0 + I.nu) * tr * tr) / (4.0 * I.mu);
        z = (double)beta[I.foff + 8 * cells + cell];
    }
    double es = block_reduce_sum(e, red);
    double zs = block_reduce_sum(z, red);
    if (threadIdx.x == 0) { bsum[2 * blockIdx.x] = es; bsum[2 * blockIdx.x + 1] = zs; }
}

__global__ void __launch_bounds__(256) k_obs_reduce(const InstDev* __restrict__ insts,
                                                    const int* __restrict__ pre,
                                                    const double* __restrict__ bsum,
                                                    double* __restrict__ obs) {
    __shared__ double red[8];
    const int ii = blockIdx.x;
    double es = 0.0, zs = 0.0;
    for (int b = pre[ii] + threadIdx.x; b < pre[ii + 1]; b += blockDim.x) {
        es += bsum[2 * b];
        zs += bsum[2 * b + 1];
    }
    es = block_reduce_sum(es, red);
    zs = block_reduce_sum(zs, red);
    if (threadIdx.x == 0) {
        obs[2 * ii] = es;
        obs[2 * ii + 1] = zs * insts[ii].inv_cells;
    }
}

// ------------------------------------------------------------------------------------------
template <typename T>
static void stencil_dispatch(const PlanCore& P, int mode, const void* bs, const void* bn, void* out,
                             void* speed, double t, const StencilMapSet& maps, cudaStream_t st) {
    const LaunchShape& L = P.stencil;
    const T* b = (const T*)bs;
    const T* n = (const T*)bn;
    T* o = (T*)out;
    const T* s = (const T*)P.d_sigma;
    // the variant carries the glide-only projection (bit 0) and the vacancy term (bit 1) only when
    // the plan has such instances
    const int var = (P.any_glide ? 1 : 0) | (P.any_vac ? 2 : 0);
#define CDD_LAUNCH_V(M, V, SP)                                                                           \
    k_stencil<T, M, V><<<L.blocks, st_threads<T>(), L.smem, st>>>(P.d_inst, P.n_inst, L.d_pre, b, n, o, s, SP,     \
                                                             P.d_clock, t, P.d_bmax, P.d_bsum, P.d_status,    \
                                                             (const T*)P.d_vac, maps)
#define CDD_LAUNCH_ST(M, SP)                                  \
    switch (var) {                                            \
        case 0: CDD_LAUNCH_V(M, 0, SP); break;                \
        case 1: CDD_LAUNCH_V(M, 1, SP); break;                \
        case 2: CDD_LAUNCH_V(M, 2, SP); break;                \
        default: CDD_LAUNCH_V(M, 3, SP); break;               \
    }
    switch (mode) {
        case M_FLUX: CDD_LAUNCH_ST(M_FLUX, (T*)speed); break;
        case M_STAGE1: CDD_LAUNCH_ST(M_STAGE1, nullptr); break;
        case M_STAGE2: CDD_LAUNCH_ST(M_STAGE2, nullptr); break;
        default: CDD_LAUNCH_ST(M_STAGE3, nullptr); break;
    }
#undef CDD_LAUNCH_V
#undef CDD_LAUNCH_ST
}

template <typename T>
static cudaError_t vac_pre_t(const PlanCore& P, const void* beta, cudaStream_t st) {
    const LaunchShape& L = P.obs;
    k_vac_trace<T><<<L.blocks, L.threads, 0, st>>>(P.d_inst, P.n_inst, L.d_pre, (const T*)beta, (T*)P.d_vtr);
    return cudaGetLastError();
}

cudaError_t launch_vacancy_pre(const PlanCore& P, const void* beta, cudaStream_t st) {
    return P.precision == CDD_F32 ? vac_pre_t<float>(P, beta, st) : vac_pre_t<double>(P, beta, st);
}

template <typename T>
static cudaError_t vac_post_t(const PlanCore& P, const void* beta, cudaStream_t st) {
    const LaunchShape& L = P.obs;
    k_vac_update<T><<<L.blocks, L.threads, 0, st>>>(P.d_inst, P.n_inst, L.d_pre, (const T*)beta,
                                                    (const T*)P.d_vtr, (T*)P.d_vac, P.d_clock);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_vacancy_diffusion(P, st);
}

cudaError_t launch_vacancy_post(const PlanCore& P, const void* beta, cudaStream_t st) {
    return P.precision == CDD_F32 ? vac_post_t<float>(P, beta, st) : vac_post_t<double>(P, beta, st);
}

cudaError_t launch_stencil(const PlanCore& P, int mode, const void* bs, const void* bn, void* out,
                           void* speed, double t_flux, const StencilMapSet& maps, cudaStream_t st) {
    if (P.precision == CDD_F32) stencil_dispatch<float>(P, mode, bs, bn, out, speed, t_flux, maps, st);
    else stencil_dispatch<double>(P, mode, bs, bn, out, speed, t_flux, maps, st);
    return cudaGetLastError();
}

bool stencil_tma_eligible(const InstDev& I, int precision) {
    const int RX = precision == CDD_F32 ? TileGeom<float>::RX : TileGeom<double>::RX;
    const int RY = precision == CDD_F32 ? tile_ry<float>() : tile_ry<double>();
    const int nX = (I.nd == 3) ? I.n2 : I.n1, nY = (I.nd == 3) ? I.n1 : I.n0;
    if (nX < RX || nY < RY) return false;
    if (precision == CDD_F32 && nX % 4) return false;   // 16-byte row strides
    if (precision != CDD_F32 && nX % 2) return false;
    return true;
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// 5-D map per run of consecutive same-shape instances: (x = last axis, y, z = axis 0 (3-D), component,
// instance of the run); box = one staged plane of all 9 components of one instance, RX x RY cells;
// out-of-grid coordinates read zeros (patched by the kernel).
bool encode_stencil_maps(const PlanCore& P, const InstDev* insts, const void* base, StencilMapSet& maps) {
    maps.enabled = 0;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || !base) return false;
    const bool f32 = (P.precision == CDD_F32);
    const size_t elt = f32 ? sizeof(float) : sizeof(double);
    const cuuint32_t RX = f32 ? TileGeom<float>::RX : TileGeom<double>::RX;
    const cuuint32_t RY = f32 ? tile_ry<float>() : tile_ry<double>();
    bool any = false;
    for (int i = 0; i < P.n_inst; ++i) {
        const InstDev& I = insts[i];
        if (I.tma_slot < 0 || I.tma_sub != 0) continue;
        int run = 1;
        while (i + run < P.n_inst && insts[i + run].tma_slot == I.tma_slot) ++run;
        const char* addr = (const char*)base + (size_t)I.foff * elt;
        if (((uintptr_t)addr) % 16) return false;
        // 2-D: (x = axis 1, y = axis 0, z of size 1)
        const cuuint64_t nX = (I.nd == 3) ? I.n2 : I.n1, nY = (I.nd == 3) ? I.n1 : I.n0;
        const cuuint64_t nZ = (I.nd == 3) ? I.n0 : 1;
        cuuint64_t dims[5] = {nX, nY, nZ, 9, (cuuint64_t)run};
        cuuint64_t strides[4] = {nX * elt, nX * nY * elt, (cuuint64_t)I.cells * elt, (cuuint64_t)9 * I.cells * elt};
        cuuint32_t box[5] = {RX, (cuuint32_t)RY, 1, 9, 1};
        cuuint32_t estr[5] = {1, 1, 1, 1, 1};
        CUresult r = enc(&maps.m[I.tma_slot], f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                         5, (void*)addr, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return false;
        any = true;
    }
    maps.enabled = any ? 1 : 0;
    return any;
}

// Start every instance's clock at t with no end time (fixed-dt steps at a caller-given time).
__global__ void k_set_clock(InstClock* __restrict__ clk, int n_inst, double t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_inst) {
        clk[i].t = t;
        clk[i].t_end = 1.0e300;
    }
}

cudaError_t launch_set_clock(const PlanCore& P, double t, cudaStream_t st) {
    k_set_clock<<<(P.n_inst + 127) / 128, 128, 0, st>>>(P.d_clock, P.n_inst, t);
    return cudaGetLastError();
}

cudaError_t launch_dt(const PlanCore& P, int fixed, double dt_fixed, cudaStream_t st) {
    k_dt<<<P.n_inst, 1024, 0, st>>>(P.d_inst, P.stencil.d_pre, P.d_bmax, P.d_bsum, P.d_clock, P.d_obs,
                                   P.d_status, fixed, dt_fixed);
    return cudaGetLastError();
}

cudaError_t launch_axpy_f0(const PlanCore& P, const void* u, void* rhs_f0, cudaStream_t st) {
    const LaunchShape& L = P.cellwise;
    if (P.precision == CDD_F32)
        k_axpy_f0<float><<<L.blocks, 256, 0, st>>>(P.d_inst, P.n_inst, L.d_pre, (const float*)u,
                                                   (float*)rhs_f0, P.d_clock);
    else
        k_axpy_f0<double><<<L.blocks, 256, 0, st>>>(P.d_inst, P.n_inst, L.d_pre, (const double*)u,
                                                    (double*)rhs_f0, P.d_clock);
    return cudaGetLastError();
}

cudaError_t launch_observe(const PlanCore& P, const void* beta, cudaStream_t st) {
    const LaunchShape& L = P.obs;
    if (P.precision == CDD_F32)
        k_observe<float><<<L.blocks, 256, 0, st>>>(P.d_inst, P.n_inst, L.d_pre, (const float*)beta,
                                                         (const float*)P.d_sigma, P.d_bsum);
    else
        k_observe<double><<<L.blocks, 256, 0, st>>>(P.d_inst, P.n_inst, L.d_pre, (const double*)beta,
                                                          (const double*)P.d_sigma, P.d_bsum);
    k_obs_reduce<<<P.n_inst, 256, 0, st>>>(P.d_inst, P.obs.d_pre, P.d_bsum, P.d_obs);
    return cudaGetLastError();
}

template <typename T>
static cudaError_t st_attr(size_t smem) {
    cudaError_t e;
#define CDD_ATTR_V(V)                                                                   \
    if ((e = set_dyn_smem_limit(k_stencil<T, M_FLUX, V>, smem))) return e;              \
    if ((e = set_dyn_smem_limit(k_stencil<T, M_STAGE1, V>, smem))) return e;            \
    if ((e = set_dyn_smem_limit(k_stencil<T, M_STAGE2, V>, smem))) return e;            \
    if ((e = set_dyn_smem_limit(k_stencil<T, M_STAGE3, V>, smem))) return e;
    CDD_ATTR_V(0)
    CDD_ATTR_V(1)
    CDD_ATTR_V(2)
    CDD_ATTR_V(3)
#undef CDD_ATTR_V
    return cudaSuccess;
}

cudaError_t stencil_set_attributes(int precision, size_t smem) {
    return precision == CDD_F32 ? st_attr<float>(smem) : st_attr<double>(smem);
}

// The plane ring plus the 6 stress slots of every thread (FP32: and its two FP64 sum slots).
size_t stencil_smem_bytes(int precision, bool any3d) {
    if (precision == CDD_F32)
        return ((size_t)(any3d ? TileGeom<float>::NS : 1) * 9 * tile_pp<float>() + 6 * st_threads<float>()) * sizeof(float) +
               2 * st_threads<float>() * sizeof(double);
    return ((size_t)(any3d ? TileGeom<double>::NS : 1) * 9 * tile_pp<double>() + 6 * st_threads<double>()) * sizeof(double);
}

// Blocks of the stencil: (x, y) tiles times chunks of planes along axis 0. Built-in rule: about
// 227K threads in all (1776 blocks of 128 threads, 888 of 256) but at least 8 planes per block (each
// block first stages a 4-plane halo, so shorter chunks spend most of their time on it); planes > 0
// sets the chunk length.
void stencil_geometry(InstDev& I, int precision, int planes) {
    const int nZ = (I.nd == 3) ? I.n0 : 1;
    const int nY = (I.nd == 3) ? I.n1 : I.n0;
    const int nX = (I.nd == 3) ? I.n2 : I.n1;
    const int TYS = precision == CDD_F32 ? TileGeom<float>::TY : TileGeom<double>::TY;
    const int tiles = ((nX + TXS - 1) / TXS) * ((nY + TYS - 1) / TYS);
    int chunks = 1;
    if (I.nd == 3) {
        const int target = 1776 * 4 / TYS;
        chunks = (target + tiles - 1) / tiles;
        if (chunks > nZ / 8) chunks = nZ / 8;
        if (planes > 0) chunks = (nZ + planes - 1) / planes;
        if (chunks > nZ) chunks = nZ;
        if (chunks < 1) chunks = 1;
    }
    I.st_zc = (nZ + chunks - 1) / chunks;
    chunks = (nZ + I.st_zc - 1) / I.st_zc;
    I.stencil_blocks = tiles * chunks;
}

}  // namespace cdd
