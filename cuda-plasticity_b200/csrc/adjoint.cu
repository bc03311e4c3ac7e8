// Vector-Jacobian product of the central-upwind flux L(beta) = flux(beta, sigma(beta) + load)
// (the forward is stencil.cu): given the cotangent gbar of rhs, produce the cotangent of beta.
//
// Phase A (one thread per cell) recomputes the cell's forward quantities -- the 54 limited
// one-sided derivatives U with the limiter selection of each, the per-axis velocity vectors A,
// |rho|^2 terms P and C, the corner velocities, the directional speeds with the corners that
// attain them, the corner weights and the contractions Q -- and then runs every step backwards,
// producing the cotangents Ubar of the 54 derivatives and sigbar of the total stress at the cell
// (6 symmetric components; its diagonal sums are the applied-load cotangent).
// Phase B gathers beta's cotangent from Ubar: the limiter minmod(a, c) returns a, c or 0, so each
// one-sided derivative is a fixed linear combination of u_{-2} .. u_{+2} once the selection is
// known (2 bits per derivative, recorded in phase A).
// The stress cotangent is mapped back through the transposed Green's function by the host
// (launch_stress_adjoint) and added in phase B.
#include "cdd_internal.cuh"

namespace cdd {

namespace {

struct Nbr {
    long long p1, p2, m1, m2;
};

__device__ __forceinline__ Nbr make_nbr(int i, int n, long long stride) {
    int ip1 = (i + 1 == n) ? 0 : i + 1;
    int ip2 = (ip1 + 1 == n) ? 0 : ip1 + 1;
    int im1 = (i == 0) ? n - 1 : i - 1;
    int im2 = (im1 == 0) ? n - 1 : im1 - 1;
    Nbr r;
    r.p1 = (long long)(ip1 - i) * stride;
    r.p2 = (long long)(ip2 - i) * stride;
    r.m1 = (long long)(im1 - i) * stride;
    r.m2 = (long long)(im2 - i) * stride;
    return r;
}

// Grid coordinates of cell cl of a 3-D (n0, n1, n2) or 2-D (n0, n1) grid; cells < 2^31, so the
// divisions are 32-bit.
__device__ __forceinline__ void cell_coords(long long cl, int nd, int n1, int n2, int& i0, int& i1, int& i2) {
    const unsigned c = (unsigned)cl;
    const unsigned nx = (unsigned)(nd == 3 ? n2 : n1);
    const unsigned r = c / nx;
    i2 = (int)(c - r * nx);
    if (nd == 3) {
        i0 = (int)(r / (unsigned)n1);
        i1 = (int)(r - (unsigned)i0 * (unsigned)n1);
    } else {
        i0 = (int)r;
        i1 = i2;
    }
}

__device__ __forceinline__ float inv_sqrt_a(float x) { return rsqrtf(x); }
__device__ __forceinline__ double inv_sqrt_a(double x) { return 1.0 / sqrt(x); }

// minmod of two values and which one it returned (1: a, 2: c, 0: neither)
template <typename T>
__device__ __forceinline__ T mm_sel(T a, T c, int& sel) {
    const bool same = (a > (T)0 && c > (T)0) || (a < (T)0 && c < (T)0);
    const bool pa = fabs(a) <= fabs(c);
    sel = same ? (pa ? 1 : 2) : 0;
    return same ? (pa ? a : c) : (T)0;
}

// The limiter arguments in the reference's difference order. The FP32 forward stencil forms e0 and
// em2 in a packed form that can differ from these in the last bit, so in an exact tie between two
// limiter arguments the FP32 reverse may take the other branch (the FP32 gradient is checked
// against the FP64 one, whose forward and reverse use the same differences).
template <typename T>
__device__ __forceinline__ void derivs_sel(const T* __restrict__ p, const Nbr& nb, T ih, T& up, T& um,
                                           int& sp, int& sm) {
    const T u0 = p[0], um2 = p[nb.m2], um1 = p[nb.m1], up1 = p[nb.p1], up2 = p[nb.p2];
    const T dm2 = um1 - um2, dm1 = u0 - um1, d0 = up1 - u0, d1 = up2 - up1;
    const T e0 = d1 - d0, em1 = d0 - dm1, em2 = dm1 - dm2;
    const T dd0 = mm_sel(e0, em1, sp);
    const T ddm = mm_sel(em1, em2, sm);
    up = (d0 - (T)0.5 * dd0) * ih;
    um = (dm1 + (T)0.5 * ddm) * ih;
}

template <typename T>
__device__ __forceinline__ double bsum(double v, double* red) {
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

constexpr int VJP_THREADS = 128;
constexpr int VJP_PARTS = 5;     // per-block partials: <sigbar, sigma>, tr tr, diag sigbar (3)

template <typename T, int ND>
__device__ __forceinline__ void vjp_cell(const InstDev& I, long long cl, bool valid, const T* __restrict__ beta,
                                         const T* __restrict__ sig, const T* __restrict__ gbar, double tload,
                                         T* __restrict__ ubar, uint32_t* __restrict__ flags,
                                         T* __restrict__ sigbar, double* lsum) {
    const long long cells = I.cells;
    Nbr nb[ND];
    {
        int i0, i1, i2;
        cell_coords(cl, ND, I.n1, I.n2, i0, i1, i2);
        if (ND == 3) {
            nb[0] = make_nbr(i0, I.n0, (long long)I.n1 * I.n2);
            nb[1] = make_nbr(i1, I.n1, I.n2);
            nb[ND - 1] = make_nbr(i2, I.n2, 1);
        } else {
            nb[0] = make_nbr(i0, I.n0, I.n1);
            nb[ND - 1] = make_nbr(i1, I.n1, 1);
        }
    }
    const T ih = (T)I.inv_h;
    const T* u = beta + I.foff + cl;

    // ---------------- forward recomputation ----------------
    T U[ND][2][9];
    uint32_t fw[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int c = 0; c < 9; ++c)
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            int sp, sm;
            derivs_sel(u + (long long)c * cells, nb[d], ih, U[d][0][c], U[d][1][c], sp, sm);
            const int slot = c * 3 + d;
            fw[slot >> 3] |= (uint32_t)(sp | (sm << 2)) << (4 * (slot & 7));
        }
    double add[3] = {0.0, 0.0, 0.0};
    if (I.has_load) {
        double eps[3];
        for (int i = 0; i < 3; ++i) eps[i] = I.load_init[i] + I.load_rate[i] * (tload - I.load_t0);
        double tr = eps[0] + eps[1] + eps[2];
        for (int i = 0; i < 3; ++i) add[i] = I.load_lamb * tr + 2.0 * I.load_mu * eps[i];
    }
    const T* sp6 = sig + I.soff + cl;
    T S[3][3];
    T s6[6];
    {
#pragma unroll
        for (int c = 0; c < 6; ++c) s6[c] = sp6[c * cells];
        S[0][0] = (T)((double)s6[0] + add[0]);
        S[1][1] = (T)((double)s6[3] + add[1]);
        S[2][2] = (T)((double)s6[5] + add[2]);
        S[0][1] = S[1][0] = s6[1];
        S[0][2] = S[2][0] = s6[2];
        S[1][2] = S[2][1] = s6[4];
    }
    const bool lam_on = (I.Lambda != 0.0);
    const T Lam = (T)I.Lambda;
    const T str = lam_on ? (S[0][0] + S[1][1] + S[2][2]) / (T)3 * Lam : (T)0;
    T A[ND][2][3], trU[ND][2], P[ND][2];
    constexpr int NP = (ND == 3) ? 3 : 1;
    const int pd[3] = {0, 1, 2}, pe[3] = {1, 2, 0};   // pair p couples axes (pd[p], pe[p])
    T Cp[NP][2][2];
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            T sd = 0, pq = 0, tu = 0;
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                T a = 0;
#pragma unroll
                for (int n = 0; n < 3; ++n) {
                    const T v = U[d][s][3 * l + n];
                    a += v * S[d][n];
                    sd += v * S[l][n];
                    if (l != d) pq += v * v;
                }
                A[d][s][l] = a;
                tu += U[d][s][4 * l];
            }
            A[d][s][d] -= sd;
            trU[d][s] = tu;
            P[d][s] = pq;
            if (lam_on) {
                A[d][s][d] += str * tu;
#pragma unroll
                for (int l = 0; l < 3; ++l) A[d][s][l] -= str * U[d][s][3 * l + d];
            }
        }
#pragma unroll
    for (int p = 0; p < NP; ++p)
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                T acc = 0;
#pragma unroll
                for (int j = 0; j < 3; ++j) acc += U[pd[p]][a][3 * pe[p] + j] * U[pe[p] % ND][b][3 * pd[p] + j];
                Cp[p][a][b] = acc;
            }
    constexpr int NC = 1 << ND;
    T V[NC][3], As[NC][3], rr[NC];
    int sg[NC][3];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        sg[c][0] = (c >> (ND - 1)) & 1;
        sg[c][1] = (c >> (ND - 2)) & 1;
        sg[c][2] = (ND == 3) ? (c & 1) : 0;
        T rho2 = (T)ME;
#pragma unroll
        for (int d = 0; d < ND; ++d) rho2 += P[d][sg[c][d]];
#pragma unroll
        for (int p = 0; p < NP; ++p) rho2 -= (T)2 * Cp[p][sg[c][pd[p]]][sg[c][pe[p] % ND]];
        rr[c] = inv_sqrt_a(rho2);
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            T a = 0;
#pragma unroll
            for (int d = 0; d < ND; ++d) a += A[d][sg[c][d]][l];
            As[c][l] = a;
            V[c][l] = a * rr[c];
        }
    }
    T pp[ND], pm[ND], tot[ND];
    int cmx[ND], cmn[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        T mx = 0, mn = 0;
        cmx[d] = -1;
        cmn[d] = -1;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            if (V[c][d] > mx) { mx = V[c][d]; cmx[d] = c; }
            if (V[c][d] < mn) { mn = V[c][d]; cmn[d] = c; }
        }
        pp[d] = mx;
        pm[d] = -mn;
        tot[d] = pp[d] + pm[d] + (T)ME;
    }
    T w[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        T ww = 1;
#pragma unroll
        for (int d = 0; d < ND; ++d) ww *= (sg[c][d] == 0) ? pm[d] : pp[d];
        w[c] = ww;
    }
    T Q[ND][2][3];
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int l = 0; l < 3; ++l) Q[d][s][l] = 0;
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int l = 0; l < 3; ++l)
#pragma unroll
            for (int d = 0; d < ND; ++d) Q[d][sg[c][d]][l] += w[c] * V[c][l];
    T prod = 1;
#pragma unroll
    for (int d = 0; d < ND; ++d) prod *= tot[d];
    // FP32: a cell without gradients has prod = ME^3, below the FP32 range; there hs = 0, and the
    // smallest normal value keeps every term finite (the forward normalises its weights instead)
    if (sizeof(T) == 4 && !(prod >= (T)1.17549435e-38f)) prod = (T)1.17549435e-38f;
    const T inv_abc = (T)1 / prod;
    T coef[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) coef[d] = pm[d] * pp[d] / tot[d];
    T hs[9];
    T Jp = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T h = 0;
#pragma unroll
            for (int d = 0; d < ND; ++d) h += Q[d][0][d] * U[d][0][3 * i + j] + Q[d][1][d] * U[d][1][3 * i + j];
            if (i < ND) {
#pragma unroll
                for (int s = 0; s < 2; ++s)
#pragma unroll
                    for (int l = 0; l < 3; ++l) h -= Q[i % ND][s][l] * U[i % ND][s][3 * l + j];
            }
            hs[3 * i + j] = h;
        }
    if (lam_on) {
#pragma unroll
        for (int d = 0; d < ND; ++d)
#pragma unroll
            for (int s = 0; s < 2; ++s) Jp += Q[d][s][d] * trU[d][s];
#pragma unroll
        for (int j = 0; j < ND; ++j)
#pragma unroll
            for (int s = 0; s < 2; ++s)
#pragma unroll
                for (int l = 0; l < 3; ++l) Jp -= Q[j][s][l] * U[j][s][3 * l + j];
    }
    const T J = -Lam / (T)3 * Jp;

    // ---------------- reverse ----------------
    T gb[9];
    const T* gp = gbar + I.foff + cl;
#pragma unroll
    for (int c = 0; c < 9; ++c) gb[c] = (valid && gbar) ? gp[c * cells] : (T)0;
    T Ub[ND][2][9];
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int c = 0; c < 9; ++c) Ub[d][s][c] = 0;
    T Qb[ND][2][3], trUb[ND][2], coefb[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        coefb[d] = 0;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            trUb[d][s] = 0;
#pragma unroll
            for (int l = 0; l < 3; ++l) Qb[d][s][l] = 0;
        }
    }
    // rhs_ij = -hs_ij inv_abc + sum_d (U+ - U-)_ij coef_d  [- J inv_abc on the diagonal]
    T inv_abc_b = 0;
    T gdiag = gb[0] + gb[4] + gb[8];
#pragma unroll
    for (int c = 0; c < 9; ++c) inv_abc_b -= gb[c] * hs[c];
    if (lam_on) inv_abc_b -= J * gdiag;
    const T Jpb = lam_on ? (-inv_abc * gdiag) * (-Lam / (T)3) : (T)0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int c = 3 * i + j;
            const T vb = gb[c];
            const T hb = -gb[c] * inv_abc;
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                Ub[d][0][c] += vb * coef[d];
                Ub[d][1][c] -= vb * coef[d];
                coefb[d] += vb * (U[d][0][c] - U[d][1][c]);
                Qb[d][0][d] += hb * U[d][0][c];
                Ub[d][0][c] += hb * Q[d][0][d];
                Qb[d][1][d] += hb * U[d][1][c];
                Ub[d][1][c] += hb * Q[d][1][d];
            }
            if (i < ND) {
#pragma unroll
                for (int s = 0; s < 2; ++s)
#pragma unroll
                    for (int l = 0; l < 3; ++l) {
                        Qb[i % ND][s][l] -= hb * U[i % ND][s][3 * l + j];
                        Ub[i % ND][s][3 * l + j] -= hb * Q[i % ND][s][l];
                    }
            }
        }
    if (lam_on) {
#pragma unroll
        for (int d = 0; d < ND; ++d)
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                Qb[d][s][d] += Jpb * trU[d][s];
                trUb[d][s] += Jpb * Q[d][s][d];
            }
#pragma unroll
        for (int j = 0; j < ND; ++j)
#pragma unroll
            for (int s = 0; s < 2; ++s)
#pragma unroll
                for (int l = 0; l < 3; ++l) {
                    Qb[j][s][l] -= Jpb * U[j][s][3 * l + j];
                    Ub[j][s][3 * l + j] -= Jpb * Q[j][s][l];
                }
    }
    T ppb[ND], pmb[ND], totb[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        pmb[d] = coefb[d] * pp[d] / tot[d];
        ppb[d] = coefb[d] * pm[d] / tot[d];
        totb[d] = -coefb[d] * coef[d] / tot[d] - inv_abc_b * inv_abc / tot[d];
    }
    T Vb[NC][3];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        T wb = 0;
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            T q = 0;
#pragma unroll
            for (int d = 0; d < ND; ++d) q += Qb[d][sg[c][d]][l];
            wb += q * V[c][l];
            Vb[c][l] = q * w[c];
        }
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            T others = 1;
#pragma unroll
            for (int e = 0; e < ND; ++e)
                if (e != d) others *= (sg[c][e] == 0) ? pm[e] : pp[e];
            if (sg[c][d] == 0) pmb[d] += wb * others;
            else ppb[d] += wb * others;
        }
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        ppb[d] += totb[d];
        pmb[d] += totb[d];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            if (c == cmx[d]) Vb[c][d] += ppb[d];
            if (c == cmn[d]) Vb[c][d] -= pmb[d];
        }
    }
    T Ab[ND][2][3], Pb[ND][2], Cpb[NP][2][2];
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            Pb[d][s] = 0;
#pragma unroll
            for (int l = 0; l < 3; ++l) Ab[d][s][l] = 0;
        }
#pragma unroll
    for (int p = 0; p < NP; ++p)
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) Cpb[p][a][b] = 0;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        T rb = 0;
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            rb += Vb[c][l] * As[c][l];
            const T asb = Vb[c][l] * rr[c];
#pragma unroll
            for (int d = 0; d < ND; ++d) Ab[d][sg[c][d]][l] += asb;
        }
        const T rho2b = rb * (T)-0.5 * rr[c] * rr[c] * rr[c];
#pragma unroll
        for (int d = 0; d < ND; ++d) Pb[d][sg[c][d]] += rho2b;
#pragma unroll
        for (int p = 0; p < NP; ++p) Cpb[p][sg[c][pd[p]]][sg[c][pe[p] % ND]] -= (T)2 * rho2b;
    }
    // P, C -> U
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int l = 0; l < 3; ++l)
                if (l != d) {
#pragma unroll
                    for (int j = 0; j < 3; ++j) Ub[d][s][3 * l + j] += (T)2 * U[d][s][3 * l + j] * Pb[d][s];
                }
#pragma unroll
    for (int p = 0; p < NP; ++p)
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const T cb = Cpb[p][a][b];
                    Ub[pd[p]][a][3 * pe[p] + j] += cb * U[pe[p] % ND][b][3 * pd[p] + j];
                    Ub[pe[p] % ND][b][3 * pd[p] + j] += cb * U[pd[p]][a][3 * pe[p] + j];
                }
    // A -> U, S
    T Sb[3][3];
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int n = 0; n < 3; ++n) Sb[m][n] = 0;
    T strb = 0;
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const T sdb = -Ab[d][s][d];
#pragma unroll
            for (int l = 0; l < 3; ++l)
#pragma unroll
                for (int n = 0; n < 3; ++n) {
                    const T v = U[d][s][3 * l + n];
                    Ub[d][s][3 * l + n] += Ab[d][s][l] * S[d][n] + sdb * S[l][n];
                    Sb[d][n] += Ab[d][s][l] * v;
                    Sb[l][n] += sdb * v;
                }
            if (lam_on) {
                strb += Ab[d][s][d] * trU[d][s];
                trUb[d][s] += Ab[d][s][d] * str;
#pragma unroll
                for (int l = 0; l < 3; ++l) {
                    strb -= Ab[d][s][l] * U[d][s][3 * l + d];
                    Ub[d][s][3 * l + d] -= Ab[d][s][l] * str;
                }
            }
#pragma unroll
            for (int j = 0; j < 3; ++j) Ub[d][s][4 * j] += trUb[d][s];
        }
    if (lam_on) {
#pragma unroll
        for (int i = 0; i < 3; ++i) Sb[i][i] += strb * Lam / (T)3;
    }
    if (!valid) return;
    if (sigbar) {
        T* sb = sigbar + I.soff + cl;
        sb[0] = Sb[0][0];
        sb[cells] = Sb[0][1] + Sb[1][0];
        sb[2 * cells] = Sb[0][2] + Sb[2][0];
        sb[3 * cells] = Sb[1][1];
        sb[4 * cells] = Sb[1][2] + Sb[2][1];
        sb[5 * cells] = Sb[2][2];
        // parameter partials: <sigbar, sigma_int> (mu), tr sigbar tr sigma_int (nu through lambda),
        // and the diagonal of sigbar (the applied load)
        const double sb6[6] = {(double)Sb[0][0], (double)(Sb[0][1] + Sb[1][0]), (double)(Sb[0][2] + Sb[2][0]),
                               (double)Sb[1][1], (double)(Sb[1][2] + Sb[2][1]), (double)Sb[2][2]};
        double dot = 0.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) dot += sb6[c] * (double)s6[c];
        lsum[0] += dot;
        lsum[1] += (sb6[0] + sb6[3] + sb6[5]) * ((double)s6[0] + (double)s6[3] + (double)s6[5]);
        lsum[2] += sb6[0];
        lsum[3] += sb6[3];
        lsum[4] += sb6[5];
    }
    if (ubar) {
        T* ub = ubar + 54 * I.coff + cl;
#pragma unroll
        for (int d = 0; d < ND; ++d)
#pragma unroll
            for (int s = 0; s < 2; ++s)
#pragma unroll
                for (int c = 0; c < 9; ++c) ub[(long long)((2 * d + s) * 9 + c) * cells] = Ub[d][s][c];
    }
    // Word 3 holds the selections of slots 24..26 in bits 0..11; bits 12..31 record the corners
    // that attain the directional max / min speeds (index + 1, 0 = the zero entry), base 9.
    {
        uint32_t code = 0u, scale = 1u;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            code += (uint32_t)(cmx[d] + 1) * scale;
            scale *= 9u;
            code += (uint32_t)(cmn[d] + 1) * scale;
            scale *= 9u;
        }
        fw[3] |= code << 12;
    }
    uint32_t* fl = flags + 4 * I.coff + cl;
#pragma unroll
    for (int q = 0; q < 4; ++q) fl[(long long)q * cells] = fw[q];
}

template <typename T>
__global__ void __launch_bounds__(VJP_THREADS) k_vjp_cells(const InstDev* __restrict__ insts, int n_inst,
                                                           const int* __restrict__ pre,
                                                           const T* __restrict__ beta, const T* __restrict__ sig,
                                                           const T* __restrict__ gbar, double t,
                                                           T* __restrict__ ubar, uint32_t* __restrict__ flags,
                                                           T* __restrict__ sigbar, double* __restrict__ bload) {
    __shared__ double red[VJP_THREADS / 32];
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    const long long cell = (long long)(blockIdx.x - pre[ii]) * VJP_THREADS + threadIdx.x;
    const bool valid = cell < I.cells;
    double lsum[VJP_PARTS] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (I.nd == 3)
        vjp_cell<T, 3>(I, valid ? cell : 0, valid, beta, sig, gbar, t, ubar, flags, sigbar, lsum);
    else
        vjp_cell<T, 2>(I, valid ? cell : 0, valid, beta, sig, gbar, t, ubar, flags, sigbar, lsum);
    if (!sigbar) return;
#pragma unroll
    for (int i = 0; i < VJP_PARTS; ++i) {
        double s = bsum<T>(lsum[i], red);
        if (threadIdx.x == 0) bload[VJP_PARTS * blockIdx.x + i] = s;
    }
}

// Coefficient of u_q (q = -2..2) in u+ * h (selection sp) and in u- * h (selection sm).
__device__ __forceinline__ float coef_p(int q, int s) {
    const float a = (s == 1) ? 1.f : 0.f, b = (s == 2) ? 1.f : 0.f;
    switch (q) {
        case -1: return -0.5f * b;
        case 0: return -1.f - 0.5f * a + b;
        case 1: return 1.f + a - 0.5f * b;
        case 2: return -0.5f * a;
        default: return 0.f;
    }
}
__device__ __forceinline__ float coef_m(int q, int s) {
    const float a = (s == 1) ? 1.f : 0.f, b = (s == 2) ? 1.f : 0.f;
    switch (q) {
        case -2: return 0.5f * b;
        case -1: return -1.f + 0.5f * a - b;
        case 0: return 1.f - a + 0.5f * b;
        case 1: return 0.5f * a;
        default: return 0.f;
    }
}

// out = c (L^T g) + a1 x1 + a2 x2 + a3 x3 (absent x terms skipped), L^T g = ih * gather + addend.
template <typename T>
struct Axpy {
    T c;
    const T* x[3];
    T a[3];
};

template <typename T, int ND>
__device__ __forceinline__ void gather_cell(const InstDev& I, long long y, const T* __restrict__ ubar,
                                            const uint32_t* __restrict__ flags, const T* __restrict__ addend,
                                            const Axpy<T>& ax, T* out) {
    const long long cells = I.cells;
    Nbr nb[ND];
    {
        int i0, i1, i2;
        cell_coords(y, ND, I.n1, I.n2, i0, i1, i2);
        if (ND == 3) {
            nb[0] = make_nbr(i0, I.n0, (long long)I.n1 * I.n2);
            nb[1] = make_nbr(i1, I.n1, I.n2);
            nb[ND - 1] = make_nbr(i2, I.n2, 1);
        } else {
            nb[0] = make_nbr(i0, I.n0, I.n1);
            nb[ND - 1] = make_nbr(i1, I.n1, 1);
        }
    }
    const T ih = (T)I.inv_h;
    const T* ub = ubar + 54 * I.coff + y;
    const uint32_t* fl = flags + 4 * I.coff + y;
    // neighbour-major: the four selection words of each of the 5 ND neighbours are read once; a
    // one-sided derivative at distance q = -2 (forward) or q = +2 (backward) does not involve y
    // (coef_p(-2, .) = coef_m(2, .) = 0), so those values are not read
    T acc[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) acc[c] = 0;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        // cell x = y - q holds y at offset q
        const long long off[5] = {nb[d].p2, nb[d].p1, 0, nb[d].m1, nb[d].m2};   // q = -2 .. 2
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const int q = k - 2;
            const long long x = off[k];
            uint32_t fw[4];
#pragma unroll
            for (int w = 0; w < 4; ++w) fw[w] = fl[x + (long long)w * cells];
            const T* up = ub + x + (long long)(2 * d * 9) * cells;
            const T* um = up + 9 * cells;
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                const int slot = c * 3 + d;
                const uint32_t f = (fw[slot >> 3] >> (4 * (slot & 7))) & 15u;
                if (q > -2) acc[c] += up[(long long)c * cells] * (T)coef_p(q, (int)(f & 3u));
                if (q < 2) acc[c] += um[(long long)c * cells] * (T)coef_m(q, (int)(f >> 2));
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        const long long o = I.foff + (long long)c * cells + y;
        T v = acc[c] * ih;
        if (addend) v += addend[o];
        v *= ax.c;
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (ax.x[k]) v += ax.a[k] * ax.x[k][o];
        out[o] = v;
    }
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2) k_vjp_gather(const InstDev* __restrict__ insts, int n_inst,
                                                    const int* __restrict__ pre, const T* __restrict__ ubar,
                                                    const uint32_t* __restrict__ flags,
                                                    const T* __restrict__ addend, const Axpy<T> ax,
                                                    T* out) {   // out may alias an x term (same element)
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    const long long y = (long long)(blockIdx.x - pre[ii]) * blockDim.x + threadIdx.x;
    if (y >= I.cells) return;
    if (I.nd == 3) gather_cell<T, 3>(I, y, ubar, flags, addend, ax, out);
    else gather_cell<T, 2>(I, y, ubar, flags, addend, ax, out);
}

// Per-instance sums of the block partials of the load cotangent, added to the caller's array.
__global__ void __launch_bounds__(256) k_vjp_load_reduce(const int* __restrict__ pre, const double* __restrict__ bload,
                                                         double* __restrict__ out) {
    __shared__ double red[8];
    const int ii = blockIdx.x;
    for (int i = 0; i < 3; ++i) {
        double acc = 0.0;
        for (int b = pre[ii] + threadIdx.x; b < pre[ii + 1]; b += blockDim.x) acc += bload[VJP_PARTS * b + 2 + i];
        acc = bsum<double>(acc, red);
        if (threadIdx.x == 0) out[3 * ii + i] += acc;
    }
}

// Parameter cotangents of one stage, scaled by the stage weight c and added to pbar (CDD_PBAR
// doubles per instance): [0] <sigbar, sigma_int>, [1] tr sigbar . tr sigma_int, [2] the k-space
// sum of the nu derivative per unit dA (from the green-block partials), [3..5] the diagonal of
// sigbar (load), [6..8] the same times (t - load_t0).
__global__ void __launch_bounds__(256) k_param_reduce(const InstDev* __restrict__ insts,
                                                      const int* __restrict__ pre_v, const double* __restrict__ bpart,
                                                      const int* __restrict__ pre_g, const double* __restrict__ gpart,
                                                      double c, double t, double* __restrict__ pbar) {
    __shared__ double red[8];
    const int ii = blockIdx.x;
    double v[VJP_PARTS + 1];
    for (int i = 0; i < VJP_PARTS; ++i) {
        double acc = 0.0;
        for (int b = pre_v[ii] + threadIdx.x; b < pre_v[ii + 1]; b += blockDim.x) acc += bpart[VJP_PARTS * b + i];
        v[i] = bsum<double>(acc, red);
    }
    {
        double acc = 0.0;
        if (gpart)
            for (int b = pre_g[ii] + threadIdx.x; b < pre_g[ii + 1]; b += blockDim.x) acc += gpart[b];
        v[VJP_PARTS] = bsum<double>(acc, red);
    }
    if (threadIdx.x == 0) {
        double* o = pbar + CDD_PBAR * ii;
        const double tl = t - insts[ii].load_t0;
        o[0] += c * v[0];
        o[1] += c * v[1];
        o[2] += c * v[5];
        for (int i = 0; i < 3; ++i) {
            o[3 + i] += c * v[2 + i];
            o[6 + i] += c * tl * v[2 + i];
        }
    }
}

}  // namespace

cudaError_t launch_flux_branches(const PlanCore& P, const void* beta, double t, uint32_t* flags, cudaStream_t st) {
    const LaunchShape& V = P.vjp;
    cudaError_t e;
    if ((e = launch_stress(P, beta, P.d_sigma, st))) return e;
    if (P.precision == CDD_F32)
        k_vjp_cells<float><<<V.blocks, VJP_THREADS, 0, st>>>(P.d_inst, P.n_inst, V.d_pre, (const float*)beta,
                                                            (const float*)P.d_sigma, nullptr, t, nullptr, flags,
                                                            nullptr, P.d_bload);
    else
        k_vjp_cells<double><<<V.blocks, VJP_THREADS, 0, st>>>(P.d_inst, P.n_inst, V.d_pre, (const double*)beta,
                                                             (const double*)P.d_sigma, nullptr, t, nullptr, flags,
                                                             nullptr, P.d_bload);
    return cudaGetLastError();
}

cudaError_t launch_vjp_stage(const PlanCore& P, const void* v, const void* sig_v, const void* phi_v, double t,
                             const void* gbar, double c, const void* const x[3], const double a[3], void* out,
                             double* pbar, cudaStream_t st) {
    const LaunchShape& V = P.vjp;
    const LaunchShape& G = P.obs;
    cudaError_t e;
    const bool f32 = (P.precision == CDD_F32);
    if (f32)
        k_vjp_cells<float><<<V.blocks, VJP_THREADS, 0, st>>>(P.d_inst, P.n_inst, V.d_pre, (const float*)v,
                                                            (const float*)sig_v, (const float*)gbar, t,
                                                            (float*)P.d_ubar, P.d_flags, (float*)P.d_sb6, P.d_bload);
    else
        k_vjp_cells<double><<<V.blocks, VJP_THREADS, 0, st>>>(P.d_inst, P.n_inst, V.d_pre, (const double*)v,
                                                             (const double*)sig_v, (const double*)gbar, t,
                                                             (double*)P.d_ubar, P.d_flags, (double*)P.d_sb6,
                                                             P.d_bload);
    if ((e = cudaGetLastError())) return e;
    if ((e = launch_stress_adjoint(P, P.d_sb6, P.d_adj9, st, pbar ? phi_v : nullptr, pbar ? P.d_gpart : nullptr)))
        return e;
    if (pbar) {
        k_param_reduce<<<P.n_inst, 256, 0, st>>>(P.d_inst, V.d_pre, P.d_bload, P.pass[PASS_GREEN].d_pre,
                                                 phi_v ? P.d_gpart : nullptr, c, t, pbar);
        if ((e = cudaGetLastError())) return e;
    }
    if (f32) {
        Axpy<float> ax{(float)c, {(const float*)x[0], (const float*)x[1], (const float*)x[2]},
                       {(float)a[0], (float)a[1], (float)a[2]}};
        k_vjp_gather<float><<<G.blocks, 256, 0, st>>>(P.d_inst, P.n_inst, G.d_pre, (const float*)P.d_ubar, P.d_flags,
                                                     (const float*)P.d_adj9, ax, (float*)out);
    } else {
        Axpy<double> ax{c, {(const double*)x[0], (const double*)x[1], (const double*)x[2]}, {a[0], a[1], a[2]}};
        k_vjp_gather<double><<<G.blocks, 256, 0, st>>>(P.d_inst, P.n_inst, G.d_pre, (const double*)P.d_ubar,
                                                      P.d_flags, (const double*)P.d_adj9, ax, (double*)out);
    }
    return cudaGetLastError();
}

cudaError_t launch_flux_vjp(const PlanCore& P, const void* beta, double t, const void* gbar, void* sigbar,
                            void* betabar, double* load_bar, cudaStream_t st) {
    const LaunchShape& V = P.vjp;
    const LaunchShape& G = P.obs;
    cudaError_t e;
    if ((e = launch_stress(P, beta, P.d_sigma, st))) return e;
    if (P.precision == CDD_F32) {
        k_vjp_cells<float><<<V.blocks, VJP_THREADS, 0, st>>>(P.d_inst, P.n_inst, V.d_pre, (const float*)beta,
                                                            (const float*)P.d_sigma, (const float*)gbar, t,
                                                            (float*)P.d_ubar, P.d_flags, (float*)sigbar, P.d_bload);
    } else {
        k_vjp_cells<double><<<V.blocks, VJP_THREADS, 0, st>>>(P.d_inst, P.n_inst, V.d_pre, (const double*)beta,
                                                             (const double*)P.d_sigma, (const double*)gbar, t,
                                                             (double*)P.d_ubar, P.d_flags, (double*)sigbar,
                                                             P.d_bload);
    }
    if ((e = cudaGetLastError())) return e;
    if (load_bar) k_vjp_load_reduce<<<P.n_inst, 256, 0, st>>>(V.d_pre, P.d_bload, load_bar);
    if ((e = launch_stress_adjoint(P, sigbar, P.d_adj9, st))) return e;
    if (P.precision == CDD_F32) {
        const Axpy<float> ax{1.f, {nullptr, nullptr, nullptr}, {0.f, 0.f, 0.f}};
        k_vjp_gather<float><<<G.blocks, 256, 0, st>>>(P.d_inst, P.n_inst, G.d_pre, (const float*)P.d_ubar, P.d_flags,
                                                     (const float*)P.d_adj9, ax, (float*)betabar);
    } else {
        const Axpy<double> ax{1.0, {nullptr, nullptr, nullptr}, {0.0, 0.0, 0.0}};
        k_vjp_gather<double><<<G.blocks, 256, 0, st>>>(P.d_inst, P.n_inst, G.d_pre, (const double*)P.d_ubar,
                                                      P.d_flags, (const double*)P.d_adj9, ax, (double*)betabar);
    }
    return cudaGetLastError();
}

}  // namespace cdd
