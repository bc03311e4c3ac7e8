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
#include "cdd_internal.cuh"

namespace cdd {

template <typename T> __device__ __forceinline__ T mm3(T a, T b, T c) {
    // NumericalMethods.MinMod3 (L367-378) for finite inputs: the smallest if all are positive,
    // the largest if none is positive, else 0.
    if (a > (T)0 && b > (T)0 && c > (T)0) return fmin(a, fmin(b, c));
    if (!(a > (T)0) && !(b > (T)0) && !(c > (T)0)) return fmax(a, fmax(b, c));
    return (T)0;
}

struct Nbr {     // offsets of the +-1, +-2 neighbours along one axis (periodic)
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

// u+ and u- of one component along one axis.
template <typename T>
__device__ __forceinline__ void derivs(const T* __restrict__ p, T u0, const Nbr& nb, T ih, T ih2,
                                       T hh, T& up, T& um) {
    T um2 = __ldg(p + nb.m2), um1 = __ldg(p + nb.m1), up1 = __ldg(p + nb.p1), up2 = __ldg(p + nb.p2);
    T dm2 = um1 - um2, dm1 = u0 - um1, d0 = up1 - u0, d1 = up2 - up1;
    T D1_0 = (d1 - d0) * ih2;
    T D2_0 = (d1 - dm1) * ih2 * (T)0.5;
    T D1_m1 = (d0 - dm1) * ih2;
    T D2_m1 = (d0 - dm2) * ih2 * (T)0.5;
    T D1_m2 = (dm1 - dm2) * ih2;
    T dd0 = mm3(D1_0, D2_0, D1_m1);
    T ddm = mm3(D1_m1, D2_m1, D1_m2);
    up = d0 * ih - hh * dd0;
    um = dm1 * ih + hh * ddm;
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

constexpr int ST_THREADS = 128;

template <typename T, int ND, int MODE>
__device__ __forceinline__ void stencil_body(const InstDev& I, int ii, long long cell,
                                             const T* __restrict__ bs, const T* bn, T* out,
                                             const T* __restrict__ sig, T* __restrict__ speed_out,
                                             const InstClock* __restrict__ clk, double t_flux,
                                             double* __restrict__ bmax, double* __restrict__ bsum,
                                             double* red) {
    const bool valid = cell < I.cells;
    const long long cl = valid ? cell : 0;

    // neighbour offsets
    Nbr nb[ND];
    if (ND == 3) {
        int i2 = (int)(cl % I.n2);
        long long r = cl / I.n2;
        int i1 = (int)(r % I.n1);
        int i0 = (int)(r / I.n1);
        nb[0] = make_nbr(i0, I.n0, (long long)I.n1 * I.n2);
        nb[1] = make_nbr(i1, I.n1, I.n2);
        if (ND == 3) nb[ND - 1] = make_nbr(i2, I.n2, 1);
    } else {
        int i1 = (int)(cl % I.n1);
        int i0 = (int)(cl / I.n1);
        nb[0] = make_nbr(i0, I.n0, I.n1);
        nb[ND - 1] = make_nbr(i1, I.n1, 1);
    }
    const T ih = (T)I.inv_h, ih2 = (T)(I.inv_h * I.inv_h), hh = (T)(0.5 * I.h);
    const long long cells = I.cells;
    const T* u = bs + I.foff + cl;

    // total stress at the cell: internal + applied load (FP64), symmetric
    // load time: the step-start time in all three stages (FieldMover.py L62, L123, L133); stage 1
    // runs before the dt kernel advances t, stages 2 and 3 after it (t_stage holds the start).
    const double tload = (MODE == M_FLUX) ? t_flux : ((MODE == M_STAGE1) ? clk[ii].t : clk[ii].t_stage);
    double ld[3];
    applied_load(I, tload, ld);
    const T* sp = sig + I.soff + cl;
    T S[3][3];
    {
        T s6[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) s6[c] = sp[c * cells];
        S[0][0] = (T)((double)s6[0] + ld[0]);
        S[1][1] = (T)((double)s6[3] + ld[1]);
        S[2][2] = (T)((double)s6[5] + ld[2]);
        if (!I.has_load) { S[0][0] = s6[0]; S[1][1] = s6[3]; S[2][2] = s6[5]; }
        S[0][1] = S[1][0] = s6[1];
        S[0][2] = S[2][0] = s6[2];
        S[1][2] = S[2][1] = s6[4];
    }
    const bool lam_on = (I.Lambda != 0.0);
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

#pragma unroll 1
    for (int j = 0; j < 3; ++j) {
        T U[ND][2][3];
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            const T* pc = u + (long long)(3 * l + j) * cells;
            T u0 = __ldg(pc);
#pragma unroll
            for (int d = 0; d < ND; ++d) derivs(pc, u0, nb[d], ih, ih2, hh, U[d][0][l], U[d][1][l]);
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
                if (lam_on) {
                    // trace of u_d (components (j, j)) and the -str (u_d)_{l d} terms
                    T dj = (j == 0) ? U[d][s][0] : ((j == 1) ? U[d][s][1] : U[d][s][2]);
                    trU[d][s] += dj;
                    if (j == d) {
#pragma unroll
                        for (int l = 0; l < 3; ++l) A[d][s][l] -= str * U[d][s][l];
                    }
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
        T inv = (T)1 / sqrt(rho2);
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            T a = A[0][sx][l] + A[1][sy][l];
            if (ND == 3) a += A[2 % ND][sz][l];
            V[c][l] = a * inv;
        }
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
        for (int d = 0; d < ND; ++d) w *= (sg[d] == 0) ? pm[d] : pp[d];
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            T wv = w * V[c][l];
#pragma unroll
            for (int d = 0; d < ND; ++d) Q[d][sg[d]][l] += wv;
        }
    }
    T inv_abc = (T)1 / (ND == 3 ? tot[0] * tot[1] * tot[2 % ND] : tot[0] * tot[1]);
    T coef[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) coef[d] = pm[d] * pp[d] / tot[d];
    T spd = tot[0] + tot[1];
    if (ND == 3) spd += tot[2 % ND];
    if (vsum != vsum) spd = vsum;

    // ---------------- pass 2: rhs ----------------
    T rhs[9];
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
#pragma unroll 1
    for (int j = 0; j < 3; ++j) {
        T U[ND][2][3];
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            const T* pc = u + (long long)(3 * l + j) * cells;
            T u0 = __ldg(pc);
#pragma unroll
            for (int d = 0; d < ND; ++d) derivs(pc, u0, nb[d], ih, ih2, hh, U[d][0][l], U[d][1][l]);
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

    // ---------------- outputs ----------------
    if (MODE == M_FLUX) {
        if (valid) {
            T* o = out + I.foff + cl;
#pragma unroll
            for (int c = 0; c < 9; ++c) o[c * cells] = rhs[c];
            if (speed_out) speed_out[I.coff + cl] = spd;
        }
    } else if (MODE == M_STAGE1) {
        if (valid) {
            T* o = out + I.foff + cl;
#pragma unroll
            for (int c = 0; c < 9; ++c) o[c * cells] = rhs[c];
        }
        double v = (double)spd;
        if (!(v <= 1.0e300)) v = __longlong_as_double(0x7ff0000000000000LL);   // NaN/Inf -> +Inf
        if (!valid) v = 0.0;
        double m = block_reduce_max(v, red);
        // observables of the step-start state: elastic energy of the internal stress, mean b_zz
        double e = 0.0, z = 0.0;
        if (valid) {
            double s0 = (double)sp[0], s1 = (double)sp[cells], s2 = (double)sp[2 * cells];
            double s3 = (double)sp[3 * cells], s4 = (double)sp[4 * cells], s5 = (double)sp[5 * cells];
            double sq = s0 * s0 + s3 * s3 + s5 * s5 + 2.0 * (s1 * s1 + s2 * s2 + s4 * s4);
            double tr = s0 + s3 + s5;
            e = (sq - I.nu / (1.0 + I.nu) * tr * tr) / (4.0 * I.mu);
            z = (double)u[8 * cells];
        }
        double es = block_reduce_sum(e, red);
        double zs = block_reduce_sum(z, red);
        if (threadIdx.x == 0) {
            bmax[blockIdx.x] = m;
            bsum[2 * blockIdx.x] = es;
            bsum[2 * blockIdx.x + 1] = zs;
        }
    } else {
        if (valid && clk[ii].active) {
            const T dt = (T)clk[ii].dt;
            const T* un = bn + I.foff + cl;
            T* o = out + I.foff + cl;
            T vn[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) vn[c] = un[c * cells];
            const T* us = bs + I.foff + cl;
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                T vs = us[c * cells];
                T L = dt * rhs[c];
                T r;
                if (MODE == M_STAGE2) r = (T)0.75 * vn[c] + (T)0.25 * vs + (T)0.25 * L;
                else r = (T)(1.0 / 3.0) * vn[c] + (T)(2.0 / 3.0) * vs + (T)(2.0 / 3.0) * L;
                o[c * cells] = r;
            }
        }
    }
}

template <typename T, int MODE>
__global__ void __launch_bounds__(ST_THREADS)
k_stencil(const InstDev* __restrict__ insts, int n_inst, const int* __restrict__ pre,
          const T* __restrict__ bs, const T* bn, T* out, const T* __restrict__ sig,
          T* __restrict__ speed_out, const InstClock* __restrict__ clk, double t_flux,
          double* __restrict__ bmax, double* __restrict__ bsum) {
    __shared__ double red[ST_THREADS / 32];
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    const long long cell = (long long)(blockIdx.x - pre[ii]) * ST_THREADS + threadIdx.x;
    if (I.nd == 3)
        stencil_body<T, 3, MODE>(I, ii, cell, bs, bn, out, sig, speed_out, clk, t_flux, bmax, bsum, red);
    else
        stencil_body<T, 2, MODE>(I, ii, cell, bs, bn, out, sig, speed_out, clk, t_flux, bmax, bsum, red);
}

// ------------------------------------------------------------------------------------------
// Per-instance time step: dt = cfl / (max(shape) * max speed), clamped to t_end
// (FieldMover.py L94-111). Non-finite maxima raise ST_NONFINITE and skip the step.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_dt(const InstDev* __restrict__ insts,
                                           const int* __restrict__ pre,
                                           const double* __restrict__ bmax,
                                           const double* __restrict__ bsum,
                                           InstClock* __restrict__ clk, double* __restrict__ obs,
                                           int* __restrict__ status, int fixed, double dt_fixed) {
    __shared__ double red[8];
    const int ii = blockIdx.x;
    const InstDev& I = insts[ii];
    const int b0 = pre[ii], b1 = pre[ii + 1];
    double m = 0.0, es = 0.0, zs = 0.0;
    for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x) {
        m = fmax(m, bmax[b]);
    }
    m = block_reduce_max(m, red);
    // observable sums in a fixed order (thread 0 walks the partials)
    if (threadIdx.x == 0) {
        for (int b = b0; b < b1; ++b) { es += bsum[2 * b]; zs += bsum[2 * b + 1]; }
        obs[2 * ii] = es;
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
        if (act && c.t + dt > c.t_end) dt = c.t_end - c.t;
        if (!act) dt = 0.0;
        c.dt = dt;
        c.active = act ? 1 : 0;
        if (act) { c.t = c.t + dt; c.steps += 1; }
        clk[ii] = c;
    }
}

// F0 = u + dt * rhs, in place on the rhs buffer, for active instances.
template <typename T>
__global__ void __launch_bounds__(256) k_axpy_f0(const InstDev* __restrict__ insts, int n_inst,
                                                 const int* __restrict__ pre, const T* __restrict__ u,
                                                 T* __restrict__ f0, const InstClock* __restrict__ clk) {
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    if (!clk[ii].active) return;
    const T dt = (T)clk[ii].dt;
    const long long n = 9 * I.cells;
    const long long i0 = (long long)(blockIdx.x - pre[ii]) * blockDim.x * 4 + threadIdx.x;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        long long i = i0 + (long long)k * blockDim.x;
        if (i < n) f0[I.foff + i] = u[I.foff + i] + dt * f0[I.foff + i];
    }
}

// Energy and mean b_zz partials of a state whose internal stress is in sig (observables).
template <typename T>
__global__ void __launch_bounds__(ST_THREADS) k_observe(const InstDev* __restrict__ insts, int n_inst,
                                                        const int* __restrict__ pre,
                                                        const T* __restrict__ beta,
                                                        const T* __restrict__ sig,
                                                        double* __restrict__ bsum) {
    __shared__ double red[ST_THREADS / 32];
    const int ii = find_instance(pre, n_inst, blockIdx.x);
    const InstDev& I = insts[ii];
    const long long cell = (long long)(blockIdx.x - pre[ii]) * ST_THREADS + threadIdx.x;
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

__global__ void k_obs_reduce(const InstDev* __restrict__ insts, const int* __restrict__ pre,
                             const double* __restrict__ bsum, double* __restrict__ obs) {
    const int ii = blockIdx.x;
    if (threadIdx.x != 0) return;
    double es = 0.0, zs = 0.0;
    for (int b = pre[ii]; b < pre[ii + 1]; ++b) { es += bsum[2 * b]; zs += bsum[2 * b + 1]; }
    obs[2 * ii] = es;
    obs[2 * ii + 1] = zs * insts[ii].inv_cells;
}

// ------------------------------------------------------------------------------------------
template <typename T>
static void stencil_dispatch(const PlanCore& P, int mode, const void* bs, const void* bn, void* out,
                             void* speed, double t, cudaStream_t st) {
    const LaunchShape& L = P.stencil;
    const T* b = (const T*)bs;
    const T* n = (const T*)bn;
    T* o = (T*)out;
    const T* s = (const T*)P.d_sigma;
#define CDD_LAUNCH_ST(M, SP)                                                                   \
    k_stencil<T, M><<<L.blocks, ST_THREADS, 0, st>>>(P.d_inst, P.n_inst, L.d_pre, b, n, o, s, SP, \
                                                     P.d_clock, t, P.d_bmax, P.d_bsum)
    switch (mode) {
        case M_FLUX: CDD_LAUNCH_ST(M_FLUX, (T*)speed); break;
        case M_STAGE1: CDD_LAUNCH_ST(M_STAGE1, nullptr); break;
        case M_STAGE2: CDD_LAUNCH_ST(M_STAGE2, nullptr); break;
        default: CDD_LAUNCH_ST(M_STAGE3, nullptr); break;
    }
#undef CDD_LAUNCH_ST
}

cudaError_t launch_stencil(const PlanCore& P, int mode, const void* bs, const void* bn, void* out,
                           void* speed, double t_flux, cudaStream_t st) {
    if (P.precision == CDD_F32) stencil_dispatch<float>(P, mode, bs, bn, out, speed, t_flux, st);
    else stencil_dispatch<double>(P, mode, bs, bn, out, speed, t_flux, st);
    return cudaGetLastError();
}

cudaError_t launch_dt(const PlanCore& P, int fixed, double dt_fixed, cudaStream_t st) {
    k_dt<<<P.n_inst, 256, 0, st>>>(P.d_inst, P.stencil.d_pre, P.d_bmax, P.d_bsum, P.d_clock, P.d_obs,
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
    const LaunchShape& L = P.stencil;
    if (P.precision == CDD_F32)
        k_observe<float><<<L.blocks, ST_THREADS, 0, st>>>(P.d_inst, P.n_inst, L.d_pre, (const float*)beta,
                                                         (const float*)P.d_sigma, P.d_bsum);
    else
        k_observe<double><<<L.blocks, ST_THREADS, 0, st>>>(P.d_inst, P.n_inst, L.d_pre, (const double*)beta,
                                                          (const double*)P.d_sigma, P.d_bsum);
    k_obs_reduce<<<P.n_inst, 32, 0, st>>>(P.d_inst, L.d_pre, P.d_bsum, P.d_obs);
    return cudaGetLastError();
}

cudaError_t stencil_set_attributes(int) { return cudaSuccess; }

}  // namespace cdd
