"""Plain-torch FP64 restatement of the CDD step -- TEST INFRASTRUCTURE for gradient checks.

Follows the oracle (oracle/cdd_oracle.py, itself pinned to the reference) with torch operations so
that torch.autograd differentiates it: stress (PlasticityState.py L357-390, L85-127), limited
derivatives (CentralUpwindHJ3D.py L11-34), corner velocities and Hamiltonian
(CentralUpwindHJBetaPDynamics3D.py L45-201), central-upwind flux (CentralUpwindHJ3D.py
L189-271), fixed-dt TVD-RK3 (FieldMover.py L38-58) with the traceless applied strain rate.
mu, nu and the strain rate are tensors so their gradients are available too.
"""
import numpy as np
import torch

import cdd_oracle as O

ME = O.ME


def ci(i, j):
    return 3 * i + j


def k_tensors(shape, device):
    k, kSq, kSqSq, kmask = O.k_tables(shape)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=device)
    return [t(v) for v in k], t(kSq), t(kSqSq), t(kmask)


def stress(beta, mu, nu):
    shape = tuple(beta.shape[1:])
    dims = tuple(range(1, len(shape) + 1))
    Kb = torch.fft.rfftn(beta, dim=dims)
    lamb = 2. * mu * nu / (1. - 2. * nu)
    k, kSq0, kSqSq0, kmask = k_tensors(shape, beta.device)
    kSq = kSq0 + ME
    kSqSq = kSqSq0 + ME
    KbE = []
    for i in range(3):
        for j in range(3):
            acc = 0
            for m in range(3):
                for n in range(3):
                    T = lamb / (lamb + 2. * mu) * k[i] * k[j] / kSq * float(m == n) + \
                        k[i] / kSq * ((k[m] * float(j == n)) + (k[n] * float(j == m))) - \
                        2. * (lamb + mu) / (lamb + 2. * mu) * (k[i] * k[j] * k[m] * k[n]) / kSqSq
                    acc = acc + Kb[ci(m, n)] * T
            KbE.append(acc * kmask)
    betaE = torch.fft.irfftn(torch.stack(KbE), s=shape, dim=dims) - beta
    tr = betaE[0] + betaE[4] + betaE[8]
    return torch.stack([lamb * tr * float(i == j) + mu * (betaE[ci(i, j)] + betaE[ci(j, i)])
                        for i in range(3) for j in range(3)])


def minmod3(a, b, c):
    pos = (a > 0) & (b > 0) & (c > 0)
    nonpos = (a <= 0) & (b <= 0) & (c <= 0)
    mn = torch.minimum(torch.minimum(a, b), c)
    mx = torch.maximum(torch.maximum(a, b), c)
    return torch.where(pos, mn, torch.where(nonpos, mx, torch.zeros_like(a)))


def find_derivatives(f, axis, Dx):
    ax = axis + 1
    r = torch.roll
    diff = r(f, -1, ax) - f
    d21 = (r(diff, -1, ax) - diff) / Dx / Dx
    d22 = (r(diff, -1, ax) - r(diff, 1, ax)) / Dx / Dx * 0.5
    d23 = r(d21, 1, ax)
    dd = minmod3(d21, d22, d23)
    return diff / Dx - 0.5 * Dx * dd, r(diff, 1, ax) / Dx + 0.5 * Dx * r(dd, 1, ax)


def velocity(us, sig, Lambda):
    nd = len(us)
    V = [0., 0., 0.]
    for n in range(3):
        for l in range(3):
            for d in range(nd):
                V[l] = V[l] + us[d][ci(l, n)] * sig[ci(d, n)]
            for d in range(nd):
                V[d] = V[d] - us[d][ci(l, n)] * sig[ci(l, n)]
    if Lambda != 0:
        st = (sig[0] + sig[4] + sig[8]) / 3. * Lambda
        for d in range(nd):
            V[d] = V[d] + st * (us[d][0] + us[d][4] + us[d][8])
        for l in range(3):
            acc = us[0][ci(l, 0)]
            for d in range(1, nd):
                acc = acc + us[d][ci(l, d)]
            V[l] = V[l] - st * acc
    rho2 = ME
    for c in range(9):
        for u in us:
            rho2 = rho2 + u[c] * u[c]
    for j in range(3):
        for d, u in enumerate(us):
            rho2 = rho2 - u[ci(d, j)] * u[ci(d, j)]
        if nd == 2:
            rho2 = rho2 - 2 * us[0][ci(1, j)] * us[1][ci(0, j)]
        else:
            rho2 = rho2 - 2 * us[0][ci(1, j)] * us[1][ci(0, j)] - 2 * us[1][ci(2, j)] * us[2][ci(1, j)] \
                - 2 * us[2][ci(0, j)] * us[0][ci(2, j)]
    rho = torch.sqrt(rho2)
    return [v / rho for v in V]


def hamiltonian(us, V, Lambda):
    nd = len(us)
    H = [sum(us[d][c] * V[d] for d in range(nd)) for c in range(9)]
    for j in range(3):
        for l in range(3):
            for i in range(nd):
                H[ci(i, j)] = H[ci(i, j)] - V[l] * us[i][ci(l, j)]
    if Lambda != 0:
        if nd == 3:
            ux, uy, uz = us
            J = -Lambda / 3. * (V[0] * (ux[4] + ux[8] - uy[1] - uz[2]) + V[1] * (uy[0] + uy[8] - ux[3] - uz[5])
                                + V[2] * (uz[0] + uz[4] - ux[6] - uy[7]))
        else:
            ux, uy = us
            J = -Lambda / 3. * (V[0] * (ux[4] + ux[8] - uy[1]) + V[1] * (uy[0] + uy[8] - ux[3])
                                - V[2] * (ux[6] + uy[7]))
        for i in range(3):
            H[ci(i, i)] = H[ci(i, i)] + J
    return torch.stack(H)


def flux(beta, sig, Lambda=0.0):
    shape = tuple(beta.shape[1:])
    nd = len(shape)
    Dx = 1. / shape[-1]
    der = [find_derivatives(beta, a, Dx) for a in range(nd)]
    corners = [(sx, sy, sz) for sx in (1, 0) for sy in (1, 0) for sz in (1, 0)] if nd == 3 else \
        [(sx, sy) for sx in (1, 0) for sy in (1, 0)]
    us_of = lambda c: [der[a][0] if c[a] else der[a][1] for a in range(nd)]
    Vs = {c: velocity(us_of(c), sig, Lambda) for c in corners}
    sp, sm, tot = [], [], []
    zero = torch.zeros(shape, dtype=beta.dtype, device=beta.device)
    for a in range(nd):
        vals = torch.stack([Vs[c][a] for c in corners] + [zero])
        p = vals.max(0).values
        m = torch.abs(vals.min(0).values)
        sp.append(p)
        sm.append(m)
        tot.append(p + m + ME)
    deriv = 0
    for c in corners:
        w = hamiltonian(us_of(c), Vs[c], Lambda)
        for a in range(nd):
            w = w * (sm[a] if c[a] else sp[a])
        deriv = deriv - w
    for a in range(nd):
        deriv = deriv / tot[a]
    for a in range(nd):
        deriv = deriv + (der[a][0] - der[a][1]) * sm[a] * sp[a] / tot[a]
    return deriv


CZZ = torch.tensor([-0.5, -0.5, 1.0], dtype=torch.float64)


def total_stress(beta, t, mu, nu, rate_zz):
    sig = stress(beta, mu, nu)
    if rate_zz is None:
        return sig
    eps = rate_zz * CZZ.to(beta.device) * t
    lamb = 2. * mu * nu / (1. - 2. * nu)
    tr = eps[0] + eps[1] + eps[2]
    add = [lamb * tr + 2. * mu * eps[i] for i in range(3)]
    out = [sig[c] for c in range(9)]
    for i in range(3):
        out[ci(i, i)] = out[ci(i, i)] + add[i]
    return torch.stack(out)


def step_fixed(beta, t, dt, mu, nu, rate_zz, Lambda=0.0):
    L = lambda v: flux(v, total_stress(v, t, mu, nu, rate_zz), Lambda)
    F0 = beta + dt * L(beta)
    F1 = 0.75 * beta + 0.25 * F0 + 0.25 * (dt * L(F0))
    return (1. / 3.) * beta + (2. / 3.) * F1 + (2. / 3.) * (dt * L(F1))


def loss(beta, mu, nu, w_zz=10.0):
    s = stress(beta, mu, nu)
    e = 0.
    for i in range(3):
        for j in range(3):
            for k in range(3):
                for m in range(3):
                    S = (2. * (i == k) * (j == m) - (i == m) * (j == k) - nu * (i == j) * (k == m) / (1. + nu)) / (2. * mu)
                    e = e + 0.5 * S * s[ci(i, j)] * s[ci(k, m)]
    return e.sum() + w_zz * beta[8].mean()
