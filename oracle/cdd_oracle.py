"""CPU oracle for the continuum-dislocation-dynamics time step -- TEST INFRASTRUCTURE ONLY.

This module restates, in vectorised numpy FP64, the reference's Python time-step path of
mattbierbaum/cuda-plasticity. It is the checker for the CUDA library: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import it, and never as
the thing measured or shipped. The product path (``cdd`` and ``Plasticity`` packages) does not
import it.

Parity is pinned: ``tests/test_oracle_golden.py`` checks every function here against golden
vectors in ``tests/golden/*.npz``, which ``tests/golden/make_golden.py`` produced by running the
reference's own (mechanically Python-3-patched) modules on the same seeded inputs.

Every function follows the operation order of the reference code it cites, so that on the same
inputs it reproduces the reference to the last bit or within a few ulps.

Layout: a 9-component field is an array ``(9,) + grid`` with components in the reference's
sorted order xx, xy, xz, yx, yy, yz, zx, zy, zz; grid axis 0 is the reference's x.
"""
import numpy as np

ME = np.finfo(float).eps          # Plasticity/NumericalMethods.py L4
XYZ = "xyz"
COMPONENTS = [(a, b) for a in XYZ for b in XYZ]   # Fields.py L247-249 (sorted)


def ci(i, j):
    """Index of component (i, j) in the 9-component layout."""
    return 3 * i + j


# ----------------------------------------------------------------------------------------------
# k-space tables: Plasticity/GridArray/FourierSpaceTools.py L5-59
# ----------------------------------------------------------------------------------------------
def _identity(a):
    """FourierSpaceTools.py L5-7: wrap angles above pi to (-pi, pi]; +pi is kept."""
    greater = (a > np.pi).astype(float)
    return a - 2 * np.pi * greater


def k_axis(n_scale, n_axis, count, sin_k=False):
    """``n_scale * func(2 pi i / n_axis)`` for i in [0, count) (FourierSpaceTools.py L29-49), func the
    identity wrap or, for the 'sinK' tools (PlasticityState.py L35-39, ``func=sin``), the sine."""
    i = np.arange(count, dtype=np.float64)
    a = 2. * np.pi * i / float(n_axis)
    return n_scale * (np.sin(a) if sin_k else _identity(a))


def k_tables(shape, sin_k=False):
    """Return (k, kSq, kSqSq, kmask) on the rfft half grid, as in FourierSpaceTools.py L26-55.

    ``k`` is a list of three broadcastable arrays (kx, ky, kz). In 2-D both wave vectors are
    scaled by ``gridShape[1]`` (L29-30) and kz is zero; in 3-D each axis uses its own size (L47-49).
    ``sin_k``: the tables of ``FourierSpaceTools(gridShape, func=sin)`` (the observables' type
    'sinK'); kmask is the same.
    """
    if len(shape) == 3:
        n0, n1, n2 = shape
        kx = k_axis(n0, n0, n0, sin_k).reshape(n0, 1, 1)
        ky = k_axis(n1, n1, n1, sin_k).reshape(1, n1, 1)
        kz = k_axis(n2, n2, n2 // 2 + 1, sin_k).reshape(1, 1, n2 // 2 + 1)
        full = (n0, n1, n2 // 2 + 1)
        kx, ky, kz = (np.broadcast_to(v, full) for v in (kx, ky, kz))
        kSq = kx * kx + ky * ky + kz * kz
        kmask = np.ones(full)
        kmask[0, 0, 0] = 0.
    elif len(shape) == 2:
        n0, n1 = shape
        kx = k_axis(n1, n0, n0, sin_k).reshape(n0, 1)
        ky = k_axis(n1, n1, n1 // 2 + 1, sin_k).reshape(1, n1 // 2 + 1)
        full = (n0, n1 // 2 + 1)
        kx, ky = (np.broadcast_to(v, full) for v in (kx, ky))
        kz = np.zeros(full)
        kSq = kx * kx + ky * ky
        kmask = np.ones(full)
        kmask[0, 0] = 0.
    else:
        raise ValueError("only 2-D and 3-D grids are supported")
    kSqSq = kSq * kSq
    return [kx, ky, kz], kSq, kSqSq, kmask


# ----------------------------------------------------------------------------------------------
# Stress: PlasticityState.CalculateSigma(type='k', source='betaE') L85-127 and
#         PlasticityState.CalculateBetaElastic L357-390
# ----------------------------------------------------------------------------------------------
def beta_elastic(beta, mu, nu, sin_k=False):
    shape = beta.shape[1:]
    axes = tuple(range(-len(shape), 0))
    KbetaP = np.fft.rfftn(beta, axes=axes)
    lamb = 2. * mu * nu / (1. - 2 * nu)
    k, kSq0, kSqSq0, kmask = k_tables(shape, sin_k)
    kSq = kSq0 + ME
    kSqSq = kSqSq0 + ME
    KbetaE = np.zeros_like(KbetaP)
    for i in range(3):
        for j in range(3):
            acc = np.zeros(KbetaP.shape[1:], dtype=complex)
            for m in range(3):
                for n in range(3):
                    T = lamb / (lamb + 2. * mu) * k[i] * k[j] / kSq * (m == n) + \
                        k[i] / kSq * ((k[m] * (j == n)) + (k[n] * (j == m))) - \
                        2. * (lamb + mu) / (lamb + 2. * mu) * (k[i] * k[j] * k[m] * k[n]) / kSqSq
                    acc += KbetaP[ci(m, n)] * T
            acc *= kmask
            KbetaE[ci(i, j)] = acc
    betaE = np.fft.irfftn(KbetaE, s=shape, axes=axes)
    return betaE - beta


def stress(beta, mu, nu):
    """Internal stress sigma (9 components, symmetric) of plastic distortion ``beta``."""
    betaE = beta_elastic(beta, mu, nu)
    lamb = 2. * mu * nu / (1. - 2. * nu)
    tr = betaE[0] + betaE[4] + betaE[8]
    sigma = np.zeros_like(beta)
    for i in range(3):
        for j in range(3):
            sigma[ci(i, j)] += lamb * tr * (i == j) + mu * (betaE[ci(i, j)] + betaE[ci(j, i)])
    return sigma


def applied_stress(t, rate, mu, nu, initial=(0., 0., 0.), t0=0.):
    """Uniform diagonal stress of an applied strain (RunPython.py L21-26, L44-47).

    ``eps = initial + rate * (t - t0)``; ``sigma_ii += lamb tr(eps) + 2 mu eps_i``. The caller
    chooses mu, nu (RunPython.py uses module-level 0.5, 0.3; the workloads use the state's).
    """
    eps = np.asarray(initial, float) + np.asarray(rate, float) * (t - t0)
    lamb = 2. * mu * nu / (1. - 2. * nu)
    tr = eps[0] + eps[1] + eps[2]
    return np.array([lamb * tr + 2. * mu * eps[i] for i in range(3)])


def elastic_energy_density(sigma, mu, nu):
    """PlasticityState.CalculateElasticEnergy L317-330 (all 81 terms, reference order)."""
    e = 0.
    for i in range(3):
        for j in range(3):
            for k in range(3):
                for m in range(3):
                    S = (2. * (i == k) * (j == m) - (i == m) * (j == k)
                         - nu * (i == j) * (k == m) / (1. + nu)) / (2. * mu)
                    e += 0.5 * S * sigma[ci(i, j)] * sigma[ci(k, m)]
    return e


def elastic_energy(beta, mu, nu):
    """Total elastic energy, summed over cells as Observers/Observer.py L99 does."""
    return float(np.sum(elastic_energy_density(stress(beta, mu, nu), mu, nu)))


def mean_strain_zz(beta):
    """``numpy.average(betaP[z,z])`` (MattTools/Run/RunLoadingMPI.py L32)."""
    return float(np.mean(beta[8]))


# ----------------------------------------------------------------------------------------------
# Limited one-sided derivatives: CentralUpwindHJ3D.py L11-34 with NumericalMethods.py L352-473
# ----------------------------------------------------------------------------------------------
def minmod3(a, b, c):
    """NumericalMethods.MinMod3 L367-378 (0/1-mask form)."""
    cond_a = (a > 0)
    cond_b = (b > 0)
    cond_c = (c > 0)
    cond_ab = (a < b)
    cond_bc = (b < c)
    cond_ac = (a < c)
    cond_abc = cond_a * cond_b * cond_c
    cond_not_abc = (1 - cond_a) * (1 - cond_b) * (1 - cond_c)
    return cond_abc * (cond_ab * cond_ac * a + (1 - cond_ab) * cond_bc * b
                       + (1 - cond_bc) * (1 - cond_ac) * c) + \
        cond_not_abc * ((1 - cond_ab) * (1 - cond_ac) * a + cond_ab * (1 - cond_bc) * b
                        + cond_bc * cond_ac * c)


THETA = 1.0   # CentralUpwindHJ3D.py L9


def find_derivatives(field, axis, Dx):
    """Return (deriv_p, deriv_m) of every component along grid ``axis`` (L11-34).

    ``field`` has the component axis first; ``axis`` counts grid axes from 0.
    """
    ax = axis + 1
    roll = np.roll
    diff = roll(field, -1, ax) - field
    diff2_1 = THETA * (roll(diff, -1, ax) - diff) / Dx / Dx
    diff2_2 = (roll(diff, -1, ax) - roll(diff, 1, ax)) / Dx / Dx * 0.5
    diff2_3 = roll(diff2_1, 1, ax)
    diff2 = minmod3(diff2_1, diff2_2, diff2_3)
    deriv_p = diff / Dx - 0.5 * Dx * diff2
    deriv_m = roll(diff, 1, ax) / Dx + 0.5 * Dx * roll(diff2, 1, ax)
    return deriv_p, deriv_m


# ----------------------------------------------------------------------------------------------
# Beta^P Hamiltonian: CentralUpwindHJBetaPDynamics3D.py L34-212 (2-D twin:
# CentralUpwindHJBetaPDynamics.py L34-134, identical arithmetic)
# ----------------------------------------------------------------------------------------------
def rho_mod(us):
    """|rho| at a corner from its derivative tensors ``us`` (2 or 3 of them), L34-58."""
    rho2 = ME
    for c in range(9):
        for u in us:
            rho2 = rho2 + u[c] * u[c]
    for j in range(3):
        for d, u in enumerate(us):
            rho2 = rho2 - u[ci(d, j)] * u[ci(d, j)]
        if len(us) == 2:
            rho2 = rho2 - 2 * us[0][ci(1, j)] * us[1][ci(0, j)]
        else:
            ux, uy, uz = us
            rho2 = rho2 - 2 * ux[ci(1, j)] * uy[ci(0, j)]
            rho2 = rho2 - 2 * uy[ci(2, j)] * uz[ci(1, j)]
            rho2 = rho2 - 2 * uz[ci(0, j)] * ux[ci(2, j)]
    return np.sqrt(rho2)


def velocity(us, sigma, Lambda):
    """Dislocation velocity V (3 components) at a corner, L77-142."""
    shape = us[0].shape[1:]
    V = [np.zeros(shape), np.zeros(shape), np.zeros(shape)]
    nd = len(us)
    for n in range(3):
        for l in range(3):
            for d in range(nd):
                V[l] = V[l] + us[d][ci(l, n)] * sigma[ci(d, n)]
            for d in range(nd):
                V[d] = V[d] - us[d][ci(l, n)] * sigma[ci(l, n)]
    if Lambda != 0:
        sigma_tr = (sigma[0] + sigma[4] + sigma[8]) / 3. * Lambda
        for d in range(nd):
            V[d] = V[d] + sigma_tr * (us[d][0] + us[d][4] + us[d][8])
        for l in range(3):
            acc = us[0][ci(l, 0)]
            for d in range(1, nd):
                acc = acc + us[d][ci(l, d)]
            V[l] = V[l] - sigma_tr * acc
    rho = rho_mod(us)
    return [v / rho for v in V]


def velocity_glide(us, sigma):
    """Glide-only velocity at a corner: the climb velocity projected as in
    CentralUpwindHJBetaPGlideOnlyDynamics.py BetaP3D_Velocity L152-201 (2-D: BetaP2D_Velocity
    L96-129), in the reference's operation order; climb velocity L131-150 / L73-94."""
    shape = us[0].shape[1:]
    nd = len(us)
    v = [np.zeros(shape), np.zeros(shape), np.zeros(shape)]
    for n in range(3):
        for l in range(3):
            for d in range(nd):
                v[l] = v[l] + us[d][ci(l, n)] * sigma[ci(d, n)]
            for d in range(nd):
                v[d] = v[d] - us[d][ci(l, n)] * sigma[ci(l, n)]
    if nd == 3:
        ux, uy, uz = us
        rhorho = ME
        uxTr = ux[0] + ux[4] + ux[8]
        uyTr = uy[0] + uy[4] + uy[8]
        uzTr = uz[0] + uz[4] + uz[8]
        rhorho = rhorho + (uxTr * uxTr + uyTr * uyTr + uzTr * uzTr)
        rhorho = rhorho - 2 * uxTr * (ux[0] + uy[1] + uz[2])
        rhorho = rhorho - 2 * uyTr * (ux[3] + uy[4] + uz[5])
        rhorho = rhorho - 2 * uzTr * (ux[6] + uy[7] + uz[8])
        for n in range(3):
            t = ux[ci(n, 0)] + uy[ci(n, 1)] + uz[ci(n, 2)]
            rhorho = rhorho + t * t
        rhov = ME
        rhov = rhov + v[0] * (ux[8] + ux[4] - uy[1] - uz[2])
        rhov = rhov + v[1] * (uy[0] + uy[8] - ux[3] - uz[5])
        rhov = rhov + v[2] * (uz[0] + uz[4] - ux[6] - uy[7])
        factor = rhov / rhorho
        v[0] = v[0] + (ux[4] + ux[8] - uy[1] - uz[2]) * factor
        v[1] = v[1] + (uy[0] + uy[8] - ux[3] - uz[5]) * factor
        v[2] = v[2] + (uz[0] + uz[4] - ux[6] - uy[7]) * factor
    else:
        ux, uy = us
        rhorho = ME
        uxTr = ux[0] + ux[4] + ux[8]
        uyTr = uy[0] + uy[4] + uy[8]
        rhorho = rhorho + (uxTr * uxTr + uyTr * uyTr)
        rhorho = rhorho - 2 * uxTr * (ux[0] + uy[1])
        rhorho = rhorho - 2 * uyTr * (ux[3] + uy[4])
        for n in range(3):
            t = ux[ci(n, 0)] + uy[ci(n, 1)]
            rhorho = rhorho + t * t
        rhov = ME
        rhov = rhov + v[0] * (ux[8] + ux[4] - uy[1])
        rhov = rhov + v[1] * (uy[0] + uy[8] - ux[3])
        rhov = rhov + (-v[2]) * (ux[6] + uy[7])
        v[0] = v[0] + (ux[4] + ux[8] - uy[1]) * rhov / rhorho
        v[1] = v[1] + (uy[0] + uy[8] - ux[3]) * rhov / rhorho
        v[2] = v[2] - (ux[6] + uy[7]) * rhov / rhorho
    rho = rho_mod(us)
    return [w / rho for w in v]


def hamiltonian(us, V, Lambda):
    """H_ij at a corner (L161-201)."""
    nd = len(us)
    H = us[0] * V[0]
    for d in range(1, nd):
        H = H + us[d] * V[d]
    for j in range(3):
        for l in range(3):
            for i in range(nd):
                H[ci(i, j)] = H[ci(i, j)] - V[l] * us[i][ci(l, j)]
    if Lambda != 0:
        if nd == 3:
            ux, uy, uz = us
            J = -Lambda / 3. * (V[0] * (ux[4] + ux[8] - uy[1] - uz[2])
                                + V[1] * (uy[0] + uy[8] - ux[3] - uz[5])
                                + V[2] * (uz[0] + uz[4] - ux[6] - uy[7]))
        else:
            ux, uy = us
            J = -Lambda / 3. * (V[0] * (ux[4] + ux[8] - uy[1])
                                + V[1] * (uy[0] + uy[8] - ux[3])
                                - V[2] * (ux[6] + uy[7]))
        for i in range(3):
            H[ci(i, i)] = H[ci(i, i)] + J
    return H


# ----------------------------------------------------------------------------------------------
# Central-upwind flux: CentralUpwindHJ3D.CalculateFlux L99-271
# ----------------------------------------------------------------------------------------------
def flux(beta, sigma, Lambda=0, Dx=None, glide=False):
    """Return (rhs, speed) for plastic distortion ``beta`` under total stress ``sigma``.
    glide: the glide-only dynamics (CentralUpwindHJBetaPGlideOnlyDynamics.py: projected velocity,
    no Lambda term)."""
    shape = beta.shape[1:]
    nd = len(shape)
    if Dx is None:
        Dx = 1. / shape[-1]                       # CentralUpwindHJ3D.py L15-16
    der = [find_derivatives(beta, a, Dx) for a in range(nd)]   # [(p, m)] per axis
    if nd == 3:
        corners = [(sx, sy, sz) for sx in (1, 0) for sy in (1, 0) for sz in (1, 0)]
    else:
        corners = [(sx, sy) for sx in (1, 0) for sy in (1, 0)]

    def us_of(c):
        return [der[a][0] if c[a] else der[a][1] for a in range(nd)]

    if glide:
        Vs = {c: velocity_glide(us_of(c), sigma) for c in corners}
        Lambda = 0
    else:
        Vs = {c: velocity(us_of(c), sigma, Lambda) for c in corners}
    sp, sm, tot = [], [], []
    for a in range(nd):
        vals = [Vs[c][a] for c in corners]
        p = np.maximum.reduce(vals + [np.zeros(shape)])          # Max9 / Max5 with 0
        m = np.fabs(np.minimum.reduce(vals + [np.zeros(shape)]))  # Min9 / Min5 with 0
        sp.append(p)
        sm.append(m)
        tot.append(p + m + ME)
    deriv = None
    for c in corners:
        H = hamiltonian(us_of(c), Vs[c], Lambda)
        w = H
        for a in range(nd):
            w = w * (sm[a] if c[a] else sp[a])
        deriv = -w if deriv is None else deriv - w
    for a in range(nd):
        deriv = deriv / tot[a]
    for a in range(nd):
        deriv = deriv + (der[a][0] - der[a][1]) * sm[a] * sp[a] / tot[a]
    speed = tot[0] + tot[1]
    if nd == 3:
        speed = speed + tot[2]
    return deriv, speed


class Params:
    """Material, loading and integrator parameters of one instance."""

    def __init__(self, mu=1.0, nu=0.3, Lambda=0, cfl=0.25, load_rate=None,
                 load_initial=(0., 0., 0.), load_t0=0., load_mu=None, load_nu=None, glide=False,
                 vacancy=None, dt_bound=None):
        self.mu, self.nu, self.Lambda, self.cfl = mu, nu, Lambda, cfl
        self.glide = glide
        self.vacancy = vacancy            # (alpha, beta, gamma) of the vacancy coupling, or None
        self.dt_bound = dt_bound          # the splitting mover's dtBound (None: no bound)
        self.load_rate = None if load_rate is None else np.asarray(load_rate, float)
        self.load_initial = np.asarray(load_initial, float)
        self.load_t0 = load_t0
        self.load_mu = mu if load_mu is None else load_mu
        self.load_nu = nu if load_nu is None else load_nu


def total_stress(beta, t, p):
    """Dynamics' GetSigma: internal stress plus the applied load at time t."""
    sigma = stress(beta, p.mu, p.nu)
    if p.load_rate is not None:
        add = applied_stress(t, p.load_rate, p.load_mu, p.load_nu, p.load_initial, p.load_t0)
        for i in range(3):
            sigma[ci(i, i)] += add[i]
    return sigma


def full_flux(beta, t, p):
    """BetaPDynamics.CalculateFlux (CentralUpwindHJBetaPDynamics3D.py L218-221)."""
    return flux(beta, total_stress(beta, t, p), p.Lambda, glide=p.glide)


# ----------------------------------------------------------------------------------------------
# TVD Runge-Kutta 3: FieldMover.py L38-141
# ----------------------------------------------------------------------------------------------
def rk3_step(beta, t, t_end, p, fixed_dt=None):
    """One TVD-RK3 step; returns (beta_new, dt).

    Adaptive (L61-141): dt = CFL / (max(gridShape) * max(speed)), clamped so t + dt <= t_end.
    Fixed (L38-58): dt = fixed_dt, clamped the same way. All three stages use the same ``t``.
    """
    rhs, speed = full_flux(beta, t, p)
    if fixed_dt is None:
        s = max(beta.shape[1:]) * speed.max()
        dt = float(p.cfl / s)
    else:
        dt = float(fixed_dt)
    if t + dt > t_end:
        dt = t_end - t
    F0 = 1.0 * beta + 1.0 * (dt * rhs)
    rhs, _ = full_flux(F0, t, p)
    F1 = 0.75 * beta + 0.25 * F0 + 0.25 * (dt * rhs)
    rhs, _ = full_flux(F1, t, p)
    F2 = (1. / 3.) * beta + (2. / 3.) * F1 + (2. / 3.) * (dt * rhs)
    return F2, dt


def run(beta, t0, t_end, p, max_steps=None, observer=None):
    """TVDRungeKutta_FieldMover.Run (L20-36): step until t >= t_end."""
    t = t0
    n = 0
    while True:
        beta, dt = rk3_step(beta, t, t_end, p)
        t += dt
        n += 1
        if observer is not None:
            observer(t, beta)
        if t >= t_end or (max_steps is not None and n >= max_steps):
            return beta, t


# ----------------------------------------------------------------------------------------------
# Vacancy coupling: BetaP_VacancyDynamics (VacancyDynamics.py L16-61) stepped by
# OperatorSplittingTVDRK_FieldMover.CalculateOneAdaptiveTimeStep (FieldMover.py L344-380).
# ----------------------------------------------------------------------------------------------
def vacancy_flux(beta, c, p):
    """CalculateFlux with GetSigma: the internal stress minus alpha c on the diagonal (no load)."""
    sigma = stress(beta, p.mu, p.nu)
    for i in range(3):
        sigma[ci(i, i)] -= p.vacancy[0] * c
    return flux(beta, sigma, p.Lambda)


def diffuse(c, gamma, dt):
    """DiffusionEvolution: c^ * exp(kSq * -gamma * dt) (kSq of the k tables, no ME)."""
    shape = c.shape
    kc = np.fft.rfftn(c)
    kt = k_tables(shape)[1] * -gamma * dt
    return np.fft.irfftn(kc * np.exp(kt), s=shape)


def vacancy_step(beta, c, t, t_end, p):
    """One operator-splitting step; returns (beta_new, c_new, dt)."""
    alpha_rk = [[1.], [3. / 4., 1. / 4.], [1. / 3., 0., 2. / 3.]]
    beta_rk = [[1.], [0., 1. / 4.], [0., 0., 2. / 3.]]
    prev_tr = beta[0] + beta[4] + beta[8]
    rhs, speed = vacancy_flux(beta, c, p)
    dt = float(p.cfl / (max(beta.shape[1:]) * speed.max()))
    if p.dt_bound is not None and dt > p.dt_bound:
        dt = p.dt_bound
    if t + dt > t_end:
        dt = t_end - t
    L0 = dt * rhs
    F0 = alpha_rk[0][0] * beta + beta_rk[0][0] * L0
    L1 = dt * vacancy_flux(F0, c, p)[0]
    F1 = alpha_rk[1][0] * beta + beta_rk[1][0] * L0 + alpha_rk[1][1] * F0 + beta_rk[1][1] * L1
    L2 = dt * vacancy_flux(F1, c, p)[0]
    F2 = (alpha_rk[2][0] * beta + beta_rk[2][0] * L0 + alpha_rk[2][1] * F0 + beta_rk[2][1] * L1
          + alpha_rk[2][2] * F1 + beta_rk[2][2] * L2)
    tr = F2[0] + F2[4] + F2[8]
    c = c + p.vacancy[1] * (tr - prev_tr)
    return F2, diffuse(c, p.vacancy[2], dt), dt


# ----------------------------------------------------------------------------------------------
# The reference CUDA solver's on-disk formats: convertStateToCUDA (Plasticity/RunCUDA.py L9-22)
# writes every component transposed (grid axis 0 fastest); ContinueWriteMatrix (assist.h
# L164-192) appends frames [t][field] in the solver's data_type; LoadStateRaw
# (Plasticity/FieldInitializers/FieldInitializer.py L61-103) reads them back.
# ----------------------------------------------------------------------------------------------
def to_file_layout(field):
    """(9,) + grid -> (9,) + reversed grid: component c transposed (all axes reversed)."""
    return np.stack([np.ascontiguousarray(np.asarray(c).transpose()) for c in field])


def from_file_layout(data, shape):
    """Inverse of to_file_layout for a flat array of 9 * prod(shape) values."""
    d = np.asarray(data).reshape((9,) + tuple(reversed(shape)))
    return np.stack([np.ascontiguousarray(c.transpose()) for c in d])


def ics_bytes(field):
    """An .ics initial condition: the field in the file layout as float64, no time."""
    return to_file_layout(np.asarray(field, dtype=np.float64)).tobytes()


def plas_frame_bytes(t, field, dtype=np.float64):
    """One .plas frame: the time, then the field in the file layout, both in `dtype`."""
    dtype = np.dtype(dtype)
    return np.array([t], dtype=dtype).tobytes() + to_file_layout(np.asarray(field).astype(dtype)).tobytes()


def read_plas(raw, shape, dtype=np.float64, time=None):
    """(t, field) of the frame LoadStateRaw selects: the last one (time None) or the first with
    t >= time (the last read when none is), from the bytes of a .plas file."""
    dtype = np.dtype(dtype)
    n = 9 * int(np.prod(shape))
    frame = (n + 1) * dtype.itemsize
    count = len(raw) // frame
    k = count - 1
    if time is not None:
        for k in range(count):
            if np.frombuffer(raw, dtype, 1, k * frame)[0] >= time:
                break
    t = np.frombuffer(raw, dtype, 1, k * frame)[0]
    data = np.frombuffer(raw, dtype, n, k * frame + dtype.itemsize)
    return float(t), from_file_layout(data, shape)


# ----------------------------------------------------------------------------------------------
# Field observables: PlasticityState.CalculateRhoFourier L264-304, CalculateRotationField
# L435-446, CalculateRotationRodrigues L447-475 (source 'betaP'); beta_elastic above is
# CalculateBetaElastic L357-390.
# ----------------------------------------------------------------------------------------------
PERM = np.zeros((3, 3, 3))                        # Constants.py L16-22
PERM[0, 1, 2] = PERM[1, 2, 0] = PERM[2, 0, 1] = 1.
PERM[0, 2, 1] = PERM[2, 1, 0] = PERM[1, 0, 2] = -1.


def rho_fourier(beta, sin_k=False):
    """Nye density rho_ij = -eps_ikl d_k beta_lj with Fourier derivatives d_k -> i k_k (no kmask)."""
    shape = beta.shape[1:]
    axes = tuple(range(-len(shape), 0))
    Kb = np.fft.rfftn(beta, axes=axes)
    k = k_tables(shape, sin_k)[0]
    D = [Kb * (1.0j * k[d]) for d in range(len(shape))]
    Kr = np.zeros_like(Kb)
    for i in range(3):
        if len(shape) == 3:
            Kr[ci(0, i)] = D[2][ci(1, i)] - D[1][ci(2, i)]
            Kr[ci(1, i)] = D[0][ci(2, i)] - D[2][ci(0, i)]
            Kr[ci(2, i)] = D[1][ci(0, i)] - D[0][ci(1, i)]
        else:
            Kr[ci(0, i)] = -D[1][ci(2, i)]
            Kr[ci(1, i)] = D[0][ci(2, i)]
            Kr[ci(2, i)] = D[1][ci(0, i)] - D[0][ci(1, i)]
    return np.fft.irfftn(Kr, s=shape, axes=axes)


def rotation_field(beta, mu, nu, sin_k=False):
    """rotE_ij = (betaE_ij - betaE_ji) / 2, 9 components."""
    be = beta_elastic(beta, mu, nu, sin_k)
    return np.stack([(be[ci(i, j)] - be[ci(j, i)]) / 2. for i in range(3) for j in range(3)])


def rodrigues(beta, sin_k=False):
    """Rodrigues vector (x, y, z) from beta^P: IFFT(kmask sum k_j (e_ijt k_s + e_ijs k_t) b_st /
    kSq / 2) minus the antisymmetric part of beta^P."""
    shape = beta.shape[1:]
    axes = tuple(range(-len(shape), 0))
    Kb = np.fft.rfftn(beta, axes=axes)
    k, kSq0, _, kmask = k_tables(shape, sin_k)
    kSq = kSq0 + ME
    Kr = np.zeros((3,) + Kb.shape[1:], dtype=complex)
    for i in range(3):
        for s in range(3):
            for t in range(3):
                for j in range(3):
                    Kr[i] += k[j] * (PERM[i, j, t] * k[s] + PERM[i, j, s] * k[t]) * Kb[ci(s, t)] / kSq / 2.
        Kr[i] *= kmask
    rod = np.fft.irfftn(Kr, s=shape, axes=axes)
    rod[0] -= (beta[ci(1, 2)] - beta[ci(2, 1)]) / 2.
    rod[1] -= (beta[ci(2, 0)] - beta[ci(0, 2)]) / 2.
    rod[2] -= (beta[ci(0, 1)] - beta[ci(1, 0)]) / 2.
    return rod


def rodrigues_from_rho(beta, sin_k=False):
    """Rodrigues vector from the Nye density (CalculateRotationRodrigues source 'rho',
    PlasticityState.py L472-494): rho = rho_fourier(beta) as a real field, then
    IFFT(kmask sum_mn D_imn FFT(rho)_mn) with D_imn = i (2 k_n d_im - k_m d_in - k_i d_mn) / (2 kSq)
    + i k_i k_n k_m / (2 kSqSq), kSq = |k|^2 + ME, kSqSq = |k|^4 + ME."""
    shape = beta.shape[1:]
    axes = tuple(range(-len(shape), 0))
    rho = rho_fourier(beta, sin_k)
    KR = np.fft.rfftn(rho, axes=axes)
    k, kSq0, kSqSq0, kmask = k_tables(shape, sin_k)
    kSq = kSq0 + ME
    kSqSq = kSqSq0 + ME
    Kr = np.zeros((3,) + KR.shape[1:], dtype=complex)
    for i in range(3):
        for m in range(3):
            for n in range(3):
                D = ((1.j) / (2. * kSq)) * (2. * k[n] * (i == m) - k[m] * (i == n) - k[i] * (m == n)) + \
                    (1.j) * k[i] * k[n] * k[m] / (2. * kSqSq)
                Kr[i] += D * KR[ci(m, n)]
        Kr[i] *= kmask
    return np.fft.irfftn(Kr, s=shape, axes=axes)
