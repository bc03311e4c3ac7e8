"""Analytic stress of a single Fourier mode (a known answer independent of the oracle and of any
FFT): beta^P = B cos(2 pi m . x) on a periodic unit box gives beta^E = (T(k) B - B) cos(2 pi m . x),
T the isotropic Green's operator of PlasticityState.CalculateBetaElastic (PlasticityState.py
L357-390) at k = 2 pi m, and sigma = lam tr(beta^E) I + mu (beta^E + beta^E^T)."""
import numpy as np


def field(shape, m, B):
    """(9,) + shape array of B_ij cos(2 pi m . x), x_d = i_d / n_d."""
    grids = np.meshgrid(*[np.arange(n) / n for n in shape], indexing="ij")
    phase = 2 * np.pi * sum(md * g for md, g in zip(m, grids))
    c = np.cos(phase)
    return np.stack([B[i, j] * c for i in range(3) for j in range(3)])


def stress(shape, m, B, mu, nu):
    """The analytic internal stress (9 components) of field(shape, m, B)."""
    k = 2 * np.pi * np.asarray(m, dtype=float)
    ksq = float(k @ k)
    lam = 2. * mu * nu / (1. - 2. * nu)
    A = lam / (lam + 2. * mu)
    Bc = 2. * (lam + mu) / (lam + 2. * mu)
    TB = (A * np.trace(B) / ksq) * np.outer(k, k) + np.outer(k, B.T @ k + B @ k) / ksq \
        - (Bc * float(k @ B @ k) / ksq ** 2) * np.outer(k, k)
    E = TB - B
    S = lam * np.trace(E) * np.eye(3) + mu * (E + E.T)
    return field(shape, m, S)
