"""The oracle's field observables (beta^E, rotation, Rodrigues vector from beta^P and from rho, Nye
density; 'k' and 'sinK' tables) against the reference's own PlasticityState methods on the same
seeded fields (tests/golden/observables.npz, made by tests/golden/make_golden.py)."""
import numpy as np
import pytest

import cdd_oracle as O
from conftest import golden_path

G = np.load(golden_path("observables"))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


@pytest.mark.parametrize("key", ["c", "a", "2d"])
def test_oracle_observables_match_reference(key):
    beta = G["beta_" + key]
    assert rel(O.beta_elastic(beta, 1.0, 0.3), G["betaE_" + key]) < 1e-13
    assert rel(O.rotation_field(beta, 1.0, 0.3), G["rot_" + key]) < 1e-13
    assert rel(O.rodrigues(beta), G["rod_" + key]) < 1e-13
    assert rel(O.rho_fourier(beta), G["rho_" + key]) < 1e-13


@pytest.mark.parametrize("key", ["c", "a", "2d"])
def test_oracle_sink_and_rho_source_match_reference(key):
    beta = G["beta_" + key]
    assert rel(O.beta_elastic(beta, 1.0, 0.3, sin_k=True), G["betaE_sink_" + key]) < 1e-13
    assert rel(O.rotation_field(beta, 1.0, 0.3, sin_k=True), G["rot_sink_" + key]) < 1e-13
    assert rel(O.rodrigues(beta, sin_k=True), G["rod_sink_" + key]) < 1e-13
    assert rel(O.rho_fourier(beta, sin_k=True), G["rho_sink_" + key]) < 1e-13
    assert rel(O.rodrigues_from_rho(beta), G["rodrho_" + key]) < 1e-13
    assert rel(O.rodrigues_from_rho(beta, sin_k=True), G["rodrho_sink_" + key]) < 1e-13
