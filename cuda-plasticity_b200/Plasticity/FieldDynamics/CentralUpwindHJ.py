"""2-D twin of CentralUpwindHJ3D (reference: Plasticity/FieldDynamics/CentralUpwindHJ.py)."""
from Plasticity.FieldDynamics.CentralUpwindHJ3D import CentralUpwindHJDynamics, FindDerivatives, theta  # noqa: F401
