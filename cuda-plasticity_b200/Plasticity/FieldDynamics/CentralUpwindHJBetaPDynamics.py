"""2-D module of the reference's beta^P dynamics (Plasticity/FieldDynamics/CentralUpwindHJBetaPDynamics.py),
the one RunPython.py imports; the GPU path is the same as the 3-D module's."""
from Plasticity.FieldDynamics.CentralUpwindHJBetaPDynamics3D import BetaPDynamics  # noqa: F401
