"""Central-upwind Hamilton-Jacobi scheme (reference: Plasticity/FieldDynamics/CentralUpwindHJ3D.py).

The scheme itself runs in libcdd.so (stencil.cu); this module keeps the reference's names:
``CentralUpwindHJDynamics`` (base of the beta^P dynamics) and ``FindDerivatives`` (limited
one-sided derivatives of a host TensorField, L11-34).
"""
import numpy

from Plasticity.FieldDynamics import FieldDynamics
from Plasticity.Fields import Fields

theta = 1.0


def FindDerivatives(field, coord=0, Dx=None):
    """(deriv_p, deriv_m) of every component along axis ``coord`` (periodic)."""
    if Dx is None:
        Dx = 1. / field.gridShape[-1]
    arr = field.stack()
    ax = coord + 1
    diff = numpy.roll(arr, -1, ax) - arr
    e = numpy.roll(diff, -1, ax) - diff            # undivided second difference at i
    em = numpy.roll(e, 1, ax)                      # ... at i - 1
    dd = numpy.where((e > 0) & (em > 0), numpy.minimum(e, em),
                     numpy.where((e < 0) & (em < 0), numpy.maximum(e, em), 0.0))
    dp = (diff - 0.5 * theta * dd) / Dx
    dm = (numpy.roll(diff, 1, ax) + 0.5 * theta * numpy.roll(dd, 1, ax)) / Dx
    return (Fields.from_stack(field.gridShape, dp, field.components),
            Fields.from_stack(field.gridShape, dm, field.components))


class CentralUpwindHJDynamics(FieldDynamics.FieldDynamics):
    def __init__(self, Dx=None):
        self.Dx = Dx
