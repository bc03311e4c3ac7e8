"""Numerical constants and the elementwise limiters of the reference
(Plasticity/NumericalMethods.py L4, L352-473), for drivers that use them on host arrays."""
import numpy

ME = numpy.finfo(float).eps


def MinMod3(a, b, c):
    """Smallest of three positive values, largest of three non-positive ones, else 0."""
    a, b, c = numpy.asarray(a), numpy.asarray(b), numpy.asarray(c)
    pos = (a > 0) & (b > 0) & (c > 0)
    nonpos = (a <= 0) & (b <= 0) & (c <= 0)
    return numpy.where(pos, numpy.minimum(numpy.minimum(a, b), c),
                       numpy.where(nonpos, numpy.maximum(numpy.maximum(a, b), c), 0.0))


def Max3(a, b, c):
    return numpy.maximum(numpy.maximum(a, b), c)


def Min3(a, b, c):
    return numpy.minimum(numpy.minimum(a, b), c)


def Max5(a, b, c, d, e):
    return Max3(a, b, Max3(c, d, e))


def Min5(a, b, c, d, e):
    return Min3(a, b, Min3(c, d, e))


def Max9(a, b, c, d, e, f, g, h, i):
    return Max5(a, b, c, d, Max5(e, f, g, h, i))


def Min9(a, b, c, d, e, f, g, h, i):
    return Min5(a, b, c, d, Min5(e, f, g, h, i))
