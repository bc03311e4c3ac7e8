"""Host array type of the facades (reference: Plasticity/GridArray/GridArray.py L7-120).

A numpy.ndarray subclass with the reference's method names; fields handed to drivers are host
copies of the device state in this type.
"""
import numpy
import numpy.fft as fft


def print_mem_usage():
    pass


class NumpyArray(numpy.ndarray):
    def __new__(subtype, data, dtype=None, copy=False):
        arr = numpy.array(data, dtype=dtype, copy=True if copy else None)
        return arr.view(subtype)

    def symbol(self):
        return self
    _s = symbol

    def evaluate(self):
        return self
    _e = evaluate

    def numpy_array(self):
        return numpy.asarray(self)

    def rfftn(self):
        return NumpyArray(fft.rfftn(numpy.asarray(self)))

    def irfftn(self, shape=None):
        return NumpyArray(fft.irfftn(numpy.asarray(self), shape))

    def roll(self, offset, direction):
        return NumpyArray(numpy.roll(numpy.asarray(self), offset, direction))

    def sqrt(self):
        return NumpyArray(numpy.sqrt(self))

    def log(self):
        return NumpyArray(numpy.log(self))

    def abs(self):
        return NumpyArray(numpy.abs(self))

    def fabs(self):
        return NumpyArray(numpy.fabs(self))

    def sign(self):
        return NumpyArray(numpy.sign(self))

    def exp(self):
        return NumpyArray(numpy.exp(self))

    def power(self, p):
        return NumpyArray(numpy.power(self, p))

    def average(self):
        return numpy.ndarray.sum(self) / self.size

    @staticmethod
    def empty(shape, dtype='float64'):
        return NumpyArray(numpy.empty(shape, dtype=dtype))

    @staticmethod
    def zeros(shape, dtype='float64'):
        return NumpyArray(numpy.zeros(shape, dtype=dtype))


GridArray = NumpyArray
random_normal = numpy.random.normal
