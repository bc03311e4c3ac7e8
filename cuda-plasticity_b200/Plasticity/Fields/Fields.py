"""Component-keyed tensor fields (reference: Plasticity/Fields/Fields.py L7-393).

A Field maps component keys (sorted; ('x','x') .. ('z','z') for a TensorField) to GridArrays.
Algebra is componentwise, as in the reference. ``stack()``/``from_stack()`` convert to and from
the (components,) + grid array layout that the GPU library uses.
"""
import numpy

from Plasticity.GridArray import GridArray
from Plasticity.GridArray import FourierSpaceTools

COMPONENTS9 = [('x', 'x'), ('x', 'y'), ('x', 'z'), ('y', 'x'), ('y', 'y'), ('y', 'z'),
               ('z', 'x'), ('z', 'y'), ('z', 'z')]


def NoneAllocator(*args, **kwargs):
    return None


class Field(object):
    def __init__(self, gridShape, components, kspace=False, allocator=None):
        self.gridShape = gridShape
        self.components = sorted(components)
        self.data = {}
        if allocator is None:
            allocator = GridArray.GridArray.zeros
        shape = FourierSpaceTools.FourierSpaceTools(gridShape).gridShape if kspace else gridShape
        for c in self.components:
            self.data[c] = allocator(shape, dtype='complex') if kspace else allocator(shape)

    def evaluate(self):
        return self

    def GridShape(self):
        return self.gridShape

    def GridDimension(self):
        return len(self.gridShape)

    def __getitem__(self, index):
        return self.data[index]

    def __setitem__(self, index, value):
        self.data[index] = value

    def _new(self):
        return self.__class__(self.gridShape, list(self.components), allocator=NoneAllocator)

    def FFT(self, out=None):
        out = self.__class__(self.gridShape, list(self.components), kspace=True,
                             allocator=NoneAllocator) if out is None else out
        for c in self.components:
            out[c] = GridArray.GridArray(numpy.fft.rfftn(numpy.asarray(self.data[c])))
        return out

    def IFFT(self, out=None):
        out = self._new() if out is None else out
        for c in self.components:
            out[c] = GridArray.GridArray(numpy.fft.irfftn(numpy.asarray(self.data[c]), self.gridShape))
        return out

    def _binary(self, other, op):
        r = self._new()
        for c in self.components:
            r[c] = op(self[c], other[c] if isinstance(other, Field) else other)
        return r

    def __add__(self, o):
        return self._binary(o, lambda a, b: a + b)

    def __radd__(self, o):
        return self.__add__(o)

    def __sub__(self, o):
        return self._binary(o, lambda a, b: a - b)

    def __rsub__(self, o):
        return self._binary(o, lambda a, b: b - a)

    def __mul__(self, o):
        return self._binary(o, lambda a, b: a * b)

    def __rmul__(self, o):
        return self.__mul__(o)

    def __truediv__(self, o):
        return self._binary(o, lambda a, b: a / b)

    def __rtruediv__(self, o):
        return self._binary(o, lambda a, b: b / a)

    def __neg__(self):
        r = self._new()
        for c in self.components:
            r[c] = -self[c]
        return r

    def numpy_arrays(self):
        r = self._new()
        for c in self.components:
            r[c] = numpy.asarray(self[c])
        return r

    def fabs(self):
        r = self._new()
        for c in self.components:
            r[c] = GridArray.GridArray(numpy.fabs(self[c]))
        return r

    def sqrt(self):
        r = self._new()
        for c in self.components:
            r[c] = GridArray.GridArray(numpy.sqrt(self[c]))
        return r

    def max(self):
        return max(numpy.max(self[c]) for c in self.components)

    def min(self):
        return min(numpy.min(self[c]) for c in self.components)

    def sum(self):
        return sum(float(numpy.sum(self[c])) for c in self.components)

    def modulus(self):
        acc = 0.
        for c in self.components:
            acc = acc + self[c] * self[c]
        return GridArray.GridArray(numpy.sqrt(acc))

    def stack(self, dtype=numpy.float64):
        """(components,) + grid array in sorted component order."""
        return numpy.stack([numpy.asarray(self.data[c], dtype=dtype) for c in self.components])

    def load_stack(self, arr):
        for i, c in enumerate(self.components):
            self.data[c] = GridArray.GridArray(numpy.array(arr[i], dtype=numpy.float64))
        return self


class TensorField(Field):
    """Rank-2 tensor field; 9 components ('x','x') .. ('z','z') by default."""

    def __init__(self, gridShape, components=None, rank=None, directions=['x', 'y', 'z'],
                 directionList=None, kspace=False, allocator=None):
        if components is None:
            if rank is not None:
                components = self.GenerateComponents(rank=rank, directions=directions)
            elif directionList is not None:
                components = self.GenerateComponentsFromList(directionList)
            else:
                components = list(COMPONENTS9)
        super(TensorField, self).__init__(gridShape, components, kspace=kspace, allocator=allocator)

    def GenerateComponents(self, rank=2, directions=['x', 'y', 'z']):
        pool = list(directions)
        for _ in range(rank - 1):
            pool = [tuple(list(e if isinstance(e, tuple) else (e,)) + [d]) for e in pool for d in directions]
        return pool

    def GenerateComponentsFromList(self, dirList):
        pool = list(dirList[0])
        for lst in dirList[1:]:
            pool = [tuple(list(e if isinstance(e, tuple) else (e,)) + [d]) for e in pool for d in lst]
        return pool


class SymmetricTensorField(TensorField):
    """Symmetric rank-2 field storing the 6 sorted components; (j, i) reads (i, j)."""

    def __init__(self, gridShape, components=None, rank=2, directions=None, kspace=False, allocator=None):
        if components is None:
            components = [('x', 'x'), ('x', 'y'), ('x', 'z'), ('y', 'y'), ('y', 'z'), ('z', 'z')]
        else:
            components = sorted({tuple(sorted(c)) for c in components})
        Field.__init__(self, gridShape, components, kspace=kspace, allocator=allocator)

    def __getitem__(self, index):
        return Field.__getitem__(self, tuple(sorted(index)))

    def __setitem__(self, index, value):
        Field.__setitem__(self, tuple(sorted(index)), value)


def from_stack(gridShape, arr, components=None):
    """TensorField whose component i is arr[i]."""
    f = TensorField(gridShape, components=components, allocator=NoneAllocator)
    return f.load_stack(arr)
