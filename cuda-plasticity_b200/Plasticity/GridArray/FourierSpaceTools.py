"""k-space tables on the rfft half grid (reference: Plasticity/GridArray/FourierSpaceTools.py L5-59).

kx, ky, kz, kSq, kSqSq and kmask with the reference's conventions: angles above pi wrap by -2 pi
(+pi kept at the Nyquist index), 3-D axes scale by their own size, 2-D axes by gridShape[1].
"""
import numpy

from Plasticity.GridArray import GridArray
from Plasticity.Constants import x, y, z


def identity(a):
    return a - 2 * numpy.pi * (a > numpy.pi).astype(float)


class NumpyFourierSpaceTools:
    def __init__(self, gridShape, func=identity):
        self.dimension = len(gridShape)
        ax = lambda scale, n, count: scale * func(2. * numpy.pi * numpy.arange(count, dtype=float) / float(n))
        if self.dimension == 1:
            n0 = gridShape[0]
            self.gridShape = (n0 // 2 + 1,)
            self.kz = GridArray.GridArray(ax(n0, n0, n0 // 2 + 1))
            self.kx = GridArray.GridArray.zeros(self.gridShape)
            self.ky = GridArray.GridArray.zeros(self.gridShape)
            self.kSq = self.kz * self.kz
            self.kmask = GridArray.GridArray(numpy.arange(n0 // 2 + 1) != 0).astype(float)
        elif self.dimension == 2:
            n0, n1 = gridShape
            self.gridShape = [n0, n1 // 2 + 1]
            self.kx = GridArray.GridArray(numpy.broadcast_to(ax(n1, n0, n0)[:, None], self.gridShape))
            self.ky = GridArray.GridArray(numpy.broadcast_to(ax(n1, n1, n1 // 2 + 1)[None, :], self.gridShape))
            self.kz = GridArray.GridArray.zeros(self.gridShape)
            self.kxkx, self.kxky, self.kyky = self.kx * self.kx, self.kx * self.ky, self.ky * self.ky
            self.kSq = self.kxkx + self.kyky
            m = numpy.ones(self.gridShape)
            m[0, 0] = 0.
            self.kmask = GridArray.GridArray(m)
        else:
            n0, n1, n2 = gridShape
            self.gridShape = [n0, n1, n2 // 2 + 1]
            sh = self.gridShape
            self.kx = GridArray.GridArray(numpy.broadcast_to(ax(n0, n0, n0)[:, None, None], sh))
            self.ky = GridArray.GridArray(numpy.broadcast_to(ax(n1, n1, n1)[None, :, None], sh))
            self.kz = GridArray.GridArray(numpy.broadcast_to(ax(n2, n2, n2 // 2 + 1)[None, None, :], sh))
            self.kxkx, self.kyky, self.kzkz = self.kx * self.kx, self.ky * self.ky, self.kz * self.kz
            self.kxky, self.kykz, self.kxkz = self.kx * self.ky, self.ky * self.kz, self.kx * self.kz
            self.kSq = self.kxkx + self.kyky + self.kzkz
            m = numpy.ones(sh)
            m[0, 0, 0] = 0.
            self.kmask = GridArray.GridArray(m)
        self.kSqSq = self.kSq * self.kSq
        self.k = {x: self.kx, y: self.ky, z: self.kz}


FourierSpaceTools = NumpyFourierSpaceTools
