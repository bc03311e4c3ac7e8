"""State loaders and savers (reference: Plasticity/FieldInitializers/FieldInitializer.py L18-103, L363-368)."""
import numpy

from Plasticity.GridArray import GridArray
from Plasticity.PlasticityStates import PlasticityState

_INDEX = {('x', 'x'): (0, 0), ('x', 'y'): (0, 1), ('x', 'z'): (0, 2),
          ('y', 'x'): (1, 0), ('y', 'y'): (1, 1), ('y', 'z'): (1, 2),
          ('z', 'x'): (2, 0), ('z', 'y'): (2, 1), ('z', 'z'): (2, 2)}


def ReformatState(state):
    field = state.GetOrderParameterField()
    for comp in field.components:
        field[comp] = GridArray.GridArray(field[comp])
    return state


def LoadStateRaw(filename, N, dim, time=None, dtype='float64', hastimes=True):
    """Frame of a raw [t][3 x 3 x N^dim] file (FieldInitializer.py L61-103).

    As in the reference, the data of each component is taken to be stored with the first axis
    fastest (the CUDA solver's layout) and is transposed on read. Returns (t, state).
    """
    dtype = numpy.dtype(dtype)
    elemsize = dtype.itemsize
    datasize = 9 * (N ** dim)
    f = open(filename, 'rb') if isinstance(filename, str) else filename
    f.seek(0, 2)
    cnt = int(f.tell() / (elemsize * (datasize + 1)))
    f.seek(0, 0)
    t = 0
    if hastimes:
        if time is None:
            f.seek((cnt - 1) * (elemsize * (datasize + 1)), 0)
            t = numpy.frombuffer(f.read(elemsize), dtype=dtype)
        else:
            for i in range(cnt):
                f.seek(i * (elemsize * (datasize + 1)), 0)
                t = numpy.frombuffer(f.read(elemsize), dtype=dtype)
                if t >= time:
                    break
    gridShape = tuple([N] * dim)
    state = PlasticityState.PlasticityState(gridShape)
    field = state.GetOrderParameterField()
    data = numpy.frombuffer(f.read(elemsize * datasize), dtype=dtype).reshape(tuple([3, 3] + list(gridShape)))
    tp = list(range(dim))[::-1]
    for c in field.components:
        field[c] = numpy.copy(data[_INDEX[c]].transpose(tp))
    state = ReformatState(state)
    return t, state


def SaveNumpyFileFromState(state, filename):
    field = state.GetOrderParameterField()
    numpy.array([numpy.asarray(field[c]) for c in field.components]).tofile(filename)
