"""State initializers, loaders and savers (reference: Plasticity/FieldInitializers/FieldInitializer.py
L18-103, L153-209, L363-368, L421-442).

These run on the host once per simulation, before any step: the random initial condition is drawn
from numpy's legacy global generator so that a seed gives the reference's field bit for bit, and the
state is uploaded to the GPU on its first step.
"""
import numpy

from Plasticity.GridArray import FourierSpaceTools
from Plasticity.GridArray import GridArray
from Plasticity.PlasticityStates import PlasticityState
from Plasticity.PlasticityStates import VacancyState

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


def ResampleArray(arr, N, Dim=2):
    """Fourier resampling of every axis to N points (FieldInitializer.py L421-428), by
    scipy.signal.resample, the routine the reference calls."""
    from scipy import signal
    out = numpy.asarray(arr)
    for axis in range(Dim):
        out = signal.resample(out, N, axis=axis)
    return out


def ResizeState(state, N, Dim=2):
    """A new state of the same class on an N^Dim grid with every component of the order-parameter
    field Fourier-resampled (FieldInitializer.py L430-442). As in the reference the new state is
    built with the class's default constructor arguments."""
    newstate = state.__class__(tuple([N] * Dim))
    field = state.GetOrderParameterField()
    newfield = newstate.GetOrderParameterField()
    for component in field.components:
        newfield[component] = ResampleArray(field[component], N, Dim)
    return newstate


def GaussianRandomInitializer(gridShape, sigma=0.2, seed=None, slipSystem=None, slipPlanes=None,
                              slipDirections=None, vacancy=None, smectic=None):
    """Random initial state (FieldInitializer.py L153-209), the one RunPython.py L161 starts from.

    Every component is drawn at 128^d (whatever the target grid, so that a seed gives the same
    physical field at every resolution) as i.i.d. normals of scale 128 from numpy's legacy global
    generator seeded with ``seed`` (0 when None), filtered in Fourier space by
    (sqrt(pi) sigma)^d exp(-k^2 sigma^2 / 4) with the reference's k tables, and transformed back;
    a grid whose first size is not 128 is then Fourier-resampled to that size on every axis
    (ResizeState). ``vacancy`` gives a VacancyState with that alpha (its concentration is drawn
    first, as it sorts first among the components). The slip-system and smectic states of the
    reference are not part of this library and raise NotImplementedError.
    """
    if slipSystem is not None or smectic is not None:
        raise NotImplementedError("GaussianRandomInitializer: slip-system and smectic states are not built")
    oldgrid = tuple(gridShape)
    dim = len(oldgrid)
    if dim not in (1, 2, 3):
        raise ValueError("GaussianRandomInitializer: 1, 2 or 3 dimensions")
    grid = (128,) * dim
    if vacancy is not None:
        state = VacancyState.VacancyState(grid, alpha=vacancy)
    else:
        state = PlasticityState.PlasticityState(grid)
    field = state.GetOrderParameterField()
    numpy.random.seed(0 if seed is None else seed)
    Ksq = numpy.asarray(FourierSpaceTools.FourierSpaceTools(grid).kSq)
    filt = (numpy.sqrt(numpy.pi) * sigma) ** dim
    for component in field.components:
        temp = numpy.random.normal(scale=grid[0], size=grid)
        ktemp = numpy.fft.rfftn(temp) * filt * numpy.exp(-Ksq * sigma ** 2 / 4.)
        field[component] = numpy.real(numpy.fft.irfftn(ktemp))
    if oldgrid[0] != 128:
        state = ResizeState(state, oldgrid[0], Dim=dim)
    return ReformatState(state)
