"""Observers called after every step (reference: Plasticity/Observers/Observer.py L7-104)."""
import pickle
import sys

import numpy


class Observer:
    def __init__(self):
        pass

    def Update(self, time=None, state=None):
        pass


class RecallStateObserver(Observer):
    def __init__(self):
        self.state = None

    def Update(self, time, state):
        self.state = state


class RecordStateObserver(Observer):
    """Pickles (time, state) pairs; the state pickles its host field."""

    def __init__(self, filename=None, mode='wb'):
        self.file = open(filename, mode) if filename is not None else sys.stdout.buffer

    def Update(self, time, state):
        pickle.dump(time, self.file, protocol=2)
        pickle.dump({'gridShape': state.gridShape, 'mu': state.mu, 'nu': state.nu,
                     'field': state.GetOrderParameterField().stack()}, self.file, protocol=2)
        self.file.flush()


class RecordStateObserverRaw(Observer):
    """Raw frames [t][9 components in sorted order, each C-order over the grid] as float64
    (Observer.py L51-69)."""

    def __init__(self, filename=None, mode='wb'):
        self.file = open(filename, mode) if filename is not None else sys.stdout.buffer

    def Update(self, time, state):
        self.file.write(numpy.array([time]).astype('float').tobytes())
        field = state.GetOrderParameterField()
        for c in field.components:
            self.file.write(numpy.asarray(field.data[c], dtype=numpy.float64).tobytes())
        self.file.flush()


class VerboseTimestepObserver(Observer):
    def Update(self, time, state):
        print("t = %f" % time)


class VerboseTotalEnergyObserver(Observer):
    def Update(self, time, state):
        print("Total Energy = %f" % numpy.sum(state.CalculateElasticEnergy()))
        print("t = %f" % time)


class EnergyDownhillObserver(Observer):
    """Counts steps where the elastic energy rises (Observer.py L89-104)."""

    def __init__(self):
        self.PreviousEnergy = None
        self.countTotal = 0
        self.countBad = 0

    def Update(self, time, state):
        Energy = float(numpy.sum(state.CalculateElasticEnergy()))
        self.countTotal += 1
        if self.PreviousEnergy is not None and self.PreviousEnergy < Energy:
            self.countBad += 1
        print("%d/%d" % (self.countBad, self.countTotal))
        self.PreviousEnergy = Energy
