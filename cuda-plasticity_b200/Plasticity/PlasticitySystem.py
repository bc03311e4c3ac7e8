"""PlasticitySystem (reference: Plasticity/PlasticitySystem.py L3-21)."""


class PlasticitySystem:
    """Holds the state, mover, dynamics and observers; Run delegates to the mover."""

    def __init__(self, gridShape, state, mover, dynamics, observers=None):
        self.gridShape = gridShape
        self.state = state
        self.mover = mover
        self.dynamics = dynamics
        self.observers = [] if observers is None else observers

    def Run(self, startTime=0.0, endTime=10.0, fixedTimeStep=None):
        self.mover.Run(self.state, self.observers, self.dynamics, startTime, endTime,
                       fixedTimeStep=fixedTimeStep)
