"""File helpers of the reference's CUDA pipeline (Plasticity/RunCUDA.py L9-22).

The reference's CUDA solver reads an .ics initial condition and writes .plas frame series (see
include/cdd.h, cdd_ics_read ... cdd_plas_read). Here the layout conversion runs on the GPU through
libcdd; the run itself stays in this process (cdd.Plan), so the header generation, make and
separate-process launch of the reference's RunCUDA driver have no counterpart.
"""
from Plasticity.FieldDynamics.engine import plan_for
from Plasticity.Observers.Observer import Observer


def convertStateToCUDA(state, filename):
    """Write the state's beta^P as an .ics file: float64, the 9 components in sorted order, each
    with grid axis 0 fastest (RunCUDA.py L9-22). States with a vacancy component are not
    supported."""
    plan = plan_for(state.gridShape, state.mu, state.nu, precision="f64")
    plan.write_ics(filename, plan.pack_state(state))


def LoadStateCUDA(filename, state, frame=-1, dtype='float64'):
    """Frame `frame` (default: the last, the restart state) of a .plas file into `state`, which
    gives the grid and material; returns the frame time. The frame is read through the GPU; for
    a host-only read use FieldInitializer.LoadStateRaw."""
    prec = {'float64': 'f64', 'float32': 'f32'}[str(dtype)]
    plan = plan_for(state.gridShape, state.mu, state.nu, precision="f64")
    t, beta = plan.read_plas(filename, frame=frame, precision=prec)
    state._set_device(plan.field_view(beta, 0).clone())
    return t


class RecordStateObserverPlas(Observer):
    """Appends each observed state as a .plas frame [t][field] in the CUDA solver's layout
    (assist.h L164-192), so FieldInitializer.LoadStateRaw and LoadStateCUDA read it back."""

    def __init__(self, filename, dtype='float64'):
        self.filename = filename
        self.prec = {'float64': 'f64', 'float32': 'f32'}[str(dtype)]

    def Update(self, time, state):
        plan = plan_for(state.gridShape, state.mu, state.nu, precision="f64")
        plan.append_plas(self.filename, time, plan.pack_state(state), precision=self.prec)
