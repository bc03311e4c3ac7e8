"""The reference CUDA solver's file formats through libcdd on the GPU: layout conversion against
the oracle (non-cubic grids, both precisions, an instance inside a batch), .ics and .plas files
against the reference's own convertStateToCUDA / LoadStateRaw outputs (io_formats.npz), restart
from the last frame, and the facade helpers."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import cdd
import cdd_oracle as O
from conftest import golden_path

pytestmark = pytest.mark.gpu

G = np.load(golden_path("io_formats"))


@pytest.mark.parametrize("shape", [(16, 12, 8), (24, 16)])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_export_import_match_oracle(shape, prec):
    f = np.random.default_rng(5).standard_normal((9,) + shape)
    # the instance under test sits second in a batch, after one of another shape
    plan = cdd.Plan([cdd.Instance((12, 12, 12)), cdd.Instance(shape)], prec)
    beta = plan.pack([np.zeros((9, 12, 12, 12)), f])
    fp = plan.field_view(beta, 1).cpu().numpy()          # the plan's values (FP32: rounded)
    for fprec, dt in (("f64", np.float64), ("f32", np.float32)):
        ex = plan.export_field(beta, 1, fprec).cpu().numpy()
        assert ex.dtype == dt and np.array_equal(ex, O.to_file_layout(fp).astype(dt)), fprec
    for dt in (np.float64, np.float32):
        src = torch.as_tensor(O.to_file_layout(f).astype(dt)).cuda()
        b2 = torch.zeros_like(beta)
        plan.import_field(src, b2, 1)
        want = torch.as_tensor(f.astype(dt)).to(plan.dtype)
        assert torch.equal(plan.field_view(b2, 1).cpu(), want)
        assert not plan.field_view(b2, 0).any()          # the other instance is untouched


@pytest.mark.parametrize("key", ["3d", "2d"])
def test_ics_and_plas_files_match_reference(key, tmp_path):
    fields, times = G["fields_" + key], G["times_" + key]
    shape = fields.shape[2:]
    plan = cdd.Plan([cdd.Instance(shape)], "f64")
    ics = os.path.join(tmp_path, "init.ics")
    beta = plan.pack([fields[0]])
    plan.write_ics(ics, beta)
    with open(ics, "rb") as f:
        assert f.read() == G["ics_" + key].tobytes()
    assert torch.equal(plan.read_ics(ics), beta)
    for dt, prec in (("float64", "f64"), ("float32", "f32")):
        path = os.path.join(tmp_path, "run_%s.plas" % dt)
        for t, f in zip(times, fields):
            plan.append_plas(path, t, plan.pack([f]), precision=prec)
        with open(path, "rb") as f:
            assert f.read() == G["plas_%s_%s" % (key, dt)].tobytes()
        assert plan.plas_frames(path, precision=prec) == 3
        for tag, frame in (("last", -1), ("t015", 1)):
            t, b = plan.read_plas(path, frame=frame, precision=prec)
            assert t == G["load_%s_%s_%s_t" % (key, dt, tag)][0]
            assert np.array_equal(plan.field_view(b, 0).cpu().numpy(), G["load_%s_%s_%s" % (key, dt, tag)])
        with pytest.raises(cdd.CDDError):
            plan.read_plas(path, frame=3, precision=prec)
    with pytest.raises(cdd.CDDError):
        plan.read_ics(os.path.join(tmp_path, "missing.ics"))


@pytest.mark.parametrize("prec,fprec", [("f64", "f64"), ("f32", "f64"), ("f32", "f32")])
def test_restart_from_last_frame(prec, fprec, tmp_path):
    """An FP64 file holds the state and the time exactly: the restarted run continues bitwise. An
    FP32 file keeps the time as float32 (the solver's data_type tag, as in the reference's FP32
    build), so the continuation starts at float32(t) and agrees to rounding."""
    from cdd.initial import gaussian_random_field
    shape = (16, 16, 16)
    inst = cdd.Instance(shape, load_rate=(-0.025, -0.025, 0.05))
    f = gaussian_random_field(shape, 0.06, 0.05, 31)
    path = os.path.join(tmp_path, "run.plas")
    a_plan = cdd.Plan([inst], prec)
    a = a_plan.pack([f])
    a_plan.set_time(0.0, 1e30)
    a_plan.run(a, 4, graph=False)
    t4 = a_plan.get_time()[0][0]
    a_plan.append_plas(path, 0.0, a, precision=fprec)   # an earlier frame: the restart takes the last
    a_plan.append_plas(path, t4, a, precision=fprec)
    a4 = a.clone()
    a_plan.run(a, 3, graph=False)
    b_plan = cdd.Plan([inst], prec)
    b_plan.set_time(0.0, 1e30)
    t, b = b_plan.restart_from_plas(path, precision=fprec)
    t_file = t4 if fprec == "f64" else float(np.float32(t4))
    assert t == t_file and b_plan.get_time()[0][0] == t_file
    assert torch.equal(b, a4)
    b_plan.run(b, 3, graph=False)
    if fprec == "f64":
        assert torch.equal(a, b)
        assert b_plan.get_time()[0][0] == a_plan.get_time()[0][0]
    else:
        assert (torch.linalg.norm((a - b).double()) / torch.linalg.norm(a.double())).item() < 1e-6


def test_facade_convertStateToCUDA_and_plas_observer(tmp_path):
    from Plasticity.Fields import Fields
    from Plasticity.FieldInitializers import FieldInitializer
    from Plasticity.PlasticityStates import PlasticityState
    from Plasticity import RunCUDA
    fields, times = G["fields_3d"], G["times_3d"]
    shape = fields.shape[2:]
    st = PlasticityState.PlasticityState(shape, mu=1.0, nu=0.3)
    st.betaP = Fields.from_stack(shape, fields[0])
    ics = os.path.join(tmp_path, "init.ics")
    RunCUDA.convertStateToCUDA(st, ics)
    with open(ics, "rb") as f:
        assert f.read() == G["ics_3d"].tobytes()
    # the .ics is a time-less frame: LoadStateRaw(hastimes=False) reads it back
    _, back = FieldInitializer.LoadStateRaw(ics, shape[0], 3, hastimes=False)
    assert np.array_equal(np.stack([np.asarray(back.betaP[c]) for c in O.COMPONENTS]), fields[0])
    plas = os.path.join(tmp_path, "run.plas")
    obs = RunCUDA.RecordStateObserverPlas(plas)
    for t, f in zip(times, fields):
        s = PlasticityState.PlasticityState(shape, mu=1.0, nu=0.3)
        s.betaP = Fields.from_stack(shape, f)
        obs.Update(t, s)
    with open(plas, "rb") as f:
        assert f.read() == G["plas_3d_float64"].tobytes()
    s2 = PlasticityState.PlasticityState(shape, mu=1.0, nu=0.3)
    t = RunCUDA.LoadStateCUDA(plas, s2, frame=1)
    assert t == times[1]
    assert np.array_equal(s2.GetOrderParameterField().stack(), fields[1])
