"""Benchmark of the CDD time step on B200: cell-stage updates per second.

Workload (per GPU): one 3-D 256^3 periodic grid, seeded Gaussian random field (sigma 0.03 L,
rms 0.05), mu = 1, nu = 0.3, applied strain rate diag(-0.025, -0.025, 0.05), glide and climb,
adaptive TVD-RK3 at CFL 0.25. The headline value is the FP32 form (FP64 CFL maximum, energy /
mean-strain sums and k = 0 mode); the plain FP64 form is measured beside it on the same input,
together with the FP32-vs-FP64 field error after 10 steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cdd|reference]

One cell-stage update = one cell through one RK3 stage (stress solve + flux + stage update);
value = cells x 3 x steps / time. Under torchrun each rank advances its own independent grid
(replicas; no data-path collective) and the time is the maximum over ranks.
``--impl reference`` times the CPU oracle (a numpy restatement of the reference's Python path)
on the host cores instead.
"""
import argparse
import json
import os
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "cuda-plasticity_b200"))

METRIC = "cell-stage updates/s at 256³: FP32 batched vs FP64 plain (≤1e-5 rel-L2); adj/fwd"
UNIT = "cell-stage updates/s"
WORDS_PER_CELL_STAGE = 48      # stress operator: read 9 + write 6; stencil + stage: read 24, write 9
STRESS_WORDS = 15               # stress operator: read beta 9, write sigma 6
FLUX_WORDS = 24                 # stencil, flux form: read beta 9 + sigma 6, write rhs 9
FLUX_TRAFFIC_BYTES_PER_CELL = 94.9    # DRAM bytes per cell of the flux-form stencil (ncu, 192^3)
# executed FP32 operations (add + mul + 2 fma, packed pairs counted per lane) and warp instructions
# per cell of the FP32 flux-form stencil, from ncu's instruction counters at 192^3
FLUX_FLOP_PER_CELL = 1308.6
FLUX_WARP_INST_PER_CELL = 39.60
FLUX_COUNTS_SOURCE = "profiles/k_stencil_flux_192cube_fp32.md"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cdd", choices=["cdd", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=96,
                    help="grid of the CPU baseline sample (one step on one core; 96^3 takes about 30 s, "
                         "128^3 about 80 s)")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="use the built-in launch shapes")
    ap.add_argument("--precision-steps", type=int, default=200,
                    help="steps of the FP32-vs-FP64 precision study (config 3: 200)")
    ap.add_argument("--clocks-csv", default=os.environ.get("CDD_BENCH_CLOCKS_CSV"),
                    help="file for the raw nvidia-smi samples of the timed region (default: none; "
                         "the environment variable CDD_BENCH_CLOCKS_CSV may give it)")
    ap.add_argument("--only-flux", nargs="?", const="f32", default=None, choices=["f32", "f64"],
                    help="run three flux evaluations of the workload at the given precision and exit "
                         "(for profiling the stencil)")
    ap.add_argument("--only-step", nargs="?", const="f32", default=None, choices=["f32", "f64"],
                    help="run three adaptive steps of the workload (eager launches) at the given precision and "
                         "exit (for the per-kernel launch list)")
    ap.add_argument("--only-vjp", action="store_true",
                    help="run three FP32 flux VJPs (cdd_flux_vjp) of the workload and exit (for profiling "
                         "the adjoint kernels)")
    return ap.parse_args()


def ensemble_instances(seed):
    """The 96-instance ensemble: 16 each of 256^2, 512^2, 48^3, 64^3, 96^3, 128^3 (58,916,864 cells
    per stage); sigma ~ U[0.02, 0.08] L, traceless strain rate with rate_zz ~ U[0, 0.1]."""
    import numpy as np
    import cdd
    rng = np.random.default_rng(seed)
    shapes = [(256, 256), (512, 512), (48, 48, 48), (64, 64, 64), (96, 96, 96), (128, 128, 128)]
    out = []
    for sh in shapes:
        for _ in range(16):
            sig = float(rng.uniform(0.02, 0.08))
            r = float(rng.uniform(0.0, 0.1))
            out.append((sh, sig, int(rng.integers(1 << 30)),
                        cdd.Instance(sh, mu=1.0, nu=0.3, cfl=0.25, load_rate=(-0.5 * r, -0.5 * r, r))))
    return out


def run_ensemble(dev, K, W, seed, tuning, barrier, max_over_ranks):
    """The 96-instance FP32 ensemble, sharded over the ranks (cdd.ensemble.ShardedEnsemble: greedy
    bin packing on cells, one batched plan per rank, no data-path collective; N = 1 is one plan
    over all instances). Each rank's stage is one launch per kernel over its instances, with
    per-instance dt and the whole step in a CUDA graph. value = all instances' cell-stages / the
    slowest rank's time (CUDA events on the launching stream)."""
    import torch
    from cdd.ensemble import ShardedEnsemble
    from cdd.initial import gaussian_random_field_torch
    spec = ensemble_instances(seed)
    ens = ShardedEnsemble([s[3] for s in spec], "f32", tuning=tuning)
    ens.load(lambda i: gaussian_random_field_torch(spec[i][0], spec[i][1], 0.05, spec[i][2], device=dev))
    ens.set_time(0.0)
    ens.run(W)
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(st)
    ens.run(K)
    e1.record(st)
    barrier()
    el = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    ens.check_status()
    table = ens.observables()            # (t, energy, mean_zz) of all 96 instances, one all-reduce
    cells = ens.total_cells
    dts = table[:, 0] / (W + K)
    return {"value": cells * 3 * K / el, "unit": UNIT, "ms_per_step": 1e3 * el / K, "steps": K,
            "instances": len(spec), "cells_per_stage": cells, "dtype": "f32",
            "ranks": ens.world, "cells_per_rank_max": int(max_over_ranks(float(ens.local_cells))),
            "dt_range": [float(dts.min()), float(dts.max())],
            "workload": "96 instances: 16 each of 256^2, 512^2, 48^3, 64^3, 96^3, 128^3; sigma U[0.02,0.08] L, "
                        "rate_zz U[0,0.1] traceless; sharded over the ranks, one plan and one CUDA graph per "
                        "step per rank"}


def run_adjoint(dev, seed, tuning):
    """Adjoint cost: 64^3 FP32, 200 fixed-dt steps (dt from the step-0 CFL 0.25), checkpoints every
    20 steps; loss = elastic energy + 10 mean beta_zz; gradients for beta0, mu, nu, rate_zz.
    adj/fwd = reverse-sweep time (segment re-runs included) / forward time."""
    import torch
    import cdd
    from cdd.adjoint import Rollout, CZZ
    from cdd.initial import gaussian_random_field_torch
    shape = (64, 64, 64)
    b0 = gaussian_random_field_torch(shape, 0.05, 0.05, seed, device=dev)
    probe = cdd.Plan([cdd.Instance(shape, load_rate=tuple(0.05 * CZZ))], "f32")
    bp = probe.pack([b0])
    _, speed = probe.flux(bp, 0.0)
    dt = 0.25 / (64 * float(speed.max()))
    del probe, bp
    n = 200
    ro = Rollout(shape, 1.0, 0.3, 0.05, dt, n, precision="f32", checkpoint_every=20, tuning=tuning)
    beta = ro.plan.pack([b0])
    ro.forward(beta)
    ro.backward()                      # warm-up (allocations, attributes)
    st = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize()
    ev[0].record(st)
    _, loss = ro.forward(beta)
    ev[1].record(st)
    _, grads = ro.backward()
    ev[2].record(st)
    torch.cuda.synchronize()
    f = ev[0].elapsed_time(ev[1]) / 1e3
    b = ev[1].elapsed_time(ev[2]) / 1e3
    return {"value": b / f, "fwd_ms_per_step": 1e3 * f / n, "adj_ms_per_step": 1e3 * b / n,
            "steps": n, "checkpoint_every": 20, "grid": list(shape), "dtype": "f32", "loss": loss,
            "grads": {k: float(v) for k, v in grads.items()},
            "workload": "64^3 FP32 rollout, 200 fixed-dt steps, checkpoints every 20; reverse sweep = "
                        "segment re-run with step records + cdd_step_adjoint per step"}


def workload(size, seed):
    import cdd
    shape = (size, size, size)
    inst = cdd.Instance(shape, mu=1.0, nu=0.3, Lambda=0.0, cfl=0.25,
                        load_rate=(-0.025, -0.025, 0.05))
    return shape, inst


def gemm_peak_tflops(dev, dtype, n=8192, reps=5):
    """Dense GEMM throughput of cuBLAS (through torch, TF32 off) on this GPU: the measured
    CUDA-core (FP32) or FP64 peak the stencil's FLOP rate is compared with."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        a = torch.randn(n, n, device=dev, dtype=dtype)
        b = torch.randn(n, n, device=dev, dtype=dtype)
        c = torch.empty(n, n, device=dev, dtype=dtype)
        for _ in range(2):
            torch.mm(a, b, out=c)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            torch.mm(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        s = e0.elapsed_time(e1) / 1e3 / reps
        del a, b, c
        torch.cuda.empty_cache()
        return 2.0 * n ** 3 / s / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling while the GPU works."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu, path=None):
        self.gpu = gpu
        self.proc = None
        self.path = path or "/dev/null"   # raw samples are kept only when a path is given
        self.out = None

    def start(self):
        try:
            self.out = open(self.path + ".tmp" if self.path != "/dev/null" else os.devnull, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            text, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            text = ""
        rows = []
        for line in text.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), float(f[3]), f[5:9]))
            except ValueError:
                continue
        if self.path != "/dev/null":
            with open(self.path, "w") as fo:
                fo.write(text)
        if not rows:
            return None
        load = [r for r in rows if r[2] > 0.35 * max(x[2] for x in rows)] or rows
        sm = sorted(r[0] for r in load)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in load for i, v in enumerate(r[3]) if v.lower().startswith("active")})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows), "samples_under_load": len(load),
                "power_w_max": max(r[2] for r in rows)}


def cpu_baseline(sample):
    """The oracle (numpy FP64 restatement of the reference path), one step on one host thread."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import cdd_oracle as O
    from cdd.initial import gaussian_random_field
    shape = (sample,) * 3
    b = gaussian_random_field(shape, 0.03, 0.05, 7)
    p = O.Params(mu=1.0, nu=0.3, cfl=0.25, load_rate=(-0.025, -0.025, 0.05))
    t0 = time.perf_counter()
    O.rk3_step(b, 0.0, 1e30, p)
    dt = time.perf_counter() - t0
    return {"value": sample ** 3 * 3 / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "1 TVD-RK3 step of the numpy FP64 oracle at %d^3 (same physics and load), "
                      "1 thread of %d host cores, %.1f s" % (sample, os.cpu_count() or 1, dt)}


def _oracle_sample_step(args):
    sample, seed = args
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    sys.path.insert(0, os.path.join(REPO, "cuda-plasticity_b200"))
    import cdd_oracle as O
    from cdd.initial import gaussian_random_field
    b = gaussian_random_field((sample,) * 3, 0.03, 0.05, seed)
    p = O.Params(mu=1.0, nu=0.3, cfl=0.25, load_rate=(-0.025, -0.025, 0.05))
    O.rk3_step(b, 0.0, 1e30, p)
    return sample ** 3 * 3


def run_reference(args):
    """CPU arm: the oracle on all usable host cores, one sample grid per worker process."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    try:
        import psutil
        mem_gb = psutil.virtual_memory().available / 2 ** 30
    except Exception:
        mem_gb = 16.0
    # one 48^3 grid per worker and step: a 256^3 step of the oracle takes about 10 minutes on one
    # core (128^3: about 80 s), so the whole-job rate is sampled on independent 48^3 grids (about
    # 3 s per step with 16 workers), which keeps a 25-step run near a minute
    sample = 48
    workers = max(1, min(cores, int(mem_gb // 1.0), 64))
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        for w in range(args.warmup):
            pool.map(_oracle_sample_step, [(sample, 100 + i) for i in range(workers)])
        t0 = time.perf_counter()
        units = 0
        for s in range(args.steps):
            units += sum(pool.map(_oracle_sample_step, [(sample, 1000 * s + i) for i in range(workers)]))
        el = time.perf_counter() - t0
    val = units / el
    line = {"metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded Gaussian random fields, sigma 0.03 L, rms 0.05",
            "config": {"workload": "3-D CDD step, numpy FP64 oracle of the reference Python path, "
                                   "%d worker processes x one %d^3 sample grid per step" % (workers, sample),
                       "grid": [sample] * 3, "workers": workers},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": workers, "kind": "port",
                             "sample": "%d processes x 1 step of a %d^3 grid per timed step" % (workers, sample)},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import numpy as np
    import torch
    import torch.distributed as dist
    import cdd
    from cdd.initial import gaussian_random_field_torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    K, W = args.steps, max(3, args.warmup)
    shape, inst = workload(args.size, 100 + rank)
    cells = int(np.prod(shape))
    clocks = ClockSampler(local, args.clocks_csv)

    b0 = gaussian_random_field_torch(shape, 0.03, 0.05, 100 + rank, device=dev)   # FP64 on device

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
            torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed_run(plan, beta, steps):
        st = torch.cuda.current_stream()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        barrier()
        ev0.record(st)
        plan.run(beta, steps, graph=True)
        ev1.record(st)
        barrier()
        return ev0.elapsed_time(ev1) / 1e3

    if args.only_vjp:
        import ctypes
        p = cdd.Plan([inst], "f32")
        b = p.empty_field()
        b.copy_(b0.reshape(-1).to(p.dtype))
        g = torch.randn(p.field_elems, dtype=p.dtype, device=dev, generator=torch.Generator(dev).manual_seed(3))
        bb, sb = torch.zeros_like(g), p.empty_stress()
        for _ in range(3):
            rc = p.lib.cdd_flux_vjp(p.handle, ctypes.c_void_p(b.data_ptr()), 0.0, ctypes.c_void_p(g.data_ptr()),
                                    ctypes.c_void_p(bb.data_ptr()), ctypes.c_void_p(sb.data_ptr()), None,
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
            if rc != 0:
                raise RuntimeError("cdd_flux_vjp failed: %d" % rc)
        torch.cuda.synchronize()
        print(json.dumps({"only_vjp": "f32", "grid": list(shape)}))
        return

    if args.only_step:
        p = cdd.Plan([inst], args.only_step, tuning=None if args.no_tune else "auto")
        b = p.empty_field()
        b.copy_(b0.reshape(-1).to(p.dtype))
        p.set_time(0.0, 1e30)
        p.run(b, 3, graph=False)
        p.check_status()
        torch.cuda.synchronize()
        print(json.dumps({"only_step": args.only_step, "grid": list(shape), "launch_shapes": p.tuning(0)}))
        return

    if args.only_flux:
        p = cdd.Plan([inst], args.only_flux, tuning=None if args.no_tune else "auto")
        b = p.empty_field()
        b.copy_(b0.reshape(-1).to(p.dtype))
        for _ in range(3):
            p.flux(b, 0.0, want_speed=False)
        torch.cuda.synchronize()
        print(json.dumps({"only_flux": args.only_flux, "grid": list(shape), "launch_shapes": p.tuning(0)}))
        return

    clocks.start()
    # ---------------- FP32 form (headline) ----------------
    # launch shapes: the autotuner's choice for this GPU and shape (tuned before any timing)
    tuning = None if args.no_tune else "auto"
    p32 = cdd.Plan([inst], "f32", tuning=tuning)
    beta32 = p32.empty_field()
    beta32.copy_(b0.reshape(-1).to(torch.float32))
    p32.set_time(0.0, 1e30)
    p32.run(beta32, W, graph=True)
    p32_tuning = p32.tuning(0)
    el32 = max_over_ranks(timed_run(p32, beta32, K))
    p32.check_status()
    rate32 = world * cells * 3 * K / el32
    ms32 = 1e3 * el32 / K

    # per-operator times (eager launches, CUDA events on the launching stream): the stress solve
    # (cdd_stress) and the stencil kernel alone (cdd_flux_with_stress on that stress)
    st = torch.cuda.current_stream()
    M = 5
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    s6 = p32.empty_stress()
    rhs32 = p32.empty_field()
    p32.stress(beta32, out=s6)
    p32.flux(beta32, want_speed=False, sigma=s6, out=rhs32)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(M):
        p32.stress(beta32, out=s6)
    e1.record(st)
    for _ in range(M):
        p32.flux(beta32, want_speed=False, sigma=s6, out=rhs32)
    e2.record(st)
    torch.cuda.synchronize()
    t_stress = e0.elapsed_time(e1) / 1e3 / M
    t_stencil = e1.elapsed_time(e2) / 1e3 / M
    del rhs32

    # ---------------- FP64 plain form and FP32 error ----------------
    fp64 = None
    err = None
    precision_study = None
    if not args.no_fp64:
        p64 = cdd.Plan([inst], "f64", tuning=tuning)
        beta64 = p64.empty_field()
        beta64.copy_(b0.reshape(-1))
        p64.set_time(0.0, 1e30)
        p64.run(beta64, W, graph=True)
        K64 = max(3, min(K, 10))
        el64 = max_over_ranks(timed_run(p64, beta64, K64))
        rate64 = world * cells * 3 * K64 / el64
        fp64 = {"value": rate64, "unit": UNIT, "ms_per_step": 1e3 * el64 / K64, "steps": K64}
        # config-3 precision study: the FP32 form against FP64 from the same field over
        # --precision-steps adaptive steps (each form takes its own CFL steps); per-field rel-L2 at
        # checkpoints, and the energy / mean-strain curves (observables after every step)
        beta64.copy_(b0.reshape(-1))
        beta32.copy_(b0.reshape(-1).to(torch.float32))
        p64.set_time(0.0, 1e30)
        p32.set_time(0.0, 1e30)
        # the conditioning of the dynamics itself: FP64 from the same field with every value
        # perturbed by a relative 1e-7 (about FP32 rounding), compared with the unperturbed FP64 run
        p64b = cdd.Plan([inst], "f64", tuning=tuning)
        beta64b = p64b.empty_field()
        gen = torch.Generator(dev).manual_seed(11)
        beta64b.copy_(b0.reshape(-1) * (1.0 + 1e-7 * torch.randn(b0.numel(), dtype=torch.float64, device=dev,
                                                                   generator=gen)))
        p64b.set_time(0.0, 1e30)
        n_prec = max(10, args.precision_steps)
        marks = sorted({m for m in (10, 50, 100, 200, n_prec) if m <= n_prec})
        e64, m64 = p64.observables(beta64)
        e32, m32 = p32.observables(beta32)
        curve64, curve32 = [(e64[0], m64[0])], [(e32[0], m32[0])]
        at_marks = {}
        for n in range(1, n_prec + 1):
            p64.run(beta64, 1, graph=True)
            p32.run(beta32, 1, graph=True)
            p64b.run(beta64b, 1, graph=True)
            e64, m64 = p64.observables(beta64)
            e32, m32 = p32.observables(beta32)
            curve64.append((e64[0], m64[0]))
            curve32.append((e32[0], m32[0]))
            if n in marks:
                a = beta64.view(9, -1)
                b = beta32.view(9, -1).to(torch.float64)
                rels = ((a - b).norm(dim=1) / a.norm(dim=1)).cpu().numpy()
                relp = ((a - beta64b.view(9, -1)).norm(dim=1) / a.norm(dim=1)).cpu().numpy()
                at_marks[str(n)] = {"per_field_rel_l2_max": float(rels.max()),
                                    "fp64_perturbed_1e-7_rel_l2_max": float(relp.max()),
                                    "per_field_rel_l2": [float(x) for x in rels],
                                    "energy_rel": float(abs(e32[0] - e64[0]) / abs(e64[0])),
                                    "mean_zz_abs": float(abs(m32[0] - m64[0]))}
        p64.check_status()
        p32.check_status()
        p64b.check_status()
        del p64b, beta64b
        t64, _, _ = p64.get_time()
        t32, _, _ = p32.get_time()
        c64 = np.array(curve64)
        c32 = np.array(curve32)
        err = dict(at_marks["10"])
        precision_study = {
            "steps": n_prec, "grid": list(shape),
            "per_field_rel_l2_at_step": at_marks,
            "energy_curve_max_rel": float(np.max(np.abs(c32[:, 0] - c64[:, 0]) / np.abs(c64[:, 0]))),
            "mean_zz_curve_max_abs": float(np.max(np.abs(c32[:, 1] - c64[:, 1]))),
            "mean_zz_curve_max_rel": float(np.max(np.abs(c32[:, 1] - c64[:, 1])) / np.max(np.abs(c64[:, 1]))),
            "t_final_fp64": float(t64[0]), "t_final_fp32": float(t32[0]),
            "note": "each form takes its own CFL steps (FP64 speed maximum in both), so the curves are "
                    "compared step by step and the times differ by the accumulated dt difference; "
                    "fp64_perturbed_1e-7 is the FP64 run from the field perturbed by a relative 1e-7 per value, "
                    "the growth the dynamics gives any rounding-sized difference"}
        del p64, beta64

    # ---------------- end to end: host buffers through the public API ----------------
    # every step copies its input in from pinned host memory and its result back (cdd.HostPipeline:
    # the copies of neighbouring steps overlap the computation on separate streams; three device
    # fields, so that the copy-in of step k + 1 need not wait for the copy-out of step k - 1)
    D = 3
    host_in = torch.empty(p32.field_elems, dtype=torch.float32, pin_memory=True)
    host_in.copy_(b0.reshape(-1).to(torch.float32).cpu())
    host_outs = [torch.empty_like(host_in, pin_memory=True) for _ in range(D)]
    p32.set_time(0.0, 1e30)
    pipe = cdd.HostPipeline(p32, depth=D)
    Ke = max(3, K)
    for k in range(D):
        pipe.step(host_in, host_outs[k % D])
    pipe.synchronize()
    barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev0.record(pipe.s_in)
    for k in range(Ke):
        if k >= D:
            pipe.wait(pipe.count - D)          # its host output buffer is about to be reused
        last = pipe.step(host_in, host_outs[k % D])
    ev1 = torch.cuda.Event(enable_timing=True)
    ev1.record(pipe.s_out)                     # after the last copy-out (stream order)
    pipe.synchronize()
    barrier()
    ele = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    # the PCIe floor of that loop: the same copies alone, both directions at once on the pipeline's
    # copy streams (no steps)
    bufs = pipe.bufs
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(pipe.s_in)
    pipe.s_out.wait_event(c0)
    for k in range(Ke):
        with torch.cuda.stream(pipe.s_in):
            bufs[k % D].copy_(host_in, non_blocking=True)
        with torch.cuda.stream(pipe.s_out):
            host_outs[k % D].copy_(bufs[(k + 1) % D], non_blocking=True)
    pipe.s_in.wait_stream(pipe.s_out)
    c1.record(pipe.s_in)
    torch.cuda.synchronize()
    copies_ms = c0.elapsed_time(c1) / Ke
    e2e = {"value": world * cells * 3 * Ke / ele, "unit": UNIT,
           "h2d_bytes_per_step": host_in.numel() * 4, "d2h_bytes_per_step": host_outs[0].numel() * 4,
           "ms_per_step": 1e3 * ele / Ke, "copies_only_ms_per_step": copies_ms,
           "pcie_gb_s_each_way": host_in.numel() * 4 / copies_ms / 1e6,
           "path": "cdd.HostPipeline (3 device fields): cdd.Plan.step on a field copied in from pinned host "
                   "memory and copied back every step, copies overlapped with the neighbouring steps' "
                   "computation; copies_only = the same copies with no steps (the PCIe floor)"}
    del pipe
    clk = clocks.stop()

    adj = None
    ens = None
    if world == 1 and not args.no_adjoint:
        adj = run_adjoint(dev, 5, tuning)
    if not args.no_ensemble:
        ens = run_ensemble(dev, max(3, min(K, 5)), W, 2024, tuning, barrier, max_over_ranks)

    if world > 1:
        dist.barrier()
        del p32
        dist.destroy_process_group()
    if rank != 0:
        return

    peak, peak_kind = peaks()
    fp32_peak = gemm_peak_tflops(dev, torch.float32)
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    issue_peak = nsm * 4 * (clk.get("sm_mhz") or 1965.0) * 1e6 / 1e9   # warp instructions per ns
    issue_ach = FLUX_WARP_INST_PER_CELL * cells / t_stencil / 1e9
    stage_s = el32 / K / 3
    achieved = WORDS_PER_CELL_STAGE * 4 * cells / stage_s / 1e9
    # per stage: the stress solve (fused plane passes: forward, mean, k-space, inverse; else six
    # passes incl. the mean) and the stencil; per step: k_dt and, unless the plane passes form F0,
    # the F0 axpy
    plane = p32_tuning.get("plane_fft") == 1
    launches_per_step = 3 * ((4 if plane else 6) + 1) + (1 if plane else 2)
    line = {
        "metric": METRIC, "value": rate32, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic: seeded Gaussian random field per rank (sigma 0.03 L, rms 0.05), generated on device",
        "config": {"workload": "3-D %d^3 CDD step, FP32 form, 1 instance per GPU" % args.size,
                   "grid": list(shape), "mu": 1.0, "nu": 0.3, "cfl": 0.25, "Lambda": 0.0,
                   "strain_rate": [-0.025, -0.025, 0.05], "parallelism": "replicas x%d" % world,
                   "l2": "inputs larger than L2 (FP32 field %.0f MB)" % (9 * cells * 4 / 1e6),
                   "timing": "CUDA graph of whole steps, CUDA events, max over ranks",
                   "launch_shapes": p32_tuning},
        # dominant kernel: k_stencil (≈47% of a step in the launch list), timed alone here in its
        # flux form; algorithmic bytes per launch = 24 words per cell (read beta 9 + stress 6,
        # write rhs 9); traffic = DRAM bytes per cell from one ncu capture at 192^3, scaled by cells
        "roofline": {"bound": "hbm", "kernel": "k_stencil (flux evaluation, cdd_flux_with_stress)",
                     "achieved": FLUX_WORDS * 4 * cells / t_stencil / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": FLUX_WORDS * 4 * cells / t_stencil / 1e9 / peak, "peak_kind": peak_kind,
                     "launch_ms": 1e3 * t_stencil,
                     "algorithmic_bytes_per_launch": FLUX_WORDS * 4 * cells,
                     "traffic": FLUX_TRAFFIC_BYTES_PER_CELL * cells,
                     "traffic_source": "profiles/k_stencil_flux_192cube_fp32.md (%.1f B/cell at 192^3, scaled)" % FLUX_TRAFFIC_BYTES_PER_CELL,
                     "flop": {"bound": "fp32", "flop_per_cell": FLUX_FLOP_PER_CELL,
                              "achieved": FLUX_FLOP_PER_CELL * cells / t_stencil / 1e12, "peak": fp32_peak,
                              "unit": "TFLOP/s", "frac": FLUX_FLOP_PER_CELL * cells / t_stencil / 1e12 / fp32_peak,
                              "peak_kind": "measured: cuBLAS FP32 GEMM (TF32 off), 8192^3, this run",
                              "counts_source": FLUX_COUNTS_SOURCE},
                     "issue": {"warp_inst_per_cell": FLUX_WARP_INST_PER_CELL, "achieved_ginst_s": issue_ach,
                               "peak_ginst_s": issue_peak, "frac": issue_ach / issue_peak,
                               "peak_kind": "4 warp instructions per cycle per SM at the median SM clock of the run"},
                     "step": {"achieved": achieved, "frac": achieved / peak,
                              "algorithmic_bytes_per_cell_stage": WORDS_PER_CELL_STAGE * 4},
                     "per_operator": {
                         "stress_fft": {"ms": 1e3 * t_stress, "GBps": STRESS_WORDS * 4 * cells / t_stress / 1e9},
                         "stencil_flux": {"ms": 1e3 * t_stencil,
                                          "GBps": FLUX_WORDS * 4 * cells / t_stencil / 1e9}}},
        "gpu_launches": launches_per_step * K,
        "e2e": e2e,
        "clocks": clk,
        "fp64_plain": fp64,
        "fp32_over_fp64": (rate32 / fp64["value"]) if fp64 else None,
        "fp32_error_10_steps": err,
        "precision_study": precision_study,
        "adj_over_fwd": adj["value"] if adj else None,
        "adjoint": adj,
        "ensemble_96": ens,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.cpu_sample)
    print(json.dumps(line))


if __name__ == "__main__":
    main()
