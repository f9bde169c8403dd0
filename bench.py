"""Benchmark of the B200 backend for VILMA v2's viscoelastic time step.

One step = one solid_earth_update interval (dt of the workload, with its
Maxwell-CFL sub-steps) of the seeded synthetic workload, driven through the
C-ABI. Prints one JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload NAME]

--workload c4_ensemble times the batched ensemble (32 instances advanced
together through vg_update_batch) against the same instances run one after
the other.

Multi-GPU: instances are independent (no collective on the data path), so N
ranks run N replicas of the workload ("scaling": "weak"); value = total steps
of all ranks / max-over-ranks device time.

The reference arm (--impl reference) times the CPU restatement of the
reference algorithm (the reference itself is Fortran and cannot be built
here) on the host cores, rank 0 only.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from fastearth3d_b200 import synth  # noqa: E402

DEFAULT_WORKLOAD = "c3_3d_l128"
DEFAULT_STEPS = {"c4_ensemble": 20, "c2_1d_sle_l128": 1000, "c1_1d_l64": 4000}
METRIC = "steps/s @lmax=128 3D visc: batched vs plain GPU, rsl err<=1e-8; grad/fwd"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: enough for each arm's timed region to last over a second: 300 "
                         "for the 3-D workload, 1000 for c2_1d_sle_l128, 4000 for c1_1d_l64; 20 for c4_ensemble)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--cpu-sample-s", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-one-thread", action="store_true",
                    help="also time one step of the oracle on one host thread (cpu_baseline_1thread)")
    ap.add_argument("--precision", default="exact_tc", choices=["exact_tc", "split_tc", "fp64"],
                    help="3-D stress products of the timed arm: exact int8-digit tensor-core products (default), "
                         "two-term TF32 tensor-core products, or FP64 on the CUDA cores")
    ap.add_argument("--plain", default="on", choices=["on", "off"],
                    help="also time the plain FP64 arm beside the tensor-core arm (and report the rsl error between them)")
    ap.add_argument("--tf32", default="on", choices=["on", "off"],
                    help="also time the two-term TF32 tensor-core arm beside the exact one (with its rsl error)")
    ap.add_argument("--ensemble-sle-ctas", default="rows", choices=["sm", "rows", "tuned"],
                    help="c4_ensemble: the fused sea-level loop's CTAs per instance (one per SM, one per grid row, "
                         "or the autotuner's choice, which also picks the exact stages' warp splits)")
    ap.add_argument("--toroidal", default="on", choices=["on", "off", "only"],
                    help="also time the FP64 path carrying the toroidal channels (toroidal = 1); "
                         "only: time that path alone as the main arm")
    ap.add_argument("--timeline", type=int, default=0, metavar="N",
                    help="instead of the benchmark: the kernel timeline of N steps of the main arm after the warm-up "
                         "(CUPTI kernel records through torch.profiler): per kernel its launches and device time a "
                         "step, and the step's busy and idle device time")
    ap.add_argument("--grad-fwd", default="on", choices=["on", "off", "only"],
                    help="also time the adjoint gradients against their forwards (grad/fwd: the coupled step's, "
                         "100 intervals with checkpoints every 50, and the response-level one); 'only' prints those "
                         "alone")
    return ap.parse_args()


PRECISION = {"fp64": 0, "split_tc": 1, "exact_tc": 2}
PRECISION_DTYPE = {"fp64": "f64",
                   "split_tc": "tf32x3 3-D stress products, f64 elsewhere",
                   "exact_tc": "int8-digit (5 x 8 bit, exact int32 accumulation) 3-D stress products, f64 elsewhere"}


def host_cpu():
    """The host's CPU model and logical cores (lscpu)."""
    info = {"nproc": os.cpu_count()}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            k, _, v = line.partition(":")
            if k.strip() in ("Model name", "Socket(s)", "Core(s) per socket", "Thread(s) per core"):
                info[k.strip()] = v.strip()
    except Exception:
        pass
    return info


def workload_config(w, n_sub, world):
    """The workload the step runs (identical in every arm, ours and the reference's)."""
    nk = (w.lmax + 1) * (w.lmax + 2) // 2 - 1
    ne = w.n_elem
    return {"workload": w.name, "lmax": w.lmax, "grid": f"{w.nlat}x{w.nphi}", "radial_elements": w.n_elem,
            "dt_yr": w.dt_yr, "n_sub": n_sub, "visc3d": w.visc3d, "sea_level": w.sle, "rotation": w.rotation,
            "parallelism": f"replicas{world}",
            "l2": ("state larger than L2 (%.0f MB streamed per sub-step)" if 6 * 4 * ne * nk * 8 > 126e6 else
                   "state fits L2 (%.0f MB), not flushed") % (6 * 4 * ne * nk * 8 / 1e6)}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def algorithmic_bytes(info, phase):
    """Algorithmic HBM bytes of one call of a phase (the state each must stream)."""
    ne, nk, nr = info.ne, info.nk, info.nr
    state = 6 * 4 * ne * nk * 8  # A/B/C re/im memory, (4, ne, nk) doubles each
    drift_nodal = 2 * 2 * nr * nk * 8  # dUn, dVn re/im
    if phase == "drift":  # read the state, write the nodal + surface drift
        return state + drift_nodal + 6 * nk * 8
    if phase == "advance_1d":  # read state + nodal drift, write state
        return 2 * state + drift_nodal
    return None


# the autotuner's cache for this run (a fresh file: every run tunes once per model key)
TUNE_CACHE = os.path.join(__import__("tempfile").mkdtemp(prefix="vg_tune_"), "tune.txt")

FP64_NOMINAL_TFLOPS = 37.0  # B200 dense FP64 (vector and tensor), datasheet figure


def cpu_baseline(w, budget_s, threads):
    from oracle import orc  # the CPU restatement: test/baseline infrastructure only

    orc.set_threads(threads)
    o = orc.Oracle(w.params(orc.default_params))
    zb, hi = w.reference()
    o.set_reference(zb, hi)
    if w.visc3d:
        o.enable_visc3d(w.pert(o.p))
    o.update(w.ice_at(1), w.dt_yr)  # warm-up step (untimed)
    t0 = time.perf_counter()
    n = 0
    while True:
        n += 1
        o.update(w.ice_at(1 + n), w.dt_yr)
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": f"{n} consecutive steps of {w.name} after 1 warm-up step, {dt:.1f} s, OMP threads={threads}",
            "host": host_cpu()}


def run_reference(args, w):
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    steps = max(1, args.steps)
    budget = 150.0
    from oracle import orc

    o = orc.Oracle(w.params(orc.default_params))
    zb, hi = w.reference()
    o.set_reference(zb, hi)
    if w.visc3d:
        o.enable_visc3d(w.pert(o.p))
    for s in range(1, args.warmup + 1):
        o.update(w.ice_at(s), w.dt_yr)
    t0 = time.perf_counter()
    n = 0
    for s in range(steps):
        o.update(w.ice_at(args.warmup + 1 + s), w.dt_yr)
        n += 1
        if time.perf_counter() - t0 > budget:
            break
    dt = time.perf_counter() - t0
    v = n / dt
    sample = f"{n} of {steps} steps of {w.name} after {args.warmup} warm-up steps (bounded at {budget:.0f} s)"
    out = {"metric": METRIC, "value": v, "unit": "steps/s", "impl": "reference", "n_gpus": args.gpus,
           "steps": n, "warmup": args.warmup, "ms_per_step": 1e3 * dt / n, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": workload_config(w, o.info().n_sub_last, args.gpus),
           "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": "port", "sample": sample,
                            "host": host_cpu()},
           "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def stage_work(w, info, precision):
    """Algorithmic work of one call of each fine-grained phase, as
    {phase: {"flop": F, "tensor_ops": T, "bytes": B}} (missing keys: not
    applicable).

    Tensor-core stages: F = 2 x rows x N x K summed over the stage's
    sub-GEMMs (parity / half-period halves, no padding), one product per
    multiply-add; T = the operations the tensor pipe executes for them (split
    TF32: three products per multiply-add; exact int8: 15 digit-pair products);
    B = the stage's input read once and its output written once (FP64
    intermediates on the exact path, FP32 on the TF32 path). The gather and
    scatter stream the Maxwell-element state and the operand rows.
    """
    L, nlat, nphi = w.lmax, w.nlat, w.nphi
    nh, half = (nlat + 1) // 2, nphi // 2
    M = L + 1
    F = 3 * info.ne3d
    NC, NCOL = 2 * F, 6 * F
    kev, kod = 2 * (L // 2), 2 * ((L + 1) // 2)
    legendre = 2.0 * NC * nh * info.nlm * 6  # sum over m of (K_E + K_O) = nlm, 6 products
    inv = 2.0 * NCOL * (half - 1) * (kev + kod) * nlat
    fwd = 2.0 * NCOL * (kev + kod) * half * nlat
    products = {"exact_tc": 15, "split_tc": 3}.get(precision, 1)
    eb = 4 if precision == "split_tc" else 8  # bytes of an intermediate value
    ne3d, nk = info.ne3d, info.nk
    X = (nk + 1) * 4 * NC * eb
    S = M * nlat * 6 * NC * eb
    Gs = nlat * 2 * half * NCOL * eb
    dy = (nk + 1) * 6 * NC * eb
    rate = nlat * nphi * ne3d * eb
    state3 = 6 * 4 * ne3d * nk * 8  # memory of the 3-D elements, one buffer
    drift = 2 * 2 * (ne3d + 1) * nk * 8
    out = {"v3_synth": {"flop": legendre, "tensor_ops": products * legendre, "bytes": X + S},
           "v3_lon_inv": {"flop": inv, "tensor_ops": products * inv, "bytes": S + Gs + rate},
           "v3_lon_fwd": {"flop": fwd, "tensor_ops": products * fwd, "bytes": Gs + S},
           "v3_analysis": {"flop": legendre, "tensor_ops": products * legendre, "bytes": S + dy},
           "v3_gather": {"bytes": state3 + drift + X},
           "v3_scatter": {"bytes": 2 * state3 + dy},
           "drift": {"bytes": algorithmic_bytes(info, "drift")},
           "advance_1d": {"bytes": algorithmic_bytes(info, "advance_1d")}}
    if precision == "fp64":  # one kernel runs the whole longitude pass
        out["v3_lon_inv"] = {"flop": inv + fwd, "bytes": 2 * S + rate}
    return out


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# tensor-core stages on the lmax-128 3-D workload, from one ncu capture per
# stage (profiles/ names the command)
NCU_TRAFFIC = {("c3_3d_l128", "split_tc", "v3_synth"): 150.75e6, ("c3_3d_l128", "split_tc", "v3_lon_inv"): 227.35e6,
               ("c3_3d_l128", "split_tc", "v3_lon_fwd"): 223.56e6,
               ("c3_3d_l128", "split_tc", "v3_analysis"): 209.04e6,
               ("c3_3d_l128", "exact_tc", "v3_lon_inv"): 490.36e6, ("c3_3d_l128", "exact_tc", "v3_lon_fwd"): 474.24e6,
               ("c3_3d_l128", "exact_tc", "v3_analysis"): 421.21e6}


def max_over_ranks(ms, dist, device):
    """Replica timing: every rank's device time of the timed region, reduced to
    the maximum (the slowest replica bounds the job)."""
    import torch

    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, steps, max_ms):
    """Whole-job steps/s of `world` independent replicas of `steps` steps each."""
    return world * steps / (max_ms * 1e-3)


def run_arm(w, precision, args, ice_dev, local, dist, want_e2e, toroidal=False):
    """Warm-up, device-timed region, phase-timer pass and end-to-end pass of one
    model instance of the workload; returns the measurements."""
    import torch

    from fastearth3d_b200 import lib as vlib

    p = w.params(vlib.default_params)
    p.visc3d_precision = precision
    p.toroidal = 1 if toroidal else 0
    m = vlib.Model(p)
    zb, hi = w.reference()
    m.set_reference(zb, hi)
    if w.visc3d:
        m.enable_visc3d(w.pert(m.p))
    ng = w.nlat * w.nphi
    total = args.warmup + args.steps
    stream = torch.cuda.ExternalStream(m.stream_ptr())
    for s in range(args.warmup):
        m.update_device(ice_dev[s].data_ptr(), w.dt_yr)
    tuned = None
    if precision == PRECISION["exact_tc"] and w.visc3d:
        # the project autotuner (bit-identical choices), timed from this state and put back
        t0 = time.perf_counter()
        cached = m.autotune(w.dt_yr, TUNE_CACHE)
        ncw, ctas = m.tuning()
        tuned = {"exact_stage_converter_warps": ncw, "sle_ctas": ctas, "from_cache": cached,
                 "tuning_s": round(time.perf_counter() - t0, 3)}
    launches0 = m.info().n_launch
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            ev0.record()
        for s in range(args.warmup, total):
            m.update_device(ice_dev[s].data_ptr(), w.dt_yr)
        with torch.cuda.stream(stream):
            ev1.record()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    out = {"ms": ms, "launches": m.info().n_launch - launches0, "info": m.info(), "clocks": clk.summary(),
           "tuning": tuned}
    out["rsl"], out["zbed"] = m.fields()[:2]
    if dist:
        out["ms"] = max_over_ranks(ms, dist, "cuda")
        dist.barrier()
    # phase timers over a few more steps (separate pass: the timers add events)
    n_prof = min(args.steps, 5)
    m.profile_enable(True)
    for s in range(total, total + n_prof):
        m.update_device(ice_dev[s].data_ptr(), w.dt_yr)
    out["ph_ms"], out["ph_calls"] = m.profile_read()
    m.profile_enable(False)
    if want_e2e:
        # end to end through the public C-ABI: host ice in pinned memory, rsl read back every step
        n_e2e = min(args.steps, 10)
        ice_host = torch.empty((n_e2e, ng), dtype=torch.float64).pin_memory()
        for s in range(n_e2e):
            ice_host[s] = torch.from_numpy(w.ice_at(total + n_prof + s + 1))
        rsl_host = np.zeros(ng)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record()
        for s in range(n_e2e):
            vlib.lib().vg_update(m.h, vlib.C.cast(ice_host[s].data_ptr(), vlib._P), w.dt_yr)
            vlib.lib().vg_get_fields(m.h, vlib.ptr(rsl_host), None, None, None)
        with torch.cuda.stream(stream):
            e1.record()
        torch.cuda.synchronize()
        out["e2e_ms"] = e0.elapsed_time(e1) / n_e2e
    del m
    torch.cuda.synchronize()
    return out


def measure_grad_fwd(w, nsteps=10, ckpt=5, nsite=200, seed=7):
    """Cost of the adjoint gradient against the forward it differentiates: a
    response-level run of the workload's earth (lateral viscosity on, FP64)
    with a seeded load per step and rsl observations at land-grid sites;
    J = vg_misfit, (J, dJ/dload, dJ/dlog10 eta) = vg_misfit_grad with
    checkpoints every `ckpt` steps (the rest recomputed). Each timed twice
    after a warm-up call, best of two, wall clock around the synchronous calls."""
    from fastearth3d_b200 import lib as vlib

    p = w.params(vlib.default_params)
    p.rotation = 0
    p.visc3d_precision = 0
    m = vlib.Model(p)
    if w.visc3d:
        m.enable_visc3d(w.pert(m.p))
    rng = np.random.default_rng(seed)
    sig = (rng.standard_normal((nsteps, m.nlm)) + 1j * rng.standard_normal((nsteps, m.nlm))) * 1e3
    sig[:, : w.lmax + 1] = sig[:, : w.lmax + 1].real
    land = np.flatnonzero(w.topo.reshape(-1) > 0)
    sites = rng.choice(land if land.size >= nsite else np.arange(m.ng), nsite, replace=False)
    obs = 0.01 * rng.standard_normal((nsteps, nsite))
    dt = w.dt_yr * synth.SEC_PER_YEAR
    m.misfit(sig, dt, sites, obs)
    m.misfit_grad(sig, dt, sites, obs, ckpt, want_pert=w.visc3d)
    tf, tg = [], []
    for _ in range(2):
        t0 = time.perf_counter()
        m.misfit(sig, dt, sites, obs)
        t1 = time.perf_counter()
        m.misfit_grad(sig, dt, sites, obs, ckpt, want_pert=w.visc3d)
        t2 = time.perf_counter()
        tf.append(t1 - t0)
        tg.append(t2 - t1)
    return {"value": min(tg) / min(tf), "unit": "gradient cost / forward cost", "steps": nsteps, "ckpt_every": ckpt,
            "sites": nsite, "fwd_ms_per_step": 1e3 * min(tf) / nsteps, "grad_ms_per_step": 1e3 * min(tg) / nsteps,
            "gradient": "dJ/dload and dJ/dlog10(eta) of the 3-D elements" if w.visc3d else "dJ/dload",
            "model": "response-level steps (no sea-level equation), FP64", "target": 3.0}


def measure_grad_fwd_sle(w, nsteps=100, ckpt=50, nsite=200, seed=7):
    """Cost of the coupled adjoint (configuration 5's gradient) against its
    forward: nsteps intervals of the workload through vg_update's own driver
    (sub-steps, sea-level equation, lateral viscosity on the FP64 path) from
    the reference state, J = the rsl misfit at `nsite` land sites;
    vg_sle_misfit (forward) and vg_sle_misfit_grad (J, dJ/dice per interval,
    dJ/dlog10 eta on the grid and as the lateral field's spectrum) with
    checkpoints every `ckpt` intervals. Each timed after a warm-up call, wall
    clock around the synchronous calls."""
    from fastearth3d_b200 import lib as vlib

    p = w.params(vlib.default_params)
    p.rotation = 0
    p.visc3d_precision = 0
    m = vlib.Model(p)
    m.set_reference(*w.reference())
    if w.visc3d:
        m.enable_visc3d(w.pert(m.p))
    rng = np.random.default_rng(seed)
    ice = np.stack([w.ice_at(s + 1) for s in range(nsteps)])
    land = np.flatnonzero(w.topo.reshape(-1) > 0)
    sites = rng.choice(land if land.size >= nsite else np.arange(m.ng), nsite, replace=False).astype(np.int32)
    obs = 0.5 * rng.standard_normal((nsteps, nsite))
    m.sle_misfit(ice, w.dt_yr, sites, obs)
    m.sle_misfit_grad(ice, w.dt_yr, sites, obs, ckpt, want_pert=w.visc3d)
    t0 = time.perf_counter()
    m.sle_misfit(ice, w.dt_yr, sites, obs)
    t1 = time.perf_counter()
    m.sle_misfit_grad(ice, w.dt_yr, sites, obs, ckpt, want_pert=w.visc3d)
    t2 = time.perf_counter()
    return {"value": (t2 - t1) / (t1 - t0), "unit": "gradient cost / forward cost", "steps": nsteps,
            "ckpt_every": ckpt, "sites": nsite,
            "fwd_ms_per_step": 1e3 * (t1 - t0) / nsteps, "grad_ms_per_step": 1e3 * (t2 - t1) / nsteps,
            "gradient": "dJ/dice per interval on the Gauss grid" + (
                ", dJ/dlog10(eta) of the 3-D elements and of the lateral field's spectrum" if w.visc3d else ""),
            "model": "the coupled step (sea-level equation, FE sub-steps), FP64", "target": 3.0}


def phases_of(arm):
    from fastearth3d_b200.abi import PHASE_NAMES

    return {n: {"ms_per_call": arm["ph_ms"][i] / arm["ph_calls"][i] if arm["ph_calls"][i] else 0.0,
                "calls": int(arm["ph_calls"][i]), "ms_total": float(arm["ph_ms"][i])}
            for i, n in enumerate(PHASE_NAMES)}


def roofline(w, arm, pk, pk_kind, precision):
    """Roofline of the dominant kernel (the fine-grained phase with the most
    time; each 3-D stage phase is one kernel launch). For a tensor-core stage
    both bounds are evaluated, the tensor pipe (operations it executes against
    the measured dense peak of its input type: int8 = 2 x bf16, tf32 = bf16 / 2,
    both from the sustained bf16 figure) and HBM (algorithmic bytes against
    the measured copy bandwidth); the binding one (larger fraction) is
    reported, the other beside it."""
    info = arm["info"]
    ph = phases_of(arm)
    work = stage_work(w, info, precision)
    # one-kernel phases first (the 3-D stages); the drift and advance phases are
    # a few kernels each and stand in only for workloads without 3-D elements
    cands = [n for n in work if n.startswith("v3_") and ph.get(n, {}).get("calls")]
    cands = cands or [n for n in work if ph.get(n, {}).get("calls")]
    dom = max(cands, key=lambda n: ph[n]["ms_total"])
    wk = work[dom]
    t = ph[dom]["ms_per_call"] * 1e-3
    hbm = {"bound": "hbm", "kernel": dom, "achieved": wk["bytes"] / t / 1e9, "peak": pk["hbm_gbs"], "unit": "GB/s",
           "peak_kind": pk_kind + " copy bandwidth", "algorithmic_bytes_per_launch": wk["bytes"]}
    hbm["frac"] = hbm["achieved"] / hbm["peak"]
    traffic = NCU_TRAFFIC.get((w.name, precision, dom))
    if "tensor_ops" in wk and precision in ("exact_tc", "split_tc"):
        if precision == "exact_tc":
            peak, kind = 2.0 * pk["bf16_tflops_sustained"], " sustained dense bf16 x 2 (int8 rate)"
        else:
            peak, kind = 0.5 * pk["bf16_tflops_sustained"], " sustained dense bf16 x 0.5 (tf32 rate)"
        ten = {"bound": "tensor", "kernel": dom, "achieved": wk["tensor_ops"] / t / 1e12, "peak": peak,
               "unit": "TOP/s" if precision == "exact_tc" else "TFLOP/s", "peak_kind": pk_kind + kind,
               "tensor_ops_per_launch": wk["tensor_ops"], "useful_flops_per_launch": wk["flop"]}
        ten["frac"] = ten["achieved"] / ten["peak"]
        main, other = (ten, hbm) if ten["frac"] >= hbm["frac"] else (hbm, ten)
        main = dict(main)
        main["traffic"] = traffic
        main["traffic_source"] = "ncu capture, DRAM bytes per launch" if traffic else None
        main["other_bound"] = {k: other[k] for k in ("bound", "achieved", "peak", "unit", "frac")}
        return main
    if "flop" in wk:  # the FP64 path's CUDA-core stages
        fp64 = wk["flop"] / t / 1e12
        out = {"bound": "fp64", "kernel": dom, "achieved": fp64, "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
               "frac": fp64 / FP64_NOMINAL_TFLOPS, "peak_kind": "nominal FP64 (no measured FP64 peak)",
               "traffic": traffic, "algorithmic_flops_per_launch": wk["flop"]}
        out["other_bound"] = {k: hbm[k] for k in ("bound", "achieved", "peak", "unit", "frac")}
        return out
    hbm["traffic"] = traffic
    return hbm


def run_ensemble(args):
    """The batched ensemble (32 instances of mixed lmax, earth and viscosity,
    half with 3-D viscosity on the tensor-core path of --precision), advanced together
    through vg_update_batch, against the same instances run one after the other
    on the plain FP64 path ("32 sequential plain runs") and, to separate the
    concurrency from the precision, sequentially on the batched precision.
    value = instance-steps/s of the batched run."""
    import torch

    from fastearth3d_b200 import lib as vlib

    members = synth.ensemble()
    n, W, K = len(members), args.warmup, args.steps
    DT = members[0].dt_yr
    ice = [[np.ascontiguousarray(mb.ice_at(s + 1)) for s in range(W + K + 1)] for mb in members]
    ice_dev = [torch.tensor(np.stack(x), device="cuda") for x in ice]

    def make(mb, split):
        p = mb.params(vlib.default_params)
        p.visc3d_precision = PRECISION[args.precision] if (split and mb.visc3d) else 0
        if args.ensemble_sle_ctas == "rows":  # the fused sea-level loop on one CTA per grid row at most
            p.sle_ctas = mb.nlat
        m = vlib.Model(p)
        zb, hi = mb.reference()
        m.set_reference(zb, hi)
        if mb.visc3d:
            m.enable_visc3d(mb.pert(m.p))
        if args.ensemble_sle_ctas == "tuned":  # once per model key (the cache), bit-identical choices
            p.sle_ctas = mb.nlat
            m.autotune(DT, TUNE_CACHE, knobs=1)  # the stages; the loop keeps one CTA per grid row
        return m

    def dev_timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        torch.cuda.synchronize()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    # batched, split precision for the 3-D instances
    models = [make(mb, True) for mb in members]
    for s in range(W):
        vlib.update_batch(models, [ice_dev[i][s].data_ptr() for i in range(n)], DT, on_device=True)
    launches0 = sum(m.info().n_launch for m in models)
    with ClockSampler(0) as clk:
        ms_batch = dev_timed(lambda: [vlib.update_batch(models, [ice_dev[i][s].data_ptr() for i in range(n)], DT,
                                                         on_device=True) for s in range(W, W + K)])
    launches = sum(m.info().n_launch for m in models) - launches0
    rsl_batch = [m.fields()[0] for m in models]
    # end to end: host ice in, every instance's rsl out, each step
    ng_tot = sum(mb.nlat * mb.nphi for mb in members)
    rsl_out = [np.zeros(mb.nlat * mb.nphi) for mb in members]

    def e2e_step():
        vlib.update_batch(models, [ice[i][W + K] for i in range(n)], DT)
        for i, m in enumerate(models):
            vlib.lib().vg_get_fields(m.h, vlib.ptr(rsl_out[i]), None, None, None)

    ms_e2e = dev_timed(e2e_step)
    del models
    torch.cuda.synchronize()
    # sequential: each instance's W + K steps, alone, one instance after another
    seq, by_class = {}, {}
    for split in (False, True):
        tot, rsl_seq = 0.0, []
        for i, mb in enumerate(members):
            m = make(mb, split)
            for s in range(W):
                m.update_device(ice_dev[i][s].data_ptr(), DT)
            t_i = dev_timed(lambda: [m.update_device(ice_dev[i][s].data_ptr(), DT) for s in range(W, W + K)])
            tot += t_i
            if split:
                key = "l%d%s" % (mb.lmax, "_3d" if mb.visc3d else "_1d")
                by_class[key] = by_class.get(key, 0.0) + t_i / K
            rsl_seq.append(m.fields()[0])
            del m
        seq[split] = (tot, rsl_seq)
    same = all(np.array_equal(a, b) for a, b in zip(rsl_batch, seq[True][1]))
    worst = max(float(np.abs(a - b).max() / np.abs(b).max()) for a, b, mb in zip(rsl_batch, seq[False][1], members)
                if mb.visc3d)
    lm = sorted({mb.lmax for mb in members})
    out = {
        "metric": "instance-steps/s, batched ensemble of %d (lmax %s, half 3-D) vs %d sequential plain runs" % (
            n, "/".join(map(str, lm)), n),
        "value": n * K / (ms_batch / 1e3),
        "unit": "instance-steps/s",
        "n_gpus": 1,
        "steps": K,
        "warmup": W,
        "ms_per_step": ms_batch / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": PRECISION_DTYPE[args.precision] + " (3-D instances)",
        "data": "synthetic",
        "config": {"workload": "c4_ensemble", "instances": n, "sle_ctas": args.ensemble_sle_ctas,
                   "lmax": [mb.lmax for mb in members],
                   "visc3d": [bool(mb.visc3d) for mb in members], "radial_elements": [mb.n_elem for mb in members],
                   "dt_yr": DT, "sea_level": True, "parallelism": "one stream and one host thread per instance"},
        "sequential_plain_fp64": {"value": n * K / (seq[False][0] / 1e3), "unit": "instance-steps/s",
                                  "ms_total": seq[False][0]},
        "sequential_same_precision": {"value": n * K / (seq[True][0] / 1e3), "unit": "instance-steps/s",
                                      "ms_total": seq[True][0]},
        "sequential_same_precision_ms_per_step_by_class": {k: round(v, 3) for k, v in sorted(by_class.items())},
        "speedup_vs_sequential_plain": seq[False][0] / ms_batch,
        "speedup_from_concurrency": seq[True][0] / ms_batch,
        "batched_equals_sequential": bool(same),
        "rsl_error_vs_fp64_3d_instances": worst,
        "e2e": {"value": n / (ms_e2e / 1e3), "unit": "instance-steps/s", "h2d_bytes_per_step": ng_tot * 8,
                "d2h_bytes_per_step": ng_tot * 8},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "cpu_baseline": None,
        "cpu_baseline_note": "not sampled: one oracle step of the lmax-256 3-D instances alone takes minutes",
    }
    print(json.dumps(out))


def run_timeline(args, w):
    """Kernel timeline of args.timeline steps of the main arm (after the warm-up
    and the autotuner), from the CUPTI kernel and copy records that
    torch.profiler collects: per kernel its launches and device time a step,
    the union of the busy intervals and the span. A profiling aid: nothing
    here is a bench value."""
    import collections

    import torch
    from torch.profiler import ProfilerActivity, profile

    from fastearth3d_b200 import lib as vlib

    prec = args.precision if w.visc3d else "fp64"
    p = w.params(vlib.default_params)
    p.visc3d_precision = PRECISION[prec]
    m = vlib.Model(p)
    m.set_reference(*w.reference())
    if w.visc3d:
        m.enable_visc3d(w.pert(m.p))
    n = args.timeline
    ice = torch.stack([torch.from_numpy(w.ice_at(s + 1)) for s in range(args.warmup + n)]).cuda()
    for s in range(args.warmup):
        m.update_device(ice[s].data_ptr(), w.dt_yr)
    if prec == "exact_tc" and w.visc3d:
        m.autotune(w.dt_yr, TUNE_CACHE)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for s in range(args.warmup, args.warmup + n):
            m.update_device(ice[s].data_ptr(), w.dt_yr)
        torch.cuda.synchronize()
    recs = sorted((e.time_range.start, e.time_range.end, e.name.split("(")[0])
                  for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA)
    tot, cnt = collections.defaultdict(float), collections.Counter()
    busy, cur_a, cur_b = 0.0, recs[0][0], recs[0][1]
    for a, b, name in recs:
        tot[name] += b - a
        cnt[name] += 1
        if a > cur_b:
            busy += cur_b - cur_a
            cur_a, cur_b = a, b
        else:
            cur_b = max(cur_b, b)
    busy += cur_b - cur_a
    span = recs[-1][1] - recs[0][0]
    kernels = [{"name": k, "launches_per_step": cnt[k] / n, "us_per_step": round(v / n, 2),
                "us_per_launch": round(v / cnt[k], 2), "share": round(v / sum(tot.values()), 4)}
               for k, v in sorted(tot.items(), key=lambda x: -x[1])]
    print(json.dumps({"workload": w.name, "precision": prec, "steps": n, "warmup": args.warmup,
                      "span_ms_per_step": round(span / n / 1e3, 4), "busy_ms_per_step": round(busy / n / 1e3, 4),
                      "records_per_step": len(recs) / n, "kernels": kernels}))


def main():
    args = parse()
    if args.steps is None:
        args.steps = DEFAULT_STEPS.get(args.workload, 300)
    if args.workload == "c4_ensemble":
        import torch

        torch.cuda.set_device(0)
        run_ensemble(args)
        return
    w = synth.workloads()[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args, w)
        return
    import torch

    if args.timeline > 0:
        if rank == 0:
            torch.cuda.set_device(local)
            run_timeline(args, w)
        return

    torch.cuda.set_device(local)
    if args.grad_fwd == "only":
        if rank == 0:
            out = {"workload": w.name, "grad_fwd_response": measure_grad_fwd(w)}
            if w.sle:
                out["grad_fwd"] = measure_grad_fwd_sle(w)
            print(json.dumps(out), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ng = w.nlat * w.nphi
    total = args.warmup + args.steps
    n_prof = min(args.steps, 5)
    ice_dev = torch.empty((total + n_prof + 1, ng), dtype=torch.float64, device="cuda")
    for s in range(total + n_prof + 1):
        ice_dev[s] = torch.from_numpy(w.ice_at(s + 1))
    tor_only = w.visc3d and args.toroidal == "only"
    prec = args.precision if (w.visc3d and not tor_only) else "fp64"
    tensor = prec in ("exact_tc", "split_tc")
    main_arm = run_arm(w, PRECISION[prec], args, ice_dev, local, dist, True, tor_only)
    plain = run_arm(w, 0, args, ice_dev, local, dist, False) if tensor and args.plain == "on" else None
    tf32 = (run_arm(w, PRECISION["split_tc"], args, ice_dev, local, dist, False)
            if prec == "exact_tc" and args.tf32 == "on" else None)
    tor = run_arm(w, 0, args, ice_dev, local, dist, False, True) if w.visc3d and args.toroidal == "on" else None
    tor_ex = (run_arm(w, PRECISION["exact_tc"], args, ice_dev, local, dist, False, True)
              if tor is not None and prec == "exact_tc" else None)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    pk, pk_kind = peaks()
    info = main_arm["info"]
    ms = main_arm["ms"]

    def error_vs(arm, ref):
        r0, r1 = ref["rsl"], arm["rsl"]
        z0, z1 = ref["zbed"], arm["zbed"]
        return {"after_steps": total, "rsl": float(np.abs(r1 - r0).max() / np.abs(r0).max()),
                "z_bed": float(np.abs(z1 - z0).max() / np.abs(z0).max()),
                "norm": "max abs diff / max abs (FP64 GPU path, same steps)"}

    out = {
        "metric": METRIC,
        "value": replica_throughput(world, args.steps, ms),
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": PRECISION_DTYPE[prec],
        "data": "synthetic",
        "config": workload_config(w, info.n_sub_last, world),
        "arm": {"visc3d_precision": prec, "toroidal": bool(tor_only), "tuning": main_arm["tuning"]},
        "e2e": {"value": 1e3 / main_arm["e2e_ms"], "unit": "steps/s", "h2d_bytes_per_step": ng * 8,
                "d2h_bytes_per_step": ng * 8},
        "gpu_launches": int(main_arm["launches"]),
        "roofline": roofline(w, main_arm, pk, pk_kind, prec),
        "phases": phases_of(main_arm),
        "clocks": main_arm["clocks"],
    }
    if plain is not None:
        out["plain_fp64"] = {
            "value": replica_throughput(world, args.steps, plain["ms"]), "unit": "steps/s",
            "ms_per_step": plain["ms"] / args.steps, "speedup_over_plain": plain["ms"] / ms, "target": 3.0,
            "gpu_launches": int(plain["launches"]), "phases": phases_of(plain), "clocks": plain["clocks"],
            "roofline": roofline(w, plain, pk, pk_kind, "fp64")}
        err = error_vs(main_arm, plain)
        err["rsl_target"] = 1e-8
        err["rsl_target_met"] = bool(err["rsl"] <= 1e-8)
        out["error_vs_fp64"] = err
        if tf32 is not None:
            e32 = error_vs(tf32, plain)
            out["split_tf32"] = {
                "value": replica_throughput(world, args.steps, tf32["ms"]), "unit": "steps/s",
                "ms_per_step": tf32["ms"] / args.steps, "speedup_over_plain": plain["ms"] / tf32["ms"],
                "error_vs_fp64": e32, "rsl_target_met": bool(e32["rsl"] <= 1e-8),
                "phases": phases_of(tf32), "clocks": tf32["clocks"]}
    if tor is not None:
        ref = plain if plain is not None else (main_arm if not tensor else None)
        out["toroidal_fp64"] = {
            "value": replica_throughput(world, args.steps, tor["ms"]), "unit": "steps/s",
            "ms_per_step": tor["ms"] / args.steps, "gpu_launches": int(tor["launches"]), "n_sub": tor["info"].n_sub_last,
            "cost_vs_spheroidal_fp64": (tor["ms"] / ref["ms"]) if ref is not None else None,
            "phases": phases_of(tor), "clocks": tor["clocks"]}
        if tor_ex is not None:
            out["toroidal_exact"] = {
                "value": replica_throughput(world, args.steps, tor_ex["ms"]), "unit": "steps/s",
                "ms_per_step": tor_ex["ms"] / args.steps, "speedup_over_toroidal_fp64": tor["ms"] / tor_ex["ms"],
                "error_vs_toroidal_fp64": error_vs(tor_ex, tor), "tuning": tor_ex["tuning"],
                "phases": phases_of(tor_ex), "clocks": tor_ex["clocks"]}
    if args.grad_fwd == "on":
        out["grad_fwd_response"] = measure_grad_fwd(w)
        if w.sle:
            out["grad_fwd"] = measure_grad_fwd_sle(w)
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(w, args.cpu_sample_s, os.cpu_count() or 1)
        if args.cpu_one_thread:  # one step at one thread (a minute or more at lmax 128): the scalar baseline
            out["cpu_baseline_1thread"] = cpu_baseline(w, 0.0, 1)
    print(json.dumps(out))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
