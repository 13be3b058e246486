"""Benchmark: RK4 steps/s of the pseudo-spectral Navier-Stokes step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--n 256] [--impl b200|reference]

Workload (the 256^3 configuration of the headline metric): Taylor-Green
vortex 256^3, float64, nu = 1/3000, dt = 0.0025, synthetic (analytic) initial
field.  A step is one full RK4 step (24 kernel launches, four stages of six
kernels).  The working set (~2.6 GB) is far larger than the 126 MB L2, so no
explicit flush is needed between steps.

value   : steps/s with the state resident in HBM, CUDA events on the
          library's stream around exactly K steps (max over ranks; N > 1 runs
          N independent replicas, one per GPU, value = N * steps / max time).
e2e     : the same run as the `dns` CLI performs it through the C ABI with
          host buffers: pinned host field -> dns_set_velocity, K steps with
          dns_diagnostics every 10 steps (D2H), dns_get_fields at the end.
roofline: the kernel with the largest share of the step, algorithmic bytes
          per launch / its mean CUDA-event duration (dns_time_kernels).
cpu_baseline: the reference main.c (oracle/_ref/dns, compiled against the
          project's FFTW-subset shim since FFTW is absent) or the C
          restatement, timed on the host cores on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NU = 1.0 / 3000.0
DT = 0.0025
METRIC = "256^3 RK4 steps/s (FP64 Taylor-Green, nu=1/3000, dt=0.0025)"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC = os.path.join(ROOT, "profiles", "traffic.json")


def mask_fractions(n: int):
    """Fractions of the half spectrum's kz columns and of the kx (or ky)
    indices inside the 2/3 rule of main.c:231-238 (|k| < 2/3 (n/2 + 1))."""
    kmax = 2.0 / 3.0 * (n // 2 + 1)
    kcut = -1
    while kcut + 1 < kmax:
        kcut += 1
    fz = min(kcut + 1, n // 2 + 1) / (n // 2 + 1)
    fxy = min(2 * kcut + 1, n) / n
    return fz, fxy


# algorithmic HBM traffic per launch of each pass, in units of one complex
# half-spectrum field (n*n*(n/2+1)*16 bytes) and one real field (n^3 * 8)
# [stage][pass] -> (complex fields moved, real fields moved).  N is needed
# only inside the 2/3 rule: C stores kz <= kcut, D and E1 move the masked
# part, E2 reads N there only.
def pass_units(n: int, pressure: bool = False):
    fz, fxy = mask_fractions(n)
    u = []
    for s in range(4):
        a = (3 + 5, 0)
        # B reads u, dv/dx, v, w, dw/dx; writes u, omega_z, v, (w), dw/dy, dw/dx
        b = (5 + 5, 0) if s == 0 else (5 + 6, 0)
        # C reads u, v, (w), dw/dx, dw/dy, omega_z (+ the stale velocity in
        # stage 0, + its store in stage 3) and writes N for kz <= kcut
        if s == 0:
            c = (5 + 3 * fz, 3)
        elif s < 3:
            c = (6 + 3 * fz, 0)
        else:
            c = (6 + 3 * fz, 3)
        d = (3 * fz + 3 * fz * fxy, 0)
        e1 = (3 * fz * fxy + 3 * fz * fxy * fxy, 0)
        nn = 3 * fz * fxy * fxy
        if s == 0:
            e2 = (nn + 3 + 6, 0)
        elif s < 3:
            e2 = (nn + 9 + 6, 0)
        else:
            e2 = (nn + 6 + 3 + (1 if pressure else 0), 0)
        u.append([a, b, c, d, e1, e2])
    return u


def pass_bytes(n: int, s: int = 8):
    """Algorithmic bytes of every pass of every stage, s bytes per real
    (8: FP64, 4: the mixed path's FP32 storage)."""
    cf = n * n * (n // 2 + 1) * 2 * s
    rf = n ** 3 * s
    return [[uc * cf + ur * rf for (uc, ur) in st] for st in pass_units(n)]


def step_bytes(n: int, s: int = 8) -> int:
    """Algorithmic bytes of one RK4 step of this implementation."""
    return int(sum(map(sum, pass_bytes(n, s))))


def step_bytes_model(n: int, s: int = 8) -> int:
    """B_step = 216 * n^2 (n/2 + 1) * 2 * s bytes: the minimal fused five-pass
    traffic model of the reference path (for the % of HBM roofline figure)."""
    return 216 * n * n * (n // 2 + 1) * 2 * s


def load_peak():
    try:
        with open(PEAKS) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            a = [x.strip() for x in line.split(",")]
            if len(a) < 9:
                continue
            try:
                sm.append(float(a[1]))
                smax = float(a[2])
            except ValueError:
                continue
            for nm, v in zip(names, a[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(ms: float, pg, device: str = "cuda") -> float:
    """Slowest rank's time (every rank calls it at the same point)."""
    if pg is None:
        return ms
    import torch

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_rate(steps: int, max_ms: float, world: int) -> float:
    """Whole-job throughput of `world` independent replicas that each ran
    `steps` steps, timed by the slowest one."""
    return world * steps / (max_ms / 1000.0)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), for the CPU baseline."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_reference_rate(n: int, budget_s: float = 25.0):
    """Steps/s of the reference's CPU implementation on this host: the
    reference main.c on the oracle's FFT (oracle/_ref/dns) when it exists,
    else the C restatement.  Bounded sample: one untimed step, then as many
    steps as fit the budget."""
    import numpy as np

    import dns_b200
    import oracle

    cores = os.cpu_count() or 1
    U, V, W, P = dns_b200.tgv_fields(n)
    if os.path.exists(oracle.REF_DNS):
        env = dict(os.environ, OMP_NUM_THREADS=str(cores))
        with tempfile.TemporaryDirectory() as tmp:
            raw = os.path.join(tmp, "tgv.raw")
            dns_b200.write_raw(raw, (U, V, W, P))

            def run(k):
                T = "%.17g" % (DT * (k - 0.5))  # exactly k steps
                t0 = time.perf_counter()
                subprocess.run([oracle.REF_DNS, "-i", raw, "-n", repr(NU), "-s", repr(DT), "-t", T],
                               check=True, env=env, stdout=subprocess.DEVNULL)
                return time.perf_counter() - t0

            t1 = run(1)
            t2 = run(2)
            per = max(t2 - t1, 1e-3)
            k = max(2, min(20, int(budget_s / per)))
            tk = run(1 + k)
            rate = k / (tk - t1)
            return rate, cores, "reference", (
                f"main.c (reference, unchanged) on the oracle's FFTW-subset FFT, {n}^3 TGV, "
                f"{k} steps timed as the difference of a {1 + k}-step and a 1-step run, "
                f"OMP_NUM_THREADS={cores}")
    oracle.set_threads(cores)
    o = oracle.Oracle(n)
    o.set_velocity(U, V, W)
    t0 = time.perf_counter()
    o.step(NU, DT, 1)
    per = time.perf_counter() - t0
    k = max(1, min(20, int(budget_s / per)))
    t0 = time.perf_counter()
    o.step(NU, DT, k)
    rate = k / (time.perf_counter() - t0)
    return rate, cores, "port", f"C restatement of main.c, {n}^3 TGV, {k} steps, {cores} threads"


def ensemble_leg(steps: int, warmup: int):
    """Batched ensemble: 48 runs (32 at 64^3, 16 at 128^3), nu log-uniform
    in [1/3000, 1/100], Taylor-Green plus a seeded solenoidal perturbation
    of rms 1e-3 of the base, FP32 fields with FP64 reductions, dt = 0.005.
    Aggregate run-steps/s of one ensemble against the same 48 runs stepped
    one after another as plain single-run contexts."""
    import numpy as np
    import torch

    import dns_b200

    sizes = [64] * 32 + [128] * 16
    rng = np.random.Generator(np.random.PCG64(2024))
    nus = np.exp(rng.uniform(np.log(1 / 3000), np.log(1 / 100), len(sizes)))
    dt = 0.005
    prec = dns_b200.DNS_PREC_MIXED
    with dns_b200.Ensemble(sizes, prec) as ens:
        st = torch.cuda.ExternalStream(ens.stream)
        # initial fields generated on the device (seed = run index)
        for r in range(len(sizes)):
            ens.set_perturbed_tgv(r, seed=r, amplitude=1e-3)
        ens.set_params(nus, dt)
        ens.step(warmup)
        ens.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        ens.step(steps)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        d = ens.diagnostics(allow_nonfinite=True)
        finite = all(np.isfinite(float(a)) and np.isfinite(float(b)) for a, b in d)
        schedule = ens.schedule()
    # the other schedule of the ensemble autotuner, timed the same way
    other = {}
    chosen = schedule.split(" ")[0]
    flag = dns_b200.DNS_FLAG_ENS_PERSISTENT if chosen == "batched" else dns_b200.DNS_FLAG_ENS_BATCHED
    with dns_b200.Ensemble(sizes, prec, flag) as eo:
        so = torch.cuda.ExternalStream(eo.stream)
        for r in range(len(sizes)):
            eo.set_perturbed_tgv(r, seed=r, amplitude=1e-3)
        eo.set_params(nus, dt)
        eo.step(warmup)
        eo.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(so)
        eo.step(min(steps, 100))
        b.record(so)
        b.synchronize()
        oms = a.elapsed_time(b) / min(steps, 100)
        eo.synchronize()
        other = {"schedule": "persistent" if chosen == "batched" else "batched",
                 "ms_per_ensemble_step": oms, "value": len(sizes) / (oms / 1000.0)}
    # the sequential arm does the ensemble's work (every run of a size steps
    # `steps` times, one after another), so that it runs as long, under the
    # same power cap, as the ensemble
    seq_ms = {}
    for n in (64, 128):
        with dns_b200.Context(n, prec) as c:
            sc = torch.cuda.ExternalStream(c.stream)
            r = sizes.index(n)
            c.set_perturbed_tgv(seed=r, amplitude=1e-3)
            c.step(float(nus[r]), dt, warmup)
            c.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            nseq = sizes.count(n) * steps
            a.record(sc)
            c.step(float(nus[r]), dt, nseq)
            b.record(sc)
            b.synchronize()
            seq_ms[n] = a.elapsed_time(b) / nseq
    agg = len(sizes) * steps / (ms / 1000.0)
    seq = len(sizes) / ((32 * seq_ms[64] + 16 * seq_ms[128]) / 1000.0)
    peak, peak_kind = load_peak()
    ens_bytes = sum(step_bytes(n, 4) for n in sizes)
    ens_model = sum(step_bytes_model(n, 4) for n in sizes)
    ens_sps = steps / (ms / 1000.0)
    return {"runs": len(sizes), "sizes": "32x64^3 + 16x128^3", "precision": "mixed",
            "init": "device (dns_ens_set_perturbed_tgv, seed = run index)",
            "steps": steps, "value": agg, "unit": "run-steps/s",
            "ms_per_ensemble_step": ms / steps, "sequential_value": seq,
            "vs_sequential": agg / seq, "all_finite": finite,
            "seq_ms_per_step": {str(k): v for k, v in seq_ms.items()},
            "bytes_per_ensemble_step": ens_bytes,
            "roofline_frac": ens_bytes * ens_sps / (peak * 1e9),
            "frac_of_model_roofline": ens_model * ens_sps / (peak * 1e9),
            "peak_source": peak_kind, "schedule": schedule.split(" (")[0],
            "autotuner": schedule.split("; n=")[0], "other_schedule": other}


def n512_leg(steps: int, warmup: int):
    """512^3 Taylor-Green (generated on the device), nu = 1/3000,
    dt = 0.0025, 200 timed steps (T = 0.5) by default: FP64 and mixed
    steps/s and the step's fraction of the
    measured HBM peak (this implementation's algorithmic bytes, and the
    216 C model)."""
    import torch

    import dns_b200

    n = 512
    peak, _ = load_peak()
    out = {}
    for name, prec, s in (("fp64", dns_b200.DNS_PREC_FP64, 8), ("mixed", dns_b200.DNS_PREC_MIXED, 4)):
        with dns_b200.Context(n, prec) as c:
            st = torch.cuda.ExternalStream(c.stream)
            c.set_tgv()
            c.step(NU, DT, warmup)
            c.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            c.step(NU, DT, steps)
            b.record(st)
            b.synchronize()
            ms = a.elapsed_time(b) / steps
        sps = 1000.0 / ms
        out[name] = {"value": sps, "unit": "steps/s", "ms_per_step": ms, "steps": steps,
                     "frac": step_bytes(n, s) * sps / (peak * 1e9),
                     "frac_of_model_roofline": step_bytes_model(n, s) * sps / (peak * 1e9)}
    out["mixed"]["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def adjoint_leg(n: int = 128, snapshots: int = 20):
    """Discrete adjoint of the final energy (dns_adjoint_energy_prec): 128^3
    unit-energy random isotropic field, nu = 0.005, dt = 0.005, T = 2
    (401 steps), 20 snapshots, FP64 and mixed.  Wall time of the whole call
    (forward sweep with checkpoints, reverse sweep with recomputation, host
    copies of the field and the gradient) per step, against the plain
    forward step of the same precision."""
    import numpy as np

    import dns_b200

    nu, dt = 0.005, 0.005
    _, nsteps = dns_b200.step_schedule(2.0, dt)
    u0 = dns_b200.solenoidal_perturbation(n, seed=0)
    with dns_b200.Context(n) as c:
        c.set_velocity(*u0)
        E0, _ = c.diagnostics()
    s = float(1.0 / np.sqrt(E0))
    u0 = [a * s for a in u0]
    out = {"n": n, "steps": nsteps, "snapshots": snapshots}
    for name, prec in (("fp64", dns_b200.DNS_PREC_FP64), ("mixed", dns_b200.DNS_PREC_MIXED)):
        with dns_b200.Context(n, prec) as c:
            c.set_velocity(*u0)
            c.step(nu, dt, 5)
            c.synchronize()
            t0 = time.perf_counter()
            c.step(nu, dt, nsteps)
            c.synchronize()
            fwd_ms = (time.perf_counter() - t0) * 1000.0 / nsteps
        # warm-up (module load, plans)
        dns_b200.adjoint_energy(*u0, nu, dt, 8, snapshots=4, precision=prec)
        t0 = time.perf_counter()
        dns_b200.adjoint_energy(*u0, nu, dt, nsteps, snapshots=snapshots, precision=prec)
        wall = time.perf_counter() - t0
        leg = {"wall_s": wall, "ms_per_step": wall * 1000.0 / nsteps,
               "forward_ms_per_step": fwd_ms, "vs_forward_step": wall * 1000.0 / nsteps / fwd_ms}
        if name == "fp64":
            out.update(leg)
        else:
            out["mixed"] = leg
    return out


def run_reference_arm(args, world, rank):
    if rank != 0:
        return 0
    rate, cores, kind, sample = cpu_reference_rate(args.n)
    line = {
        "impl": "reference", "metric": METRIC if args.n == 256 else METRIC.replace("256^3", f"{args.n}^3"),
        "value": rate, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 / rate, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"taylor-green {args.n}^3 fp64 nu=1/3000 dt=0.0025",
                   "n": args.n, "nu": NU, "dt": DT},
        "cpu_baseline": {"value": rate, "unit": "steps/s", "cores": cores, "kind": kind, "sample": sample,
                         "cpu_model": cpu_model()},
        "e2e": {"value": rate, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-n512", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--profile", choices=["fp64", "mixed"], default=None,
                    help="profiling run: set-up and --warmup steps, then exactly one RK4 "
                         "step between cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference_arm(args, world, rank)

    import numpy as np
    import torch

    import dns_b200

    torch.cuda.set_device(local)
    if args.profile:
        prec = dns_b200.DNS_PREC_FP64 if args.profile == "fp64" else dns_b200.DNS_PREC_MIXED
        with dns_b200.Context(args.n, prec) as c:
            c.set_tgv()
            c.step(NU, DT, max(1, args.warmup))
            c.synchronize()
            torch.cuda.profiler.start()
            c.step(NU, DT, 1)
            c.synchronize()
            torch.cuda.profiler.stop()
            print(json.dumps({"profile": args.profile, "n": args.n, "schedule": c.schedule()}))
        return 0
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    n = args.n
    U, V, W, _ = dns_b200.tgv_fields(n)
    ctx = dns_b200.Context(n)
    stream = torch.cuda.ExternalStream(ctx.stream)
    ctx.set_velocity(U, V, W)
    ctx.step(NU, DT, args.warmup)
    ctx.synchronize()

    def barrier():
        if pg is not None:
            pg.barrier()

    # -- device-resident throughput --
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        gpu_id = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        gpu_id = str(local)
    clocks = ClockSampler(gpu_id)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    ctx.step(NU, DT, args.steps)
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(ms, pg)
    steps_per_s = args.steps / (ms / 1000.0)
    value = replica_rate(args.steps, ms, world)

    # -- per-kernel timing for the roofline --
    K = dns_b200.KERNELS_PER_STAGE
    kms = ctx.time_kernels(NU, DT, 3).reshape(4, K)
    pb = pass_bytes(n)
    share = kms.sum(axis=0)
    dom = int(np.argmax(share))
    dom_bytes = sum(pb[s][dom] for s in range(4)) / 4.0
    dom_ms = float(kms[:, dom].mean())
    peak, peak_kind = load_peak()
    achieved = dom_bytes / (dom_ms / 1000.0) / 1e9
    traffic = None
    try:
        with open(TRAFFIC) as f:
            tj = json.load(f)
        traffic = tj.get(str(n), {}).get(dns_b200.PASS_NAMES[dom])
    except Exception:
        pass
    sbytes = step_bytes(n)

    # -- mixed precision (FP32 fields/FFTs, FP64 reductions/coefficients) --
    E64, O64 = ctx.diagnostics()  # after warmup + timed + 3 kernel-timing steps
    done64 = args.warmup + args.steps + 3
    with dns_b200.Context(n, dns_b200.DNS_PREC_MIXED) as cm:
        sm = torch.cuda.ExternalStream(cm.stream)
        cm.set_velocity(U, V, W)
        cm.step(NU, DT, args.warmup)
        cm.synchronize()
        barrier()
        torch.cuda.synchronize()
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m0.record(sm)
        cm.step(NU, DT, args.steps)
        m1.record(sm)
        m1.synchronize()
        mixed_ms = m0.elapsed_time(m1)
        cm.step(NU, DT, done64 - args.warmup - args.steps)
        E32, O32 = cm.diagnostics()
        mkms = cm.time_kernels(NU, DT, 2).reshape(4, K)
    mixed_ms = max_over_ranks(mixed_ms, pg)
    mixed_sps = args.steps / (mixed_ms / 1000.0)
    mixed = {
        "value": replica_rate(args.steps, mixed_ms, world), "unit": "steps/s",
        "ms_per_step": mixed_ms / args.steps,
        "speedup_vs_fp64": mixed_sps / steps_per_s,
        "energy_rel_err_vs_fp64": float(abs(E32 - E64) / E64),
        "enstrophy_rel_err_vs_fp64": float(abs(O32 - O64) / O64),
        "compared_after_steps": done64,
        "step_hbm_frac": step_bytes(n, 4) * mixed_sps / (peak * 1e9),
        "step_hbm_frac_of_model_roofline": step_bytes_model(n, 4) * mixed_sps / (peak * 1e9),
        "kernel_ms": {dns_b200.PASS_NAMES[p]: [float(mkms[s, p]) for s in range(4)] for p in range(K)},
    }

    # -- end to end through the C ABI with host buffers --
    pinned = [torch.from_numpy(a.reshape(-1)).pin_memory() for a in (U, V, W)]
    outs = [torch.empty(n ** 3, dtype=torch.float64).pin_memory() for _ in range(3)]
    with dns_b200.Context(n) as c2:
        s2 = torch.cuda.ExternalStream(c2.stream)
        c2.set_velocity(*[p.numpy() for p in pinned])
        c2.step(NU, DT, 2)
        c2.synchronize()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s2)
        c2.set_velocity(*[p.numpy() for p in pinned])
        done, ndiag = 0, 0
        while done < args.steps:
            c2.diagnostics_dd()
            ndiag += 1
            k = min(10, args.steps - done)
            c2.step(NU, DT, k)
            done += k
        c2.diagnostics_dd()
        ndiag += 1
        lib = dns_b200.load_library()
        import ctypes

        st = lib.dns_get_fields(c2._h, *[ctypes.c_void_p(o.data_ptr()) for o in outs], None)
        assert st == 0
        e1.record(s2)
        e1.synchronize()
        e2e_ms = e0.elapsed_time(e1)
        wall = time.perf_counter() - t0
    e2e_ms = max_over_ranks(e2e_ms, pg)
    e2e = replica_rate(args.steps, e2e_ms, world)
    h2d = 3 * n ** 3 * 8 / args.steps
    d2h = (3 * n ** 3 * 8 + 32 * ndiag) / args.steps

    ens = ensemble_leg(500, args.warmup) if not args.no_ensemble else None
    big = n512_leg(200, 3) if (n == 256 and not args.no_n512) else None
    adj = adjoint_leg() if (n == 256 and not args.no_adjoint) else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, cores, kind, sample = cpu_reference_rate(n)
            cpu = {"value": rate, "unit": "steps/s", "cores": cores, "kind": kind, "sample": sample,
                   "cpu_model": cpu_model()}
        except Exception as ex:  # the CPU leg is a reported baseline only
            cpu = {"value": None, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC if n == 256 else METRIC.replace("256^3", f"{n}^3"),
            "value": value,
            "unit": "steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"taylor-green {n}^3 fp64 nu=1/3000 dt=0.0025", "n": n,
                       "nu": NU, "dt": DT, "precision": "fp64",
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "working set %.2f GB >> 126 MB L2, no flush" % (ctx.info()["device_bytes"] / 1e9)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": dns_b200.PASS_NAMES[dom], "peak_source": peak_kind,
                         "kernel_ms": dom_ms, "kernel_bytes": dom_bytes},
            "step_hbm": {"algorithmic_bytes": sbytes, "achieved_gbs": sbytes * steps_per_s / 1e9,
                         "frac": sbytes * steps_per_s / (peak * 1e9),
                         "model_bytes_216C": step_bytes_model(n),
                         "frac_of_model_roofline": step_bytes_model(n) * steps_per_s / (peak * 1e9)},
            "kernel_ms": {dns_b200.PASS_NAMES[p]: [float(kms[s, p]) for s in range(4)] for p in range(K)},
            "e2e": {"value": e2e, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "wall_s": wall},
            "gpu_launches": dns_b200.KERNELS_PER_STEP * args.steps,
            "mixed": mixed,
            "ensemble": ens,
            "n512": big,
            "adjoint": adj,
            "clocks": clk,
            "cpu_baseline": cpu,
            "schedule": ctx.schedule(),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
