"""Benchmark of the HyDFT solver step on B200.

Workload (one "step" = one low-storage RK3 step, 3 stages, of the whole
grid): Yukawa ions with the Maxwell closure, tau from the Ichimaru form
(HNC u_ex and du/dGamma), 256^3 periodic box L = 64 a, Gamma = 50,
kappa = 2, eta from the Bastea MD fit, Gaussian random delta n with power
spectrum ~ exp(-q^2), rms 1e-2 (seeded counter-based stream), u = 0,
Pi = 0; fields in FP32 with FP64 conserved sums.  The FP64 path is timed
beside it ("FP32 vs FP64-plain"), and the FP32 field error is measured
against the FP64 run after the timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs independent replicas, one per GPU (the solver step does not
shard; no collective is on the data path).  --impl reference times the
reference algorithm's CPU path (the FP64 oracle restatement of the
Fortran code, OpenMP over all host cores) on a bounded sample of the same
workload.  One JSON line is printed by rank 0.
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

METRIC = "RK3 cell-steps/s FP32-batched vs FP64-plain on B200 at ≤1e-5 rel err; p50/p99"
UNIT = "cell-steps/s"
# algorithmic bytes per cell-step of the minimal exact transform schedule,
# Maxwell ions: 3 stages x (8 B x 44 transforms + 16 B x 10 state fields), FP32
STEP_BYTES_FP32 = 3 * (8 * 44 + 16 * 10)
# Newtonian ions: 3 stages x (8 B x 20 transforms + 16 B x 4 state fields)
STEP_BYTES_FP32_NEWTONIAN = 3 * (8 * 20 + 16 * 4)


def workload_params(hg, n, precision, L=64.0):
    return hg.default_params(
        kind="ion", gamma=50.0, kappa=2.0, nx=n, ny=n, nz=n, lx=L, ly=L, lz=L,
        closure="maxwell", transport="yukawa_fit", tau_model="ichimaru",
        hnc_nr=4096, hnc_rmax=80.0, cfl=0.4, dt=0.0, gpu_precision=precision)


def initial_density(n, L, n0, seed=2024):
    from hydft_b200 import ic
    d = ic.gaussian_spectrum_field(n, n, n, L, L, L, seed, qc=1.0)
    return n0 * (1.0 + 1e-2 * d)


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled through NVML
    every 10 ms while the timed region runs (nvidia-smi every 100 ms when
    NVML is unavailable).  Reading only: no clock or device setting is
    changed."""

    # NVML clock-event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}

    def __init__(self, cuda_device, period=0.01):
        self.dev = cuda_device
        self.period = period
        self.samples = []          # (wall time, sm MHz, max sm MHz, reasons bitmask, power W)
        self.window = None
        self.source = None
        self._stop = threading.Event()
        self.thread = None

    def mark(self, t0, t1):
        """Keep only the samples taken between wall-clock times t0 and t1."""
        self.window = (t0, t1)

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.dev)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [x for x in vis.split(",") if x.strip()]
            idx = int(ids[self.dev]) if self.dev < len(ids) and ids[self.dev].isdigit() else self.dev
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)

    def _run_nvml(self, nv, h):
        smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while not self._stop.is_set():
            t = time.time()
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
            except Exception:
                break
            self.samples.append((t, sm, smax, rs, pw))
            self._stop.wait(self.period)

    def _run_smi(self, proc):
        import datetime
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rs = 0
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        rs |= self.REASONS[nm]
                self.samples.append((ts, float(parts[1]), float(parts[2]), rs, float(parts[3])))
            except ValueError:
                continue

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.source = "nvml, 10 ms"
            self.thread = threading.Thread(target=self._run_nvml, args=(nv, h), daemon=True)
            self.thread.start()
            return
        except Exception:
            pass
        fields = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                  "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                  "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + fields, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi, 100 ms"
            self.thread = threading.Thread(target=self._run_smi, args=(self.proc,), daemon=True)
            self.thread.start()
        except OSError:
            self.source = None

    def stop(self):
        self._stop.set()
        if self.source and self.source.startswith("nvidia-smi"):
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)
        if self.source is None:
            return None
        out = self._summary(self.window)
        if out is None and self.window is not None:
            out = self._summary(None)
            if out is not None:
                out["window"] = "no sample inside the timed region; all samples"
        return out

    def _summary(self, window):
        sel = [s for s in self.samples if window is None or window[0] - 0.005 <= s[0] <= window[1] + 0.005]
        if not sel:
            return None
        reasons = sorted(nm for nm, bit in self.REASONS.items() if any(s[3] & bit for s in sel))
        return {"sm_mhz": float(np.median([s[1] for s in sel])), "sm_max_mhz": float(max(s[2] for s in sel)),
                "reasons": reasons, "samples": len(sel), "power_w_max": float(max(s[4] for s in sel)),
                "source": self.source}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic(kernel, precision):
    """DRAM read + write bytes of one launch of `kernel` from the committed
    ncu summary of the step (profiles/maxwell256_<precision>_dram_per_kernel.md)."""
    path = os.path.join(ROOT, "profiles", "maxwell256_%s_dram_per_kernel.md" % precision)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("| %s |" % kernel):
                    cols = [c.strip() for c in line.strip().strip("|").split("|")]
                    if len(cols) == 2:
                        return float(cols[1])
    except (OSError, ValueError, IndexError):
        pass
    return None


def workload_config(n, L, world):
    """The workload's description, identical in both arms."""
    return {"workload": "maxwell_ion_%d^3" % n, "grid": [n, n, n], "box_L": L,
            "gamma": 50.0, "kappa": 2.0, "closure": "maxwell", "tau_model": "ichimaru",
            "transport": "yukawa_fit", "hnc": "yukawa, nr 4096, rmax 80, tol 1e-9",
            "ic": "gaussian random delta n, power ~ exp(-q^2), rms 1e-2, seed 2024; u = 0, Pi = 0",
            "dt": "compute_dt at t = 0, cfl 0.4",
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (working set ~GBs)"}


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    return orc


def _ic_module():
    """hydft_b200/ic.py loaded as a plain module (numpy only), so that the
    reference arm does not import the package or load its GPU library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_hydft_ic", os.path.join(ROOT, "hydft_b200", "ic.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def oracle_workload_model(orc, n, L, structure):
    """The oracle (the reference's FP64 CPU algorithm, literal transform
    schedule) set up on the workload: structure = dict(k, c, u_ex,
    du_dgamma) from an HNC solve."""
    n0 = 3 / (4 * np.pi)
    p = orc.params(kind="ion", gamma=50.0, kappa=2.0, nx=n, ny=n, nz=n, lx=L, ly=L, lz=L,
                   closure="maxwell", transport="yukawa_fit", tau_model="ichimaru", cfl=0.4,
                   hnc_nr=4096, hnc_rmax=80.0)
    st = orc.Structure(structure["k"], structure["c"], n0, structure["u_ex"], structure["du_dgamma"], True)
    m = orc.Model(p, st)
    d = _ic_module().gaussian_spectrum_field(n, n, n, L, L, L, 2024, qc=1.0)
    m.set_state(n0 * (1.0 + 1e-2 * d))
    m.compute_dt()
    return m


def time_oracle_stages(m, warmup, samples):
    """Time `samples` RK3 stages of the oracle after `warmup` stages; the
    stages cycle 1, 2, 3, so three consecutive samples are one RK3 step.
    Returns (seconds, stages run before the timed ones)."""
    s = 0
    for _ in range(warmup):
        m.stage(s % 3)
        s += 1
    t0 = time.perf_counter()
    for _ in range(samples):
        m.stage(s % 3)
        s += 1
    return time.perf_counter() - t0


STAGE_SAMPLE = ("each sample is one of the three RK3 stages of the full %d^3 workload step (rhs + stage update "
                "+ relaxation + dealias, the reference's literal 123-transform stage), stages cycling 1,2,3; "
                "a sample counts as 1/3 cell-step per cell; FP64 oracle restatement of the reference CPU path "
                "(model.f90:186-227), OpenMP over %d host threads (%s)")


def run_reference(args):
    """The reference's algorithm on the host cores: the FP64 oracle on the
    same workload (grid, box, physics, initial state, dt) as the GPU arm,
    with its HNC solved on the CPU too; nothing of the GPU library is
    loaded.  Each of the K timed steps is one RK3 stage of the full grid."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    orc = _oracle()
    threads = host_threads()
    orc.set_threads(threads)
    n, L = args.n, 64.0
    t0 = time.perf_counter()
    s = orc.structure_from_hnc(orc.make_pot("yukawa", 50.0, 2.0), 3 / (4 * np.pi), 4096, 80.0, 1e-9, 0.2,
                               20000, with_derivative=True)
    m = oracle_workload_model(orc, n, L, dict(k=s.k, c=s.c, u_ex=s.u_ex, du_dgamma=s.du_dgamma))
    setup_s = time.perf_counter() - t0
    samples = max(1, args.steps)
    el = time_oracle_stages(m, args.warmup, samples)
    v = float(n) ** 3 * (samples / 3.0) / el
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": samples, "warmup": args.warmup, "ms_per_step": 1e3 * el / samples,
            "ms_per_rk3_step": 3e3 * el / samples,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(n, L, world),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": STAGE_SAMPLE % (n, threads, cpu_model())},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "setup_s": setup_s, "dt": m.dt, "host": {"threads": threads, "cpu": cpu_model()}}
    print(json.dumps(line), flush=True)
    return 0


# transforms per RK3 step of the Maxwell ion step: the minimal exact schedule
# this library runs (per stage 24 inverse + 20 forward) and the reference's
# literal schedule (369 3-D transforms per step)
MIN_C2R, MIN_R2C = 3 * 24, 3 * 20
LITERAL_TRANSFORMS = 369


def cufft_comparator(torch, dev, n):
    """cuFFT (through torch.fft) timed on the same grid, as a comparator only:
    the transforms alone, no physics.  FP32 at the minimal schedule's count,
    FP64 at the reference's literal count (split evenly between r2c and c2r)."""
    out = {}
    for dt, name in ((torch.float32, "fp32"), (torch.float64, "fp64")):
        x = torch.randn((n, n, n), dtype=dt, device=dev)
        xh = torch.fft.rfftn(x)
        for _ in range(3):
            torch.fft.irfftn(torch.fft.rfftn(x), s=x.shape)
        reps = 10
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize(dev)
        e[0].record()
        for _ in range(reps):
            torch.fft.rfftn(x)
        e[1].record()
        for _ in range(reps):
            torch.fft.irfftn(xh, s=x.shape)
        e[2].record()
        torch.cuda.synchronize(dev)
        r2c = e[0].elapsed_time(e[1]) / reps
        c2r = e[1].elapsed_time(e[2]) / reps
        out[name] = {"r2c_ms": r2c, "c2r_ms": c2r}
        del x, xh
    f32, f64 = out["fp32"], out["fp64"]
    out["fp32_min_schedule_ms_per_step"] = MIN_C2R * f32["c2r_ms"] + MIN_R2C * f32["r2c_ms"]
    out["fp64_literal_schedule_ms_per_step"] = LITERAL_TRANSFORMS / 2 * (f64["c2r_ms"] + f64["r2c_ms"])
    out["note"] = ("torch.fft (cuFFT) transforms only, full half spectrum, no band pruning, no physics; "
                   "a lower bound on a cuFFT-based step at each schedule")
    return out


def batch_members(hg, count, seed=2025):
    """The ensemble workload: grids from {32,48,64,96,128}^3 (dx of the
    32^3, L = 20 a case), Gamma log-uniform in [1, 100], kappa uniform in
    [0.5, 3], Newtonian / Maxwell 50/50, one Fourier mode from the lowest
    four shells at amplitude 1e-3, FP32 fields."""
    rng = np.random.default_rng(seed)
    shells = [m for m in np.ndindex(5, 5, 5) if 1 <= sum(x * x for x in m) <= 4]
    out = []
    for _ in range(count):
        n = int(rng.choice([32, 48, 64, 96, 128]))
        L = 20.0 * n / 32.0
        gamma = float(10 ** rng.uniform(0.0, 2.0))
        kappa = float(rng.uniform(0.5, 3.0))
        maxwell = bool(rng.integers(0, 2))
        mode = shells[int(rng.integers(0, len(shells)))]
        kw = dict(kind="ion", gamma=gamma, kappa=kappa, nx=n, ny=n, nz=n, lx=L, ly=L, lz=L,
                  transport="yukawa_fit", hnc_nr=4096, hnc_rmax=80.0, cfl=0.4, dt=0.0, gpu_precision="fp32",
                  closure="maxwell" if maxwell else "newtonian", ic="mode", ic_amplitude=1e-3,
                  ic_mode=tuple(int(x) for x in mode))
        if maxwell:
            kw["tau_model"] = "ichimaru"
        out.append(kw)
    return out


def run_batch_leg(torch, hg, count, steps, warmup, dev):
    """The ensemble advanced by one graph launch per step; cell-steps/s over
    all members, with the roofline of the minimal schedule's bytes."""
    members = batch_members(hg, count)
    t0 = time.perf_counter()
    b = hg.Batch([hg.default_params(**kw) for kw in members], device=dev)
    setup_s = time.perf_counter() - t0
    cells = 0.0
    bytes_step = 0.0
    for kw, m in zip(members, b.members):
        m.set_initial_condition("mode", kw["ic_amplitude"], kw["ic_mode"])
        m.compute_dt()
        c = float(kw["nx"]) ** 3
        cells += c
        bytes_step += c * (STEP_BYTES_FP32 if kw["closure"] == "maxwell" else STEP_BYTES_FP32_NEWTONIAN)
    b.advance(warmup)
    stream = torch.cuda.ExternalStream(b.stream_ptr(), device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    l0 = b.launch_count()
    e0.record(stream)
    b.advance(steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    launches = b.launch_count() - l0
    # per-step device times: p50 / p99
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    evs[0].record(stream)
    for i in range(steps):
        b.advance(1)
        evs[i + 1].record(stream)
    torch.cuda.synchronize(dev)
    per = np.array([evs[i].elapsed_time(evs[i + 1]) for i in range(steps)])
    peak, _ = measured_peak()
    achieved = bytes_step * steps / (ms * 1e-3) / 1e9
    sizes = {}
    for kw in members:
        sizes[kw["nx"]] = sizes.get(kw["nx"], 0) + 1
    out = {"workload": "ensemble of %d ion runs, grids {32,48,64,96,128}^3, Gamma log-uniform [1,100], "
                       "kappa uniform [0.5,3], Newtonian/Maxwell 50/50, one mode amplitude 1e-3, FP32" % count,
           "members": count, "members_per_grid": {str(k): v for k, v in sorted(sizes.items())},
           "maxwell_members": sum(1 for kw in members if kw["closure"] == "maxwell"),
           "cells": cells, "value": cells * steps / (ms * 1e-3), "unit": UNIT, "steps": steps,
           "ms_per_step": ms / steps, "step_ms_p50": float(np.percentile(per, 50)),
           "step_ms_p99": float(np.percentile(per, 99)), "gpu_launches": int(launches),
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "bytes_per_step": bytes_step},
           "setup_s": setup_s}
    b.close()
    return out


def chi_members(hg, n, omegas, precision):
    """The driven-response sweep: electrons r_s = 1, theta = 1 (Thomas-Fermi,
    gradient, Hartree, RY), n^3 box of L = 40, constant eta = 0.2, driven
    v_ext = 1e-4 cos(q.x - w t) at q = 2 pi/L (3, 0, 0), one member per w.
    dt from compute_dt with cfl 0.8 (inside the RK3 limits the reference's
    compute_dt builds in, model.f90:176-181), so that the 4000 steps span
    t = 230, about seven damping times of the driven mode."""
    return [dict(kind="electron", rs=1.0, theta=1.0, nx=n, ny=n, nz=n, lx=40.0, ly=40.0, lz=40.0,
                 closure="newtonian", transport="constant", eta=0.2, vext="driven", vext_amplitude=1e-4,
                 vext_mode=(3, 0, 0), vext_omega=float(w), hnc_nr=4096, hnc_rmax=80.0, cfl=0.8, dt=0.0,
                 gpu_precision=precision) for w in omegas]


def chi_linear(m, q, w):
    """chi(q, w) = -q^2 n0 / (-w^2 + q^2 c^2(q) - i q^2 (eta_l/m) w/(1 - i w tau))
    (linear_response.f90:59-76) from the model's own functional kernel K(q),
    c^2 = n0 K(q)/m."""
    n0, mass = m.scalar("n0"), m.scalar("mass")
    eta_l = m.scalar("eta_l")
    tau = m.scalar("tau") if m.has_pi else 0.0
    c2 = n0 * m.kernel(q) / mass
    den = -w * w + q * q * c2 - 1j * q * q * (eta_l / mass) * w / (1.0 - 1j * w * tau)
    return -q * q * n0 / den


def run_chi_leg(torch, hg, dev, n=128, nw=32, steps=4000, every=10):
    """C3: the driven chi(k, w) sweep, nw drive frequencies in [0.5, 3] w_p
    as one ensemble (one member per frequency), `steps` RK3 steps each, in
    FP32 and in FP64.  chi from the steady response of the driven mode
    (the window after 60 % of the run) against linear theory; FP32 against
    FP64 per frequency and per field after the steps."""
    omegas = np.linspace(0.5, 3.0, nw)
    q = 2.0 * np.pi * 3 / 40.0
    out = {"workload": "driven chi(k,w) sweep: %d electron runs (r_s 1, theta 1, TF + gradient + Hartree + RY), "
                       "%d^3, L = 40, w in [0.5, 3] w_p, v_ext 1e-4 at q = 2 pi/L (3,0,0), %d RK3 steps each"
                       % (nw, n, steps), "members": nw, "steps": steps}
    states, chis = {}, {}
    for prec in ("fp32", "fp64"):
        b = hg.Batch([hg.default_params(**kw) for kw in chi_members(hg, n, omegas, prec)], device=dev)
        try:
            dt = None
            for m in b.members:
                m.set_state(np.full((n, n, n), m.scalar("n0")))
                d = m.compute_dt()
                dt = d if dt is None else min(dt, d)
            for m in b.members:
                m.set_time(0.0, dt)
            stream = torch.cuda.ExternalStream(b.stream_ptr(), device=dev)
            ts, zs = [], [[] for _ in omegas]
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            ms = 0.0
            done = 0
            while done < steps:
                k = min(every, steps - done)
                e0.record(stream)
                b.advance(k)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                ms += e0.elapsed_time(e1)
                done += k
                ts.append(done * dt)
                for i, m in enumerate(b.members):
                    zs[i].append(m.mode(0, 3, 0, 0))
            ts = np.array(ts)
            sel = ts >= 0.6 * ts[-1]
            errs, scat, chi = [], [], []
            for i, w in enumerate(omegas):
                z = np.array(zs[i])[sel] * np.exp(1j * w * ts[sel])
                a = z.mean()
                chi_sim = 2.0 * a / 1e-4
                chi_lin = chi_linear(b.members[i], q, w)
                chi.append(chi_sim)
                errs.append(abs(chi_sim - chi_lin) / abs(chi_lin))
                scat.append(float(np.abs(z - a).max() / abs(a)))
            chis[prec] = np.array(chi)
            states[prec] = [m.get_state() for m in b.members]
            out[prec] = {"value": nw * float(n) ** 3 * steps / (ms * 1e-3), "unit": UNIT,
                         "ms_per_ensemble_step": ms / steps, "dt": dt, "t_end": steps * dt,
                         "chi_rel_err_vs_linear_max": float(max(errs)), "chi_rel_err_vs_linear": [float(e) for e in errs],
                         "transient_scatter_max": float(max(scat)), "grouped": b.grouped()}
        finally:
            b.close()
    fe = []
    for s32, s64 in zip(states["fp32"], states["fp64"]):
        n0 = s64[0].mean()
        fe.append(max(float(np.linalg.norm(s32[0] - s64[0]) / np.linalg.norm(s64[0])),
                      float(np.linalg.norm(s32[1] - s64[1]) / np.linalg.norm(s64[1]))))
    out["fp32_rel_err_vs_fp64_max"] = max(fe)
    out["chi_fp32_vs_fp64_max"] = float(np.max(np.abs(chis["fp32"] - chis["fp64"]) / np.abs(chis["fp64"])))
    out["omegas"] = [float(w) for w in omegas]
    return out


# even 2^a 3^b lengths in [32, 256] (the GPU path's FFT lengths)
SERVE_SIZES = [32, 36, 48, 54, 64, 72, 96, 108, 128, 144, 162, 192, 216, 256]


def serve_request(hg, rng, step_scale):
    """One request of the serving stream: an ion Newtonian (Gamma 10, kappa 1,
    dx 0.625), ion Maxwell (Gamma 50, kappa 2, Ichimaru tau, dx 0.25) or
    electron driven (r_s 1, theta 1, dx 0.3125) solve on an N^3 grid drawn
    uniformly from SERVE_SIZES, 500-5000 RK3 steps, FP32 fields."""
    n = int(rng.choice(SERVE_SIZES))
    kind = int(rng.integers(0, 3))
    steps = max(1, int(round(int(rng.integers(500, 5001)) * step_scale)))
    common = dict(nx=n, ny=n, nz=n, gpu_precision="fp32", hnc_nr=4096, hnc_rmax=80.0, cfl=0.4, dt=0.0,
                  ic="mode", ic_amplitude=1e-3, ic_mode=(1, 0, 0))
    if kind == 0:
        L = 0.625 * n
        kw = dict(kind="ion", gamma=10.0, kappa=1.0, transport="yukawa_fit", lx=L, ly=L, lz=L, **common)
    elif kind == 1:
        L = 0.25 * n
        kw = dict(kind="ion", gamma=50.0, kappa=2.0, closure="maxwell", transport="yukawa_fit",
                  tau_model="ichimaru", lx=L, ly=L, lz=L, **common)
    else:
        L = 0.3125 * n
        kw = dict(kind="electron", rs=1.0, theta=1.0, transport="constant", eta=0.2, vext="driven",
                  vext_amplitude=1e-4, vext_mode=(3, 0, 0), vext_omega=1.0, lx=L, ly=L, lz=L, **common)
        kw["ic"] = "uniform"
    return ("ion_newtonian", "ion_maxwell", "electron_driven")[kind], n, steps, kw


def run_serve_leg(hg, dev, rates, per_rate, step_scale, seed=7):
    """Poisson arrivals at each rate into one continuous-batching server;
    latency (submit to completion) p50/p99 and throughput per rate."""
    rng = np.random.default_rng(seed)
    srv = hg.Server(device=dev, max_slots=64, chunk_steps=25)
    out = {"workload": "serving stream: Poisson arrivals; ion Newtonian / ion Maxwell / electron driven solves on "
                       "N^3, N uniform over %s, 500-5000 RK3 steps x %g, FP32" % (SERVE_SIZES, step_scale),
           "per_rate": per_rate, "rates": []}
    try:
        for lam in rates:
            reqs = [serve_request(hg, rng, step_scale) for _ in range(per_rate)]
            gaps = rng.exponential(1.0 / lam, size=per_rate)
            ids = []
            t0 = time.perf_counter()
            at = 0.0
            for (name, n, steps, kw), gap in zip(reqs, gaps):
                at += gap
                delay = at - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                ids.append(srv.submit(hg.default_params(**kw), steps))
            lat, lat_nosetup, work, first, last = [], [], 0.0, None, None
            failed = 0
            for rid, (name, n, steps, kw) in zip(ids, reqs):
                srv.wait(rid)
                try:
                    info, _ = srv.result(rid)
                except hg.HydftError:
                    failed += 1
                    continue
                lat.append(info["t_done"] - info["t_submit"])
                lat_nosetup.append(info["t_done"] - info["t_submit"] - (info["t_start"] - info["t_admit"]))
                work += float(n) ** 3 * steps
                first = info["t_submit"] if first is None else min(first, info["t_submit"])
                last = info["t_done"] if last is None else max(last, info["t_done"])
            st = srv.stats()
            out["rates"].append({
                "lambda_per_s": lam, "requests": per_rate, "failed": failed,
                "latency_s_p50": float(np.percentile(lat, 50)) if lat else None,
                "latency_s_p99": float(np.percentile(lat, 99)) if lat else None,
                "latency_excl_setup_s_p50": float(np.percentile(lat_nosetup, 50)) if lat else None,
                "latency_excl_setup_s_p99": float(np.percentile(lat_nosetup, 99)) if lat else None,
                "throughput_cell_steps_per_s": work / (last - first) if lat else None,
                "throughput_req_per_s": len(lat) / (last - first) if lat else None,
                "max_requests_resident": st["max_holding"]})
    finally:
        srv.close()
    return out


def structure_for_workload(hg, device):
    m = hg.Model(workload_params(hg, 8, "fp64"), device=device)
    k, c = m.structure()
    st = dict(k=k, c=c, u_ex=m.scalar("u_ex"), du_dgamma=m.scalar("du_dgamma"))
    m.close()
    return st


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--err-steps", type=int, default=2000,
                    help="RK3 steps of the FP32-vs-FP64 field error check (the workload's 2000)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-plain leg")
    ap.add_argument("--no-cufft", action="store_true", help="skip the cuFFT comparator")
    ap.add_argument("--quick", action="store_true",
                    help="setup, warm-up and the timed steps only (for profiler captures)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--batch-members", type=int, default=256,
                    help="also time the ensemble workload with this many members (0: skip)")
    ap.add_argument("--workload", default="maxwell256", choices=["maxwell256", "batch", "serve", "chi"],
                    help="batch: time only the ensemble workload (256 members unless --batch-members); "
                         "serve: the serving stream at --rates")
    ap.add_argument("--chi-omegas", type=int, default=32, help="chi sweep: drive frequencies")
    ap.add_argument("--chi-steps", type=int, default=4000, help="chi sweep: RK3 steps per run")
    ap.add_argument("--rates", default="10,30,100,300,1000", help="serving arrival rates (requests/s)")
    ap.add_argument("--per-rate", type=int, default=6, help="serving requests per rate")
    ap.add_argument("--step-scale", type=float, default=1.0, help="serving steps scale (1: 500-5000)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import hydft_b200 as hg

    if args.workload == "serve":
        dev = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(dev)
        res = run_serve_leg(hg, dev, [float(x) for x in args.rates.split(",")], args.per_rate, args.step_scale)
        print(json.dumps(res), flush=True)
        return 0
    if args.workload == "chi":
        dev = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(dev)
        print(json.dumps(run_chi_leg(torch, hg, dev, n=args.n if args.n != 256 else 128,
                                     nw=args.chi_omegas, steps=args.chi_steps)), flush=True)
        return 0
    if args.workload == "batch":
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        res = run_batch_leg(torch, hg, args.batch_members or 256, args.steps, args.warmup,
                            int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps(res), flush=True)
        return 0

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = local

    n = args.n
    L = 64.0
    st = structure_for_workload(hg, dev)
    m32 = hg.Model(workload_params(hg, n, args.precision), structure=st, device=dev)
    n0 = m32.scalar("n0")
    nin = initial_density(n, L, n0)
    zeros3 = np.zeros((3, n, n, n))
    zeros6 = np.zeros((6, n, n, n))
    m32.set_state(nin, zeros3, zeros6)
    dt = m32.compute_dt()
    stream = torch.cuda.ExternalStream(m32.stream_ptr(), device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    # warm-up (graph capture, first touches)
    m32.advance(args.warmup)
    torch.cuda.synchronize(dev)
    barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.4)
    launches0 = m32.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    barrier()
    w0 = time.time()
    e0.record(stream)
    m32.advance(args.steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    w1 = time.time()
    barrier()
    clocks.mark(w0, w1)
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    gpu_launches = m32.launch_count() - launches0
    ms_max = ms
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    cells = float(n) ** 3
    value = cells * args.steps * world / (ms_max * 1e-3)
    ms_step = ms_max / args.steps
    # the autotuned tile shapes the timed steps ran with
    tiles = {"yz_inverse": [int(m32.scalar("yz_tile")), int(m32.scalar("yz_threads"))],
             "yz_forward": [int(m32.scalar("yz_tile_fwd")), int(m32.scalar("yz_threads_fwd"))],
             "x_threads": int(m32.scalar("x_threads"))}
    if args.quick:
        if rank == 0:
            print(json.dumps({"quick": True, "grid": n, "precision": args.precision, "value": value, "tiles": tiles,
                              "ms_per_step": ms_step, "gpu_launches": int(gpu_launches)}), flush=True)
        m32.close()
        if dist is not None:
            dist.destroy_process_group()
        return 0

    # per-kernel device time of 2 uncaptured steps, CUDA events on the stream
    prof = m32.profile(2)
    tot = sum(v[0] for v in prof.values())
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    dname, (dms, dbytes, dn) = dom
    peak, peak_kind = measured_peak()
    achieved = dbytes / (dms / dn * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "share": dms / tot,
            "bytes_per_launch": dbytes, "avg_launch_ms": dms / dn,
            "traffic": profile_traffic(dname, "fp32"),
            "traffic_source": "profiles/maxwell256_fp32_dram_per_kernel.md (ncu dram read + write bytes of one "
                              "full-size launch, committed capture; not measured in this run)"}
    kernels = {k: {"ms_per_step": v[0] / 2, "launches_per_step": v[2] / 2,
                   "GBps": (v[1] / (v[0] / v[2] * 1e-3) / 1e9) if v[0] > 0 and v[1] > 0 else None}
               for k, v in prof.items()}

    extra = {}
    # per-step device times (one graph replay each, CUDA events between steps)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    torch.cuda.synchronize(dev)
    evs[0].record(stream)
    for i in range(args.steps):
        m32.advance(1)
        evs[i + 1].record(stream)
    torch.cuda.synchronize(dev)
    per_step = np.array([evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)])
    extra["step_ms"] = {"p50": float(np.percentile(per_step, 50)), "p99": float(np.percentile(per_step, 99)),
                        "min": float(per_step.min()), "max": float(per_step.max()), "n": int(args.steps)}
    if not args.no_cufft:
        extra["cufft_comparator"] = cufft_comparator(torch, dev, n)
    if args.batch_members > 0:
        extra["batch"] = run_batch_leg(torch, hg, args.batch_members, max(3, args.steps // 3), args.warmup, dev)
    # FP64-plain leg and the FP32 field error against it
    if not args.no_fp64:
        m64 = hg.Model(workload_params(hg, n, "fp64"), structure=st, device=dev)
        m64.set_state(nin, zeros3, zeros6)
        m64.set_time(0.0, dt)
        s64 = torch.cuda.ExternalStream(m64.stream_ptr(), device=dev)
        k64 = max(1, args.steps)
        m64.advance(max(3, args.warmup))
        torch.cuda.synchronize(dev)
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(s64)
        m64.advance(k64)
        f1.record(s64)
        torch.cuda.synchronize(dev)
        v64 = cells * k64 / (f0.elapsed_time(f1) * 1e-3)
        # the workload's 2000 steps from the same initial state in FP32 and
        # FP64 (a fresh FP64 model), then the relative l2 error per field
        nerr = max(1, args.err_steps)
        m64.close()
        m64 = hg.Model(workload_params(hg, n, "fp64"), structure=st, device=dev)
        m64.set_state(nin, zeros3, zeros6)
        m64.set_time(0.0, dt)
        m32b = hg.Model(workload_params(hg, n, "fp32"), structure=st, device=dev)
        m32b.set_state(nin, zeros3, zeros6)
        m32b.set_time(0.0, dt)
        t_err = time.perf_counter()
        m64.advance(nerr)
        m32b.advance(nerr)
        a = m32b.get_state()
        b = m64.get_state()
        t_err = time.perf_counter() - t_err
        errs = {}
        for name, x, y in (("n", a[0], b[0]), ("mom", a[1], b[1]), ("pi", a[2], b[2])):
            errs[name] = float(np.linalg.norm(x - y) / np.linalg.norm(y))
        errs["dn"] = float(np.linalg.norm((a[0] - n0) - (b[0] - n0)) / np.linalg.norm(b[0] - n0))
        errs["max"] = max(errs["n"], errs["mom"], errs["pi"])
        errs["within_1e-5"] = bool(errs["max"] <= 1e-5)
        extra["fp64_plain"] = {"value": v64, "unit": UNIT, "steps": k64, "ratio_fp32_over_fp64": value / world / v64}
        extra["fp32_rel_err_vs_fp64"] = dict(errs, steps=nerr, t=nerr * dt, wall_s=t_err,
                                             definition="||x32 - x64||_2 / ||x64||_2 over each field after "
                                                        "the steps, same initial state and dt")
        del a, b
        m64.close()
        m32b.close()

    # end to end through the public API: host arrays in, per-step advance()
    # calls with a probe of one mode read back each step (the driver's loop,
    # src/hydft.f90:41-51), the final state read back
    me = hg.Model(workload_params(hg, n, "fp32"), structure=st, device=dev)

    def pinned(shape):
        return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()

    # host state in pinned memory, as a caller that streams states would keep it
    host_in = (pinned((n, n, n)), pinned((3, n, n, n)), pinned((6, n, n, n)))
    host_in[0][...] = nin
    host_in[1][...] = 0.0
    host_in[2][...] = 0.0
    host_out = (pinned((n, n, n)), pinned((3, n, n, n)), pinned((6, n, n, n)))
    torch.cuda.synchronize(dev)
    barrier()
    t0 = time.perf_counter()
    me.set_state(*host_in)
    me.set_time(0.0, dt)
    for _ in range(args.steps):
        me.advance(1)
        me.mode(0, 1, 0, 0)
    fin = me.get_state(out=host_out)
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    state_bytes = 8 * (1 + 3 + 6) * cells
    e2e = {"value": cells * args.steps * world / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": state_bytes / args.steps,
           "d2h_bytes_per_step": 16 + state_bytes / args.steps,
           "path": "set_state from pinned FP64 host arrays, per step advance(1) + one mode read "
                   "(src/hydft.f90:41-51 with iprobe = 1), get_state into pinned arrays; wall clock"}
    me.close()
    del fin

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # the oracle on the same 256^3 workload, one warm-up stage and one
        # RK3 step (three stage samples) timed, all host threads
        orc = _oracle()
        threads = host_threads()
        orc.set_threads(threads)
        om = oracle_workload_model(orc, n, L, st)
        el = time_oracle_stages(om, 1, 3)
        v = cells * 1.0 / el
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": (STAGE_SAMPLE % (n, threads, cpu_model())) + "; 3 samples (one RK3 step, %.1f s) "
                         "after one warm-up stage" % el}
        del om

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": workload_config(n, L, world),
                "precision": "fp32 fields and transforms, fp64 conserved sums", "dt": dt, "tiles": tiles,
                "roofline": roof,
                "step_roofline": {"bytes_per_cell_step": STEP_BYTES_FP32,
                                  "achieved_GBps": STEP_BYTES_FP32 * value / world / 1e9,
                                  "frac": STEP_BYTES_FP32 * value / world / 1e9 / peak},
                "kernels": kernels,
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(gpu_launches),
                "clocks": ck}
        line.update(extra)
        print(json.dumps(line), flush=True)
    m32.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
