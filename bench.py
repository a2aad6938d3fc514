#!/usr/bin/env python
"""Benchmark of the split-operator Gross-Pitaevskii step on B200.

Headline workload: the 3D imaginary-time ground state on a 256^3 grid on
[-12,12)^3, hbar = m = 1, anisotropic trap (wx, wy, wz) = (1, 1, 4), g = 1000,
dt = 1e-4, renormalised every step, from a seeded Gaussian of width 1 times
(1 + 0.01 xi), xi ~ N(0,1) iid (PCG64 seed 3), normalised.  It is the largest
configuration that fits one GPU and the one the ground-state accuracy gate
(dE/E <= 1e-6 against the FP64 form) applies to.  The field (128 MiB complex64,
256 MiB complex128) is larger than L2 (126 MB), so no flush is needed between
timed steps.

One bench step = one gpue_evolve call of 100 imaginary time steps of the fused
complex64 form through the C ABI (three full-field passes per time step: the
XY-plane pass, the z pass with the kinetic phase, the inverse XY-plane pass),
timed with CUDA events on the library's stream.  The same protocol times the
plain FP64 form (five line passes per step) for the fused-FP32 vs plain-FP64
ratio.  Extra legs: end to end through the C ABI with host buffers, the full
5000-step relaxation per form with its energies, the 1024^2 rotating
real-time case, the 256^2 FP64 ground state (10,000 steps), the 96-solve
batched sweep and the serving stream.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl reference times GPUE's path on the host CPU: the reference has no CPU
implementation, so this arm runs the FP64 CPU restatement of it (oracle/,
OpenMP over all host threads) on the same workload from the same initial
state; when GPUE's own CUDA build is present (oracle/_ref) the arm also times
it on this GPU on the full-size configurations, as an extra key.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from gpue_b200 import replicas  # noqa: E402  (pure Python; loads no library)

METRIC = ("grid-point-steps/s fused-FP32 vs plain-FP64 (same B200, ΔE/E≤1e-6); "
          "p99 lat")
UNIT = "grid-point-steps/s"
HEAD = dict(dim=3, n=256, box=12.0, wz=4.0, g=1000.0, gdt=1e-4, total_steps=5000,
            polish=50, seed=3)
WORKLOAD_NAME = ("3D imaginary-time ground state 256^3 on [-12,12)^3, (wx,wy,wz)=(1,1,4), "
                 "g=1000, dt=1e-4, renormalised every step")
STEPS_PER_BENCH_STEP = 100
REF_STEPS_PER_BENCH_STEP = 4  # the CPU arm's bench step (about a second of host work)
# the 1024^2 rotating real-time case (extra leg)
ROT = dict(dim=2, n=1024, box=16.0, g=500.0, omega=0.7, dt=5e-5, gdt=1e-4, total_steps=20000)
ROT_NAME = ("2D real-time rotating condensate 1024^2 on [-16,16)^2, g=500, Omega=0.7 gauge, "
            "dt=5e-5")
# the 256^2 plain FP64 ground state (extra leg)
SMALL = dict(dim=2, n=256, box=10.0, g=100.0, gdt=1e-4, steps=10000, every=1000, seed=1)
FLUSH_BYTES = 256 << 20
# passes per time step of each form on the headline workload
PASSES = {"fp32": 3, "fp64": 5}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="headline and e2e only")
    ap.add_argument("--only", choices=["batch", "serve", "accuracy", "rot2d", "small2d"],
                    default=None, help="run one auxiliary leg alone and print its JSON")
    ap.add_argument("--profile", choices=["fp32", "fp64", "fp32_3d", "fp64_3d", "batch"],
                    default=None,
                    help="profiling case for ncu: --warmup + --steps time steps of one form "
                         "(3D: the headline workload; 2D: the rotating case; batch: segments "
                         "of 100 steps of the 96-solve sweep), no timing output")
    return ap.parse_args()


# ----------------------------------------------------------- inputs -------

def gauss_start(dim, n, box, seed, normalise=False):
    """exp(-r^2/2) (1 + 0.01 xi), xi ~ N(0,1) iid (PCG64 seed), complex128,
    optionally normalised to sum |psi|^2 dV = 1."""
    import numpy as np
    dx = box / (n >> 1)
    x = -box + dx * np.arange(n)
    rng = np.random.Generator(np.random.PCG64(seed))
    if dim == 2:
        r2 = x[None, :] ** 2 + x[:, None] ** 2
    else:
        r2 = x[None, None, :] ** 2 + x[None, :, None] ** 2 + x[:, None, None] ** 2
    psi = np.exp(-r2 / 2.0) * (1.0 + 0.01 * rng.standard_normal(r2.shape))
    psi = psi.astype(np.complex128)
    if normalise:
        psi /= np.sqrt(np.sum(np.abs(psi) ** 2) * dx ** dim)
    return psi


def head_state():
    return gauss_start(3, HEAD["n"], HEAD["box"], HEAD["seed"], normalise=True)


def head_params(G, precision, device=0):
    return G.make_params(3, HEAD["n"], HEAD["box"], wz=HEAD["wz"], g=HEAD["g"],
                         gdt=HEAD["gdt"], precision=precision, device=device)


def phase_field(n, box, seed=2):
    import numpy as np
    dx = box / (n >> 1)
    rng = np.random.Generator(np.random.PCG64(seed))
    theta = 2 * np.pi * rng.random((n, n))
    k = 2 * np.pi * np.fft.fftfreq(n, d=dx)
    k2 = k[:, None] ** 2 + k[None, :] ** 2
    return np.real(np.fft.ifft2(np.fft.fft2(theta) * np.exp(-0.5 * k2 * 0.25)))


def rot_state(G, device):
    """FP64 imaginary-time relaxation (GPU) times a smoothed random phase."""
    import numpy as np
    n, box = ROT["n"], ROT["box"]
    dx = box / (n >> 1)
    x = -box + dx * np.arange(n)
    r2 = x[None, :] ** 2 + x[:, None] ** 2
    psi = np.exp(-r2 / 8.0).astype(np.complex128)
    p = G.make_params(2, n, box, g=ROT["g"], omega=ROT["omega"], gauge=True, gdt=2e-3,
                      dt=ROT["dt"], precision=G.PREC_FP64, device=device)
    with G.Solver(p) as s:
        s.set_wfc(psi)
        s.evolve(5000, 0)
        gs = s.get_wfc()
    return np.ascontiguousarray(gs * np.exp(1j * phase_field(n, box)))


def rot_params(G, precision, device):
    return G.make_params(2, ROT["n"], ROT["box"], g=ROT["g"], omega=ROT["omega"], gauge=True,
                         gdt=ROT["gdt"], dt=ROT["dt"], precision=precision, device=device)


# ------------------------------------------------------------ clocks ------

class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 50 ms from a reader
    thread; mark() brackets the timed region, stop() returns the samples
    taken inside it."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.window = [None, None]

    def start(self):
        import threading
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return

        def reader():
            for line in self.proc.stdout:
                self.lines.append((time.perf_counter(), line))

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()
        t_end = time.perf_counter() + 5.0
        while not self.lines and time.perf_counter() < t_end:  # first sample seen
            time.sleep(0.01)

    def mark(self, which):
        self.window[which] = time.perf_counter()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.thread.join(timeout=10)
        t0, t1 = self.window
        inside = [ln for t, ln in self.lines if t0 is None or (t0 <= t <= t1 + 0.06)]
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in inside:
            f = [t.strip() for t in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "power_w": statistics.median(power) if power else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "window_s": (t1 - t0) if t0 is not None and t1 is not None else None}


# ------------------------------------------------------- GPU timing -------

def timed_steps(G, torch, s, steps, warmup, dev, barrier, gstate, flush=None, sampler=None):
    """Per bench step one gpue_evolve call of STEPS_PER_BENCH_STEP time steps
    between CUDA events on the library's stream (after an L2 flush when
    `flush` is given)."""
    stream = torch.cuda.ExternalStream(s.stream(), device=dev)
    launches = 0
    off = 0
    for _ in range(warmup):
        if flush is not None:
            with torch.cuda.stream(stream):
                flush.fill_(1)
        s.evolve(STEPS_PER_BENCH_STEP, gstate, no_sync=True, step_offset=off)
        off += STEPS_PER_BENCH_STEP
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    if sampler:
        sampler.start()
        sampler.mark(0)
    for k in range(steps):
        with torch.cuda.stream(stream):
            if flush is not None:
                flush.fill_(float(k & 7))
            ev[k][0].record(stream)
        r = s.evolve(STEPS_PER_BENCH_STEP, gstate, no_sync=True, step_offset=off)
        launches += r["kernel_launches"]
        off += STEPS_PER_BENCH_STEP
        with torch.cuda.stream(stream):
            ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    if sampler:
        sampler.mark(1)
    clocks = sampler.stop() if sampler else None
    barrier()
    torch.cuda.synchronize(dev)
    ms = sum(a.elapsed_time(b) for a, b in ev)
    return ms, launches, clocks


def e2e_leg(G, torch, psi0, dev, calls=5, dist=None):
    """Through the C ABI with pinned host buffers on the headline workload:
    upload psi (complex128), evolve one bench step (100 imaginary time steps,
    fused complex64), download psi (complex128) and the energy."""
    import ctypes as C
    shape = psi0.shape
    pin_in = torch.empty(shape, dtype=torch.complex128, pin_memory=True)
    pin_out = torch.empty(shape, dtype=torch.complex128, pin_memory=True)
    hin = pin_in.numpy()
    hin[...] = psi0
    hout = pin_out.numpy()
    with G.Solver(head_params(G, G.PREC_FP32, dev)) as s:
        stream = torch.cuda.ExternalStream(s.stream(), device=dev)
        L = G.lib()
        # warm the graphs once
        L.gpue_set_wfc(s._h, C.c_void_p(hin.ctypes.data), G.MEM_HOST, G.C128)
        s.evolve(STEPS_PER_BENCH_STEP, 0)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
        off = 0
        for _ in range(calls):
            assert L.gpue_set_wfc(s._h, C.c_void_p(hin.ctypes.data), G.MEM_HOST, G.C128) == 0
            s.evolve(STEPS_PER_BENCH_STEP, 0, no_sync=True, step_offset=off)
            off += STEPS_PER_BENCH_STEP
            assert L.gpue_get_wfc(s._h, C.c_void_p(hout.ctypes.data), G.MEM_HOST, G.C128) == 0
            s.energy()
        with torch.cuda.stream(stream):
            e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
    pts = psi0.size
    rate, _, secs = replicas.job_rate(pts * STEPS_PER_BENCH_STEP * calls, ms * 1e-3, dist, dev)
    return {"value": rate, "unit": UNIT,
            "h2d_bytes_per_step": pts * 16, "d2h_bytes_per_step": pts * 16 + 8,
            "step": "one gpue_evolve() call of %d imaginary time steps with psi uploaded "
                    "from pinned host memory (complex128) before it and psi (complex128) "
                    "plus the energy read back after it" % STEPS_PER_BENCH_STEP,
            "calls": calls, "ms": secs * 1e3}


def accuracy_leg(G, dev, peak):
    """The full relaxation of the headline workload per form: 5000 imaginary
    time steps (steady state, graph-replayed) and the energies, then 50 FP64
    polish steps on both; the FP64 form is pinned to GPUE's own build."""
    psi0 = head_state()
    pts = HEAD["n"] ** 3
    out = {"workload": WORKLOAD_NAME + ", %d steps (+%d FP64 polish steps)"
           % (HEAD["total_steps"], HEAD["polish"])}
    res = {}
    for name, prec in (("fp64", G.PREC_FP64), ("fp32", G.PREC_FP32)):
        with G.Solver(head_params(G, prec, dev)) as s:
            s.autotune()
            s.set_wfc(psi0)
            r = s.evolve(HEAD["total_steps"], 0)
            E = s.energy()
            if name == "fp64":
                s.evolve(HEAD["polish"], 0, step_offset=HEAD["total_steps"])
            else:
                s.evolve(0, 0, polish_steps=HEAD["polish"], step_offset=HEAD["total_steps"])
            res[name] = (r["device_ms"] * 1e-3 / HEAD["total_steps"], E, s.energy())
    t64, E64, E64p = res["fp64"]
    t32, E32, E32p = res["fp32"]
    out.update({
        "fp32_value": pts / t32, "fp64_value": pts / t64, "unit": UNIT,
        "fp32_over_fp64": t64 / t32,
        "E_fp64": E64, "E_fp32": E32, "dE_rel_fp32": abs(E32 - E64) / abs(E64),
        "E_fp64_polished": E64p, "E_fp32_polished": E32p,
        "dE_rel_fp32_polished": abs(E32p - E64p) / abs(E64p),
        "alg_frac_80B": 80 * pts / t32 / 1e9 / peak,
        "note": "steady-state device time of one gpue_evolve call of 5000 steps per form; "
                "alg_frac_80B = 80 bytes per point and step (five full-field complex64 "
                "read+write passes, the line schedule) x points/s over the measured HBM "
                "copy rate"})
    return out


def rot2d_leg(G, torch, dev, barrier, steps=20, warmup=3):
    """The 1024^2 rotating real-time case: flushed bench steps per form."""
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    psi0 = rot_state(G, dev)
    pts = ROT["n"] ** 2
    out = {"workload": ROT_NAME}
    for name, prec in (("fp64", G.PREC_FP64), ("fp32", G.PREC_FP32)):
        with G.Solver(rot_params(G, prec, dev)) as s:
            s.autotune()
            s.set_wfc(psi0)
            ms, _, _ = timed_steps(G, torch, s, steps, warmup, dev, barrier, 1, flush=flush)
            r = s.evolve(ROT["total_steps"], 1)
        out[name + "_value"] = pts * steps * STEPS_PER_BENCH_STEP / (ms * 1e-3)
        out[name + "_steady_value"] = pts * ROT["total_steps"] / (r["device_ms"] * 1e-3)
    out["fp32_over_fp64"] = out["fp32_value"] / out["fp64_value"]
    out["unit"] = UNIT
    out["note"] = ("value: %d flushed bench steps of %d real-time steps; steady: one "
                   "gpue_evolve call of %d steps, graph-replayed"
                   % (steps, STEPS_PER_BENCH_STEP, ROT["total_steps"]))
    return out


def small2d_leg(G, dev):
    """The 256^2 ground state on [-10,10)^2, g = 100, dt = 1e-4, 10,000 steps
    with energy checks every 1000: one gpue_evolve call per form."""
    psi0 = gauss_start(2, SMALL["n"], SMALL["box"], SMALL["seed"], normalise=True)
    pts = SMALL["n"] ** 2
    out = {"workload": "2D imaginary-time ground state 256^2 on [-10,10)^2, g=100, dt=1e-4, "
                       "10000 steps, renormalised every step"}
    for name, prec in (("fp64", G.PREC_FP64), ("fp32", G.PREC_FP32)):
        with G.Solver(G.make_params(2, SMALL["n"], SMALL["box"], g=SMALL["g"],
                                    gdt=SMALL["gdt"], precision=prec, device=dev)) as s:
            s.autotune()
            s.set_wfc(psi0)
            s.evolve(SMALL["every"], 0)  # graphs
            s.set_wfc(psi0)
            r = s.evolve(SMALL["steps"], 0, energy_every=SMALL["every"])
            out[name + "_value"] = pts * SMALL["steps"] / (r["device_ms"] * 1e-3)
            out[name + "_energy"] = s.energy()
            out[name + "_us_per_step"] = r["device_ms"] * 1e3 / SMALL["steps"]
    out["unit"] = UNIT
    return out


# ------------------------------------------------- batched sweep ----------

# 96 independent 2D ground-state solves (seed 4): n ~ U{128,192,256,384,512},
# g ~ U[10,1000], wy/wx ~ U[0.8,1.25], box [-10,10)^2, dt = 1e-4, checks
# every 100 steps with the absolute |dE| < 1e-10 stop, fused complex64.
BATCH = dict(solves=96, sizes=(128, 192, 256, 384, 512), box=10.0, gdt=1e-4, every=100,
             thr=1e-10, seed=4)
# the sample timed both ways: steps 0..1000 (checks at 0, 100, ..., 1000)
BATCH_STEPS = 1001
# the run to convergence stops every solve at this many steps at most
BATCH_CAP = 100000


def batch_cases():
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(BATCH["seed"]))
    out = []
    for k in range(BATCH["solves"]):
        n = int(rng.choice(BATCH["sizes"]))
        g = float(rng.uniform(10.0, 1000.0))
        wy = float(rng.uniform(0.8, 1.25))
        out.append(dict(n=n, g=g, wy=wy, seed=1000 + k))
    return out


def batch_leg(G, dev, steps=BATCH_STEPS, dist=None, converge=True):
    """The 96 solves as one gpue_batch against the same solves run one after
    another through gpue_evolve (same form, same checks): steps 0..1000 both
    ways, then the batch run on until every solve has converged (|dE| < 1e-10
    between 100-step checks, capped at BATCH_CAP steps), with the sequential
    time of that run estimated from each solve's measured per-step time times
    the steps it ran.  Under several ranks each GPU takes every world-th solve
    (no communication) and the rates are all ranks' point-steps over the
    slowest rank's time."""
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    cs = [batch_cases()[i] for i in replicas.shard(BATCH["solves"], world, rank)]
    psi0 = [gauss_start(2, c["n"], BATCH["box"], c["seed"]) for c in cs]

    def params(c):
        return G.make_params(2, c["n"], BATCH["box"], wy=c["wy"], g=c["g"], gdt=BATCH["gdt"],
                             precision=G.PREC_FP32, device=dev)

    kw = dict(energy_every=BATCH["every"], threshold=BATCH["thr"], threshold_abs=True)
    solvers = [G.Solver(params(c)) for c in cs]
    conv = None
    try:
        for s, p in zip(solvers, psi0):
            s.set_wfc(p)
        with G.Batch(solvers) as b:
            b.evolve(0, 2 * BATCH["every"] + 1, autotune=True, **kw)  # tunes, captures graphs
            for s, p in zip(solvers, psi0):
                s.set_wfc(p)
            res, st = b.evolve(0, steps, **kw)
            if converge:
                for s, p in zip(solvers, psi0):
                    s.set_wfc(p)
                cres, cst = b.evolve(0, BATCH_CAP, **kw)
        batched, _, bsecs = replicas.job_rate(st["point_steps"], st["device_ms"] * 1e-3, dist,
                                              dev)
        # sequential: the same solves, one gpue_evolve call each
        seq_ms, seq_pts, seq_conv_ms = 0.0, 0.0, 0.0
        for k, (s, p, c) in enumerate(zip(solvers, psi0, cs)):
            s.set_wfc(p)
            s.evolve(2 * BATCH["every"] + 1, 0, **kw)  # graphs of this solve
            s.set_wfc(p)
            r = s.evolve(steps, 0, **kw)
            seq_ms += r["device_ms"]
            seq_pts += c["n"] ** 2 * r["steps_done"]
            if converge:
                seq_conv_ms += r["device_ms"] / r["steps_done"] * cres[k]["steps_done"]
    finally:
        for s in solvers:
            s.close()
    sequential, _, ssecs = replicas.job_rate(seq_pts, seq_ms * 1e-3, dist, dev)
    out = {"solves": BATCH["solves"], "ranks": world, "steps": steps, "value": batched,
           "unit": UNIT, "device_ms": bsecs * 1e3, "kernel_launches": st["kernel_launches"],
           "graph_launches": st["graph_launches"],
           "stopped": sum(r["early_stop"] for r in res),
           "sequential_value": sequential, "sequential_device_ms": ssecs * 1e3,
           "batched_over_sequential": batched / sequential,
           "sample": "steps 0..%d of all 96 solves (checks every 100 steps, |dE|<1e-10 "
                     "absolute stop), complex64 with FP64 reductions; sequential = the same "
                     "solves through gpue_evolve one after another (sum of their device "
                     "times)" % (steps - 1)}
    if converge:
        cval, _, csecs = replicas.job_rate(cst["point_steps"], cst["device_ms"] * 1e-3, dist,
                                           dev)
        sval, _, sconv = replicas.job_rate(cst["point_steps"], seq_conv_ms * 1e-3, dist, dev)
        steps_done = sorted(r["steps_done"] for r in cres)
        out["to_convergence"] = {
            "value": cval, "unit": UNIT, "device_ms": csecs * 1e3,
            "converged": sum(r["early_stop"] for r in cres), "cap_steps": BATCH_CAP,
            "steps_min": steps_done[0], "steps_median": steps_done[len(steps_done) // 2],
            "steps_max": steps_done[-1], "kernel_launches": cst["kernel_launches"],
            "sequential_value_estimated": sval, "sequential_device_ms_estimated": sconv * 1e3,
            "batched_over_sequential": cval / sval,
            "note": "every solve from its seeded start until |dE|<1e-10 between 100-step "
                    "checks (or the cap), converged solves frozen while the rest run on; "
                    "sequential estimated as each solve's per-step device time through "
                    "gpue_evolve (measured over steps 0..1000) times the steps it ran here"}
    return out


# -------------------------------------------------------------- serving ---

# Poisson arrivals at 200/s (seed 5): 70% 2D with n ~ U{128..1024}, 30% 3D
# with n ~ U{64..192}, each rounded up to the next compiled FFT length; half
# imaginary time (|dE| < 1e-10 between 100-step checks), half real time for
# 2000 steps with Omega ~ U[0, 0.8]; g ~ U[10, 1000]; 150 GB HBM budget.
SERVE = dict(rate=200.0, seed=5, budget=150e9, check=100, thr=1e-10, real_steps=2000,
             imag_cap=2000, requests=200)


def round_up_length(G, n, precision):
    m = n
    while not G.supported_length(m, precision):
        m += 1
    return m


def serve_requests(G):
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(SERVE["seed"]))
    t, out = 0.0, []
    for k in range(SERVE["requests"]):
        t += float(rng.exponential(1.0 / SERVE["rate"]))
        dim = 2 if rng.random() < 0.7 else 3
        n = int(rng.integers(128, 1025)) if dim == 2 else int(rng.integers(64, 193))
        n = round_up_length(G, n, G.PREC_FP32)
        gs = 0 if rng.random() < 0.5 else 1
        omega = float(rng.uniform(0.0, 0.8)) if gs == 1 else 0.0
        g = float(rng.uniform(10.0, 1000.0))
        out.append(dict(t=t, dim=dim, n=n, gstate=gs, omega=omega, g=g, seed=5000 + k,
                        box=10.0 if dim == 2 else 8.0,
                        steps=SERVE["real_steps"] if gs == 1 else SERVE["imag_cap"]))
    return out


def serve_params(G, q, precision, dev):
    return G.make_params(q["dim"], q["n"], q["box"], g=q["g"], omega=q["omega"],
                         gauge=q["omega"] != 0.0, gdt=1e-4, dt=5e-5, precision=precision,
                         device=dev)


def serve_leg(G, dev):
    """The request stream through gpue_server (fused complex64, continuous
    batching) against the same requests as sequential plain FP64 solves."""
    import threading
    import numpy as np
    reqs = serve_requests(G)
    psi0 = [gauss_start(q["dim"], q["n"], q["box"], q["seed"]) for q in reqs]
    results = {}
    # default plans: timing every fresh shape of the burst before its first
    # tick costs more (~0.6 s) than the tuned plans save over a 2000-step solve
    with G.Server(precision=G.PREC_FP32, check_steps=SERVE["check"], threshold=SERVE["thr"],
                  threshold_abs=True, hbm_budget=SERVE["budget"], device=dev,
                  autotune=False) as srv:
        t0 = time.perf_counter()

        def submitter():
            for k, q in enumerate(reqs):
                delay = q["t"] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                srv.submit(serve_params(G, q, G.PREC_FP32, dev), q["gstate"], q["steps"],
                           psi0[k], k)

        th = threading.Thread(target=submitter)
        th.start()
        deadline = time.perf_counter() + 600
        while len(results) < len(reqs) and time.perf_counter() < deadline:
            for r in srv.poll(timeout=0.5):
                results[r["tag"]] = r
        th.join()
        wall = time.perf_counter() - t0
        stats = srv.stats()
    done = [r for r in results.values() if r["status"] == 0]
    lat = np.array([r["t_done"] - r["t_submit"] for r in done])
    queue = np.array([r["t_admit"] - r["t_submit"] for r in done])
    service = np.array([r["t_done"] - r["t_admit"] for r in done])
    ok = len(done)
    # steady window: requests from the second fifth of arrivals onwards
    late = [r for r in done if r["tag"] >= len(reqs) // 5]
    lat_late = np.array([r["t_done"] - r["t_submit"] for r in late])
    # sequential plain FP64, one gpue_evolve per request, host buffers in and out
    t1 = time.perf_counter()
    for k, q in enumerate(reqs):
        with G.Solver(serve_params(G, q, G.PREC_FP64, dev)) as s:
            s.set_wfc(psi0[k])
            if q["gstate"] == 0:
                s.evolve(q["steps"], 0, energy_every=SERVE["check"], threshold=SERVE["thr"],
                         threshold_abs=True)
            else:
                s.evolve(q["steps"], 1)
            s.get_wfc()
    seq_wall = time.perf_counter() - t1
    pct = lambda a, p: float(np.percentile(a, p)) if len(a) else None  # noqa: E731
    return {"requests": len(reqs), "completed": ok, "wall_s": wall,
            "solves_per_s": ok / wall,
            "latency_p50_s": pct(lat, 50), "latency_p99_s": pct(lat, 99),
            "queue_p50_s": pct(queue, 50), "queue_p99_s": pct(queue, 99),
            "service_p50_s": pct(service, 50), "service_p99_s": pct(service, 99),
            "steady_latency_p50_s": pct(lat_late, 50), "steady_latency_p99_s": pct(lat_late, 99),
            "sequential_plain_fp64_solves_per_s": len(reqs) / seq_wall,
            "sequential_wall_s": seq_wall,
            "served_over_sequential": (ok / wall) / (len(reqs) / seq_wall),
            "device_busy_s": stats["busy_s"], "ticks": stats["ticks"],
            "worker_host_s": {"admit": stats["admit_s"], "issue": stats["issue_s"],
                              "finish": stats["finish_s"]},
            "admitted_in_tick": stats["admitted_in_tick"],
            "kernel_launches": stats["kernel_launches"],
            "point_steps_per_s": stats["point_steps"] / wall,
            "bytes_peak": stats["bytes_peak"],
            "sample": "the first %d requests of the seeded Poisson stream (arrivals over "
                      "%.2f s: an overload, the queue grows); imaginary-time solves to "
                      "|dE|<1e-10 between 100-step checks, capped at %d steps; real-time "
                      "solves %d steps; wall-clock from the first arrival to the last "
                      "result, results copied to host buffers; latency = queueing (submit "
                      "to admission) + service (admission to result); steady = requests "
                      "after the first fifth of arrivals"
                      % (len(reqs), reqs[-1]["t"], SERVE["imag_cap"], SERVE["real_steps"])}


# ------------------------------------------------------------- CPU --------

def cpu_oracle_rate(psi0, budget_s=15.0, threads=0):
    """FP64 CPU restatement (oracle) on the headline workload from the same
    initial state: a bounded sample of imaginary time steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    n = HEAD["n"]
    P = oracle.Problem(3, n, HEAD["box"], wz=HEAD["wz"], g=HEAD["g"], gdt=HEAD["gdt"],
                       threads=threads)
    psi, _, _ = P.evolve(psi0, 1, 0)  # warm-up (first-call set-up)
    t = time.time()
    psi, _, _ = P.evolve(psi, 2, 0)
    per = (time.time() - t) / 2
    # a sample of about budget_s seconds
    steps = max(1, min(100, int(budget_s / max(per, 1e-6))))
    t = time.time()
    P.evolve(psi, steps, 0)
    dt = time.time() - t
    cores = threads or os.cpu_count()
    return {"value": n ** 3 * steps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d imaginary time steps of the 256^3 ground state from the headline's "
                      "initial state (FP64, OpenMP over lines, %d threads)" % (steps, cores),
            "seconds": dt}


def gpue_cuda_build_leg():
    """GPUE's own CUDA build (oracle/_ref, compiled from the reference sources)
    timed on this GPU by its harness: evolve() on the full-size workloads with
    the step counts below, GPUE's per-step device-to-host copy of psi included
    as GPUE does it.  None when the build is absent."""
    harness = os.path.join(ROOT, "oracle", "_ref", "gpue_ref_harness")
    if not os.path.exists(harness):
        return {"unavailable": "oracle/_ref/gpue_ref_harness not built"}
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import numpy as np
    import cases
    out = {}
    for name, steps in (("cfg3_256_imag", 100), ("cfg2_1024_real_gauge", 1000),
                        ("cfg1_256_imag", 10000)):
        c = cases.case(name)
        c["gsteps" if c["gsteps"] else "esteps"] = steps
        c["energy_every"] = 0
        psi0 = cases.initial_psi(c)
        with tempfile.TemporaryDirectory() as td:
            p0 = os.path.join(td, "psi0.bin")
            psi0.tofile(p0)
            prefix = os.path.join(td, "out")
            r = subprocess.run([harness] + cases.harness_args(c, p0, prefix,
                                                              os.path.join(td, "d")),
                               stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                               timeout=600)
            if r.returncode != 0:
                out[name] = {"failed": r.stdout[-300:]}
                continue
            phase = "imag" if c["gsteps"] > 0 else "real"
            info = dict(l.split() for l in open(prefix + "_%s.txt" % phase))
        secs = float(info["evolve_s"])
        pts = c["n"] ** c["dim"]
        out[name] = {"steps": steps, "evolve_s": secs,
                     "value": pts * steps / secs, "unit": UNIT,
                     "energy": float(info["energy"])}
        del psi0
    out["note"] = ("GPUE's build (FP64, cuFFT) timed by its harness around evolve(); "
                   "cfg3 = the headline 256^3 workload, cfg2 = the 1024^2 rotating case, "
                   "cfg1 = the 256^2 ground state")
    _ = np
    return out


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    n = HEAD["n"]
    psi0 = head_state()
    P = oracle.Problem(3, n, HEAD["box"], wz=HEAD["wz"], g=HEAD["g"], gdt=HEAD["gdt"])
    budget = 150.0
    per = REF_STEPS_PER_BENCH_STEP
    psi = psi0
    # one reference bench step = one evolve call of `per` imaginary time steps
    # of the headline workload
    for _ in range(min(args.warmup, 1)):
        psi, _, _ = P.evolve(psi, per, 0)
    t0 = time.time()
    done = 0
    while done < args.steps and time.time() - t0 < budget:
        psi, _, _ = P.evolve(psi, per, 0)
        done += 1
    secs = time.time() - t0
    val = n ** 3 * per * done / secs
    cores = os.cpu_count()
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": done, "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(done, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded; the headline's initial state)", "impl": "reference",
            "config": {"workload": WORKLOAD_NAME, "grid": n,
                       "step": "one evolve call of %d imaginary time steps (the reference "
                               "arm's bench step; points x time steps / seconds is the same "
                               "metric)" % per,
                       "steps_requested": args.steps, "budget_s": budget,
                       "initial_state": "the headline's (seed 3 Gaussian, normalised)"},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "%d imaginary time steps of the headline workload "
                                       "on the FP64 CPU restatement, OpenMP over %d threads"
                                       % (done * per, cores)},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    try:
        line["gpue_cuda_build"] = gpue_cuda_build_leg()
    except Exception as e:  # the CPU arm stands without it
        line["gpue_cuda_build"] = {"unavailable": str(e)[:200]}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- main -------

def measured_peak():
    """HBM copy bandwidth (GB/s) from MEASURED_PEAKS.json, else the fallback."""
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(peaks["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_case(args):
    """Small deterministic run for ncu captures (the timed legs' kernels)."""
    import gpue_b200 as G
    if args.profile == "batch":
        # the 96-solve sweep as one batch: one persistent launch per 100-step
        # segment (checks every 100 steps), default plans
        cs = batch_cases()
        ss = [G.Solver(G.make_params(2, c["n"], BATCH["box"], wy=c["wy"], g=c["g"],
                                     gdt=BATCH["gdt"], precision=G.PREC_FP32)) for c in cs]
        try:
            for s, c in zip(ss, cs):
                s.set_wfc(gauss_start(2, c["n"], BATCH["box"], c["seed"]))
            with G.Batch(ss) as b:
                kw = dict(energy_every=BATCH["every"], threshold=BATCH["thr"],
                          threshold_abs=True)
                _, st0 = b.evolve(0, 100 * args.warmup + 1, **kw)
                _, st1 = b.evolve(0, 100 * args.steps, **kw)
        finally:
            for s in ss:
                s.close()
        print(json.dumps({"profile": "batch", "warmup_launches": st0["kernel_launches"],
                          "launches": st1["kernel_launches"], "device_ms": st1["device_ms"]}))
        return
    if args.profile.endswith("_3d"):
        # the headline workload with fixed launch shapes for the z pass (and
        # the x/y line passes of the FP64 form), so a capture does not depend
        # on timings taken under the profiler; one step is one imaginary time
        # step (3 passes complex64, 5 passes complex128)
        prec = G.PREC_FP32 if args.profile == "fp32_3d" else G.PREC_FP64
        with G.Solver(head_params(G, prec)) as s:
            for axis, lines in enumerate((2, 4, 4)):
                s.set_plan(axis, 16, 0, 0, 16, lines)
            plans = [s.plan(a) for a in range(3)]
            s.set_wfc(head_state())
            r0 = s.evolve(args.warmup, 0)
            r1 = s.evolve(args.steps, 0, step_offset=args.warmup)
        print(json.dumps({"profile": args.profile, "warmup_launches": r0["kernel_launches"],
                          "launches": r1["kernel_launches"], "device_ms": r1["device_ms"],
                          "plans": plans}))
        return
    import numpy as np
    n, box = ROT["n"], ROT["box"]
    dx = box / (n >> 1)
    x = -box + dx * np.arange(n)
    psi0 = (np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / 8.0) *
            np.exp(1j * phase_field(n, box))).astype(np.complex128)
    prec = G.PREC_FP32 if args.profile == "fp32" else G.PREC_FP64
    with G.Solver(rot_params(G, prec, 0)) as s:
        s.set_wfc(psi0)
        # here a step is 2 time steps (one x/y gauge-order cycle), so that
        # captures can pick single launches out of a short run
        r0 = s.evolve(args.warmup * 2, 1)
        r1 = s.evolve(args.steps * 2, 1, step_offset=args.warmup * 2)
    print(json.dumps({"profile": args.profile, "warmup_launches": r0["kernel_launches"],
                      "launches": r1["kernel_launches"], "device_ms": r1["device_ms"]}))


def main():
    args = parse_args()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.profile:
        profile_case(args)
        return
    import torch
    import gpue_b200 as G
    peak, peak_src = measured_peak()
    if args.only:
        legs = {"batch": lambda: batch_leg(G, 0), "serve": lambda: serve_leg(G, 0),
                "accuracy": lambda: accuracy_leg(G, 0, peak),
                "rot2d": lambda: rot2d_leg(G, torch, 0, lambda: None),
                "small2d": lambda: small2d_leg(G, 0)}
        print(json.dumps({args.only: legs[args.only]()}), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = local
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", dev))

    def barrier():
        if dist is not None:
            dist.barrier()

    psi0 = head_state()
    pts = HEAD["n"] ** 3
    res = {}
    plans = {}
    for name, prec in (("fp64", G.PREC_FP64), ("fp32", G.PREC_FP32)):
        with G.Solver(head_params(G, prec, dev)) as s:
            plans[name] = [(p["ra"], p["rb"], p["threads_per_line"], p["lines_per_cta"])
                           for p in s.autotune()]  # later solvers of this shape reuse it
            s.set_wfc(psi0)
            sampler = ClockSampler(dev) if name == "fp32" else None
            ms, launches, clocks = timed_steps(G, torch, s, args.steps, args.warmup, dev,
                                               barrier, 0, sampler=sampler)
            E = s.energy()
            # each pass kernel of a step timed alone (event pair per launch on
            # the library's stream, state restored), after the timed region
            passes = s.time_passes(0, nsteps=8)
        ms = replicas.max_over_ranks(ms, dist, dev)
        res[name] = dict(ms=ms, launches=launches, clocks=clocks, E=E, passes=passes)

    tsteps = args.steps * STEPS_PER_BENCH_STEP
    v32 = world * pts * tsteps / (res["fp32"]["ms"] * 1e-3)
    v64 = world * pts * tsteps / (res["fp64"]["ms"] * 1e-3)
    # legs every rank takes part in (same collectives, same order)
    e2e = e2e_leg(G, torch, psi0, dev, dist=dist)
    batched = None if args.quick else batch_leg(G, dev, dist=dist)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    # roofline of the dominant kernel: of the step's pass kernels (each reads
    # and writes the complex64 field once: 2 * 8 bytes per point), the one
    # with the longest duration, timed alone on the library's stream
    per_time_step_s = res["fp32"]["ms"] * 1e-3 / tsteps
    kind_names = {0: "x line pass", 1: "y line pass", 2: "z tile pass (Fz K Iz)",
                  3: "forward XY tile pass ([scale] V/2 Fx Fy)",
                  4: "inverse XY tile pass (Ix Iy V/2 norm)"}
    passes = res["fp32"]["passes"]
    dom_kind, dom_us = max(passes, key=lambda kv: kv[1])
    achieved = 2 * 8 * pts / (dom_us * 1e-6) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            per_kind = json.load(open(tpath)).get("head_fp32_pass_bytes_per_launch", {})
            traffic = per_kind.get({3: "forward_xy", 2: "z", 4: "inverse_xy"}.get(dom_kind))
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "kernel": kind_names.get(dom_kind, str(dom_kind)),
                "kernel_us": dom_us,
                "passes_us": [[kind_names.get(k, str(k)), us] for k, us in passes],
                "peak_source": (peak_src + " (MEASURED_PEAKS.json hbm_gbs)")
                if peak_src == "measured" else "fallback 6.65 TB/s",
                "step_frac_48B": 48 * pts / per_time_step_s / 1e9 / peak,
                "alg_frac_80B": 80 * pts / per_time_step_s / 1e9 / peak,
                "note": "achieved = 256 MiB algorithmic bytes per launch (one read and one "
                        "write of the complex64 field) / the dominant pass kernel's mean "
                        "duration, timed with CUDA events on the library's stream after the "
                        "timed region (gpue_time_passes: 8 steps, one event pair per launch); "
                        "step_frac_48B counts the three-pass step's 48 B per point against "
                        "the bench step time, alg_frac_80B the five-pass line schedule's "
                        "80 B per point; traffic = dram read+write bytes per launch of that "
                        "kernel from an ncu capture (profiles/traffic.json), not measured "
                        "in this run"}

    # rank 0 alone; the CPU baseline and the extra legs only at N = 1
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cpu = cpu_oracle_rate(psi0)
    extra = {}
    if not args.quick and world == 1:
        extra["accuracy_3d"] = accuracy_leg(G, dev, peak)
        extra["rotating_2d"] = rot2d_leg(G, torch, dev, barrier)
        extra["small_2d_fp64"] = small2d_leg(G, dev)
        extra["serving"] = serve_leg(G, dev)
    line = {
        "metric": METRIC, "value": v32, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": res["fp32"]["ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian start, normalised)",
        "config": {"workload": WORKLOAD_NAME, "grid": HEAD["n"], "form": "fused complex64, "
                   "FP64-formed operator phases rounded once, FP64 reductions",
                   "step": "one gpue_evolve call of %d imaginary time steps"
                           % STEPS_PER_BENCH_STEP,
                   "l2": "inputs larger than L2: the 128 MiB complex64 field (256 MiB "
                         "complex128) exceeds the 126 MB L2, no flush",
                   "plans": plans,
                   "parallelism": "replicas" if world > 1 else "single"},
        "plain_fp64": {"value": v64, "ms_per_step": res["fp64"]["ms"] / args.steps,
                       "fused_fp32_over_plain_fp64": v32 / v64,
                       "E_after_timed_steps": res["fp64"]["E"]},
        "E_fp32_after_timed_steps": res["fp32"]["E"],
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
        "batched_sweep": batched,
        "clocks": res["fp32"]["clocks"],
        "gpu_launches": res["fp32"]["launches"],
    }
    line.update(extra)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
