"""Generate the golden fixtures by running GPUE's own CUDA build.

Needs a GPU and oracle/_ref/gpue_ref_harness (built here from the reference
sources by ``make -C oracle ref``).  For each case in cases.py it writes the
seeded initial wavefunction, runs the harness (GPUE's parseArgs, init,
set_variables, evolve and energy_calc), and stores the final wavefunction and
energy as ``<case>.npz`` in --outdir, plus the harness wall time.

    python tests/golden/make_golden.py --outdir tests/golden [case ...]

With --vortex it instead runs the harness's host-only findVortex mode (no GPU
needed) on each VORTEX_CASES state and stores the marker array and the count
as ``<case>.npz``.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import cases  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "gpue_ref_harness")


def run_case(name, outdir):
    c = cases.case(name)
    psi0 = cases.initial_psi(c)
    with tempfile.TemporaryDirectory() as td:
        p0 = os.path.join(td, "psi0.bin")
        psi0.tofile(p0)
        prefix = os.path.join(td, "out")
        data = os.path.join(td, "data")
        t0 = time.time()
        r = subprocess.run([HARNESS] + cases.harness_args(c, p0, prefix, data),
                           stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                           timeout=1800)
        wall = time.time() - t0
        if r.returncode != 0:
            print(r.stdout[-3000:])
            raise RuntimeError("harness failed for %s" % name)
        phase = "imag" if c["gsteps"] > 0 else "real"
        psi = np.fromfile(prefix + "_%s.bin" % phase, dtype=np.complex128)
        info = {}
        for line in open(prefix + "_%s.txt" % phase):
            k, v = line.split()
            info[k] = float(v)
        stopped = [l for l in r.stdout.splitlines() if "Stopping early" in l]
    psi = psi.reshape(psi0.shape)
    meta = dict(case=name, params=c, input_sha=cases.checksum(psi0), energy=info["energy"],
                last_check_energy=info["last_check_energy"], harness_wall_s=wall,
                evolve_s=info.get("evolve_s"),
                early_stop_line=stopped[0] if stopped else "")
    np.savez_compressed(os.path.join(outdir, name + ".npz"), psi=psi,
                        meta=np.array(json.dumps(meta)))
    print(json.dumps(dict(case=name, energy=info["energy"], wall_s=round(wall, 3))))


def run_vortex_case(name, outdir):
    v = cases.VORTEX_CASES[name]
    psi = cases.vortex_psi(v)
    with tempfile.TemporaryDirectory() as td:
        p0 = os.path.join(td, "psi0.bin")
        psi.tofile(p0)
        prefix = os.path.join(td, "out")
        r = subprocess.run([HARNESS] + cases.vortex_harness_args(v, p0, prefix),
                           stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                           timeout=600)
        if r.returncode != 0:
            print(r.stdout[-3000:])
            raise RuntimeError("harness failed for %s" % name)
        marker = np.fromfile(prefix + "_vortex.bin", dtype=np.int32).reshape(psi.shape)
        found = int(open(prefix + "_vortex.txt").read().split()[1])
    meta = dict(case=name, params=v, input_sha=cases.checksum(psi), found=found)
    np.savez_compressed(os.path.join(outdir, name + ".npz"), marker=marker.astype(np.int8),
                        meta=np.array(json.dumps(meta)))
    print(json.dumps(dict(case=name, found=found)))


def time_case(name, steps):
    """Time GPUE's evolve() on a full-size configuration (no fixture kept)."""
    c = cases.case(name)
    c["gsteps" if c["gsteps"] else "esteps"] = steps
    psi0 = cases.initial_psi(c)
    with tempfile.TemporaryDirectory() as td:
        p0 = os.path.join(td, "psi0.bin")
        psi0.tofile(p0)
        prefix = os.path.join(td, "out")
        r = subprocess.run([HARNESS] + cases.harness_args(c, p0, prefix, os.path.join(td, "d")),
                           stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                           timeout=3600)
        if r.returncode != 0:
            print(r.stdout[-3000:])
            raise RuntimeError("harness failed for %s" % name)
        phase = "imag" if c["gsteps"] > 0 else "real"
        info = dict(l.split() for l in open(prefix + "_%s.txt" % phase))
    pts = c["n"] ** c["dim"]
    secs = float(info["evolve_s"])
    print(json.dumps(dict(timing=name, n=c["n"], dim=c["dim"], steps=steps, evolve_s=secs,
                          grid_point_steps_per_s=pts * steps / secs,
                          energy=float(info["energy"]))))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--outdir", default=HERE)
    ap.add_argument("--timing", action="store_true",
                    help="time GPUE's evolve on the full-size configurations instead")
    ap.add_argument("--vortex", action="store_true",
                    help="findVortex fixtures (host code only, no GPU)")
    ap.add_argument("names", nargs="*")
    a = ap.parse_args()
    if a.vortex:
        os.makedirs(a.outdir, exist_ok=True)
        for name in (a.names or list(cases.VORTEX_CASES)):
            run_vortex_case(name, a.outdir)
        return
    if a.timing:
        for name, steps in cases.TIMING:
            time_case(name, steps)
        return
    os.makedirs(a.outdir, exist_ok=True)
    for name in (a.names or cases.FIXTURES):
        run_case(name, a.outdir)


if __name__ == "__main__":
    main()
