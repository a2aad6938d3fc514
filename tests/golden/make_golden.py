"""Generate the golden fixtures by running GPUE's own CUDA build.

Needs a GPU and oracle/_ref/gpue_ref_harness (built here from the reference
sources by ``make -C oracle ref``).  For each case in cases.py it writes the
seeded initial wavefunction, runs the harness (GPUE's parseArgs, init,
set_variables, evolve and energy_calc), and stores the final wavefunction and
energy as ``<case>.npz`` in --outdir, plus the harness wall time.

    python tests/golden/make_golden.py --outdir tests/golden [case ...]

With --digest it runs the full-size 1024^2 rotating real-time case (1000
steps) and the 256^3 ground state (100 steps) and keeps a digest of each final
state (energy, norm, per-row or per-plane L2 norms, a seeded sample of 4096
values) as ``<case>_digest.npz``: the full states are too large to commit.

With --ast it runs the harness's host-only parser mode (no GPU needed) on the
AST corpus and parameter texts of cases.py and on GPUE's own example
parameter files (read from $GPUE_REFERENCE_DIR, default /root/reference) and
stores GPUE's flat node arrays as ``ast_gpue.json``.

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


def parse_ast_output(path):
    """prefix_ast.txt of the harness -> [{name, count, time, nodes}]."""
    out = []
    for line in open(path):
        f = line.split()
        if f[0] == "entry":
            out.append(dict(name=f[1], count=int(f[2]), time=int(f[3]), nodes=[]))
        else:
            out[-1]["nodes"].append([float.fromhex(f[0])] + [int(v) for v in f[1:]])
    return out


def run_ast(outdir):
    """GPUE's parse_eqn/tree_to_array on the AST corpus and parameter texts."""
    ref = os.environ.get("GPUE_REFERENCE_DIR", "/root/reference")
    res = dict(doubles=cases.AST_DOUBLES, corpus=[], param_files=[])
    with tempfile.TemporaryDirectory() as td:
        dpath = os.path.join(td, "doubles.txt")
        with open(dpath, "w") as f:
            for k, v in cases.AST_DOUBLES.items():
                f.write("%s %r\n" % (k, v))
        epath = os.path.join(td, "exprs.txt")
        with open(epath, "w") as f:
            f.write("\n".join(cases.AST_CORPUS) + "\n")
        prefix = os.path.join(td, "corpus")
        subprocess.run([HARNESS, "mode=ast", "doubles=" + dpath, "exprs=" + epath,
                        "out=" + prefix], check=True, timeout=120)
        for expr, e in zip(cases.AST_CORPUS, parse_ast_output(prefix + "_ast.txt")):
            res["corpus"].append(dict(expr=expr, count=e["count"], time=e["time"],
                                      nodes=e["nodes"]))
        res["rejected"] = []
        for expr in cases.AST_REJECTED:
            with open(epath, "w") as f:
                f.write(expr + "\n")
            r = subprocess.run([HARNESS, "mode=ast", "doubles=" + dpath, "exprs=" + epath,
                                "out=" + prefix], stdout=subprocess.PIPE,
                               stderr=subprocess.STDOUT, text=True, timeout=120)
            res["rejected"].append(dict(expr=expr, exit_code=r.returncode,
                                        message=r.stdout.strip()[-200:]))
        texts = dict(cases.AST_PARAM_TEXTS)
        for rel in cases.AST_REFERENCE_FILES:
            texts[rel] = open(os.path.join(ref, rel)).read()
        for name, text in texts.items():
            ppath = os.path.join(td, "param.cfg")
            with open(ppath, "w") as f:
                f.write(text)
            prefix = os.path.join(td, "param")
            subprocess.run([HARNESS, "mode=ast", "doubles=" + dpath, "param=" + ppath,
                            "out=" + prefix], check=True, timeout=120)
            res["param_files"].append(dict(name=name, text=text,
                                           entries=parse_ast_output(prefix + "_ast.txt")))
    with open(os.path.join(outdir, "ast_gpue.json"), "w") as f:
        json.dump(res, f, indent=0)
    print(json.dumps(dict(ast_corpus=len(res["corpus"]),
                          param_files=len(res["param_files"]))))


def digest(psi, c, nsample=4096, seed=99):
    """A compact record of a full-size state: sum |psi|^2 dV, the L2 norm of every
    row (2D) or z-plane (3D), and a fixed-seed sample of values with their flat
    indices (x fastest)."""
    dV = (c["box"] / (c["n"] >> 1)) ** c["dim"]
    a2 = np.abs(psi) ** 2
    axes = tuple(range(1, psi.ndim))
    slab = np.sqrt(a2.sum(axis=axes) * dV)
    rng = np.random.Generator(np.random.PCG64(seed))
    idx = np.sort(rng.choice(psi.size, size=nsample, replace=False)).astype(np.int64)
    return dict(norm=float(a2.sum() * dV), slab_norms=slab, sample_idx=idx,
                sample=psi.reshape(-1)[idx].copy())


def time_case(name, steps, outdir=None):
    """Time GPUE's evolve() on a full-size configuration; with outdir, keep a
    digest of its final state as ``<name>_digest.npz``."""
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
        psi = None
        if outdir:
            psi = np.fromfile(prefix + "_%s.bin" % phase, dtype=np.complex128)
            psi = psi.reshape(psi0.shape)
    pts = c["n"] ** c["dim"]
    secs = float(info["evolve_s"])
    rec = dict(timing=name, n=c["n"], dim=c["dim"], steps=steps, evolve_s=secs,
               grid_point_steps_per_s=pts * steps / secs, energy=float(info["energy"]))
    if psi is not None:
        d = digest(psi, c)
        meta = dict(case=name, params=c, input_sha=cases.checksum(psi0),
                    energy=float(info["energy"]),
                    last_check_energy=float(info["last_check_energy"]), evolve_s=secs,
                    norm=d["norm"])
        np.savez_compressed(os.path.join(outdir, name + "_digest.npz"),
                            slab_norms=d["slab_norms"], sample_idx=d["sample_idx"],
                            sample=d["sample"], meta=np.array(json.dumps(meta)))
        rec["norm"] = d["norm"]
    print(json.dumps(rec))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--outdir", default=HERE)
    ap.add_argument("--timing", action="store_true",
                    help="time GPUE's evolve on the full-size configurations instead")
    ap.add_argument("--digest", action="store_true",
                    help="run the full-size configurations of cases.DIGESTS and keep a "
                         "digest of each final state (<case>_digest.npz)")
    ap.add_argument("--ast", action="store_true",
                    help="GPUE's equation parser on the AST corpus (host code only, no GPU)")
    ap.add_argument("--vortex", action="store_true",
                    help="findVortex fixtures (host code only, no GPU)")
    ap.add_argument("names", nargs="*")
    a = ap.parse_args()
    if a.ast:
        os.makedirs(a.outdir, exist_ok=True)
        run_ast(a.outdir)
        return
    if a.vortex:
        os.makedirs(a.outdir, exist_ok=True)
        for name in (a.names or list(cases.VORTEX_CASES)):
            run_vortex_case(name, a.outdir)
        return
    if a.timing or a.digest:
        if a.digest:
            os.makedirs(a.outdir, exist_ok=True)
        for name, steps in cases.TIMING:
            if a.digest and name not in cases.DIGESTS:
                continue
            time_case(name, steps, a.outdir if a.digest else None)
        return
    os.makedirs(a.outdir, exist_ok=True)
    for name in (a.names or cases.FIXTURES):
        run_case(name, a.outdir)


if __name__ == "__main__":
    main()
