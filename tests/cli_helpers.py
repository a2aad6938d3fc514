"""Running the gpue command line (gpue_b200/host) from the tests."""
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "gpue_b200", "gpue")


def ensure_cli():
    if not os.path.exists(CLI):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "gpue_b200"), "gpue"])
    return CLI


def run(args, data_dir, check=True):
    cmd = [ensure_cli(), "-d", str(data_dir)] + [str(a) for a in args]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    if check and p.returncode != 0:
        raise AssertionError("gpue failed (%d): %s %s" % (p.returncode, p.stdout[-2000:],
                                                          p.stderr[-2000:]))
    return p


def params(args, data_dir):
    out = run(list(args) + ["--print-params"], data_dir).stdout
    d = {}
    for line in out.splitlines():
        if "=" in line:
            k, v = line.split("=", 1)
            d[k] = float(v) if any(ch in v for ch in ".e") else int(v)
    return d


def read_wfc(data_dir, name, step, shape):
    re = np.loadtxt(os.path.join(str(data_dir), "%s_%d" % (name, step)))
    im = np.loadtxt(os.path.join(str(data_dir), "%si_%d" % (name, step)))
    return (re + 1j * im).reshape(shape)


def write_wfc(data_dir, psi):
    """GPUE's -r input files: wfc_load and wfci_load, one %.16e per line."""
    np.savetxt(os.path.join(str(data_dir), "wfc_load"), psi.real.ravel(), fmt="%.16e")
    np.savetxt(os.path.join(str(data_dir), "wfci_load"), psi.imag.ravel(), fmt="%.16e")
