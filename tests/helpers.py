"""Shared helpers for the parity tests."""
import json
import os

import numpy as np

import cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return d["psi"], json.loads(str(d["meta"]))


def dV(c):
    return (c["box"] / (c["n"] >> 1)) ** c["dim"]


def l2(a, b, c):
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) * dV(c)))


def steps_gstate(c):
    return (c["gsteps"], 0) if c["gsteps"] else (c["esteps"], 1)


def oracle_problem(c, **kw):
    import oracle
    return oracle.Problem(c["dim"], c["n"], c["box"], wx=c["wx"], wy=c["wy"], wz=c["wz"],
                          gamma=c["gamma"], g=c["g"], gpe=c["gpe"], omega=c["omega"],
                          gauge=c["gauge"], gdt=c["gdt"], dt=c["dt"],
                          energy_every=c["energy_every"], ramp=c.get("ramp", False),
                          ramp_type=c.get("ramp_type", 1), **kw)


def product_params(c, precision):
    import gpue_b200 as G
    return G.make_params(c["dim"], c["n"], c["box"], wx=c["wx"], wy=c["wy"], wz=c["wz"],
                         gamma=c["gamma"], g=c["g"], gpe=c["gpe"], omega=c["omega"],
                         gauge=c["gauge"], gdt=c["gdt"], dt=c["dt"], precision=precision,
                         ramp=c.get("ramp", False), ramp_type=c.get("ramp_type", 1))


def run_product(c, precision, psi0=None, **evolve_kw):
    import gpue_b200 as G
    steps, gs = steps_gstate(c)
    with G.Solver(product_params(c, precision)) as s:
        s.set_wfc(cases.initial_psi(c) if psi0 is None else psi0)
        r = s.evolve(steps, gs, energy_every=c["energy_every"], **evolve_kw)
        psi = s.get_wfc()
        E = s.energy()
    return psi, E, r
