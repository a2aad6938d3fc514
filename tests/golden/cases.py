"""Seeded parity cases shared by the golden-fixture generator and the tests.

Every case is a GPUE run in hbar = m = 1 units on a square/cubic grid
x_i = -box + i*dx, dx = box/(n/2) (GPUE's generate_p_space), with a harmonic
trap, optional rotation gauge A = omega*(-y wx, x wy) and optional nonlinear
term.  Initial wavefunctions are built from numpy PCG64 streams so the
fixtures only need to store outputs; each fixture records a checksum of its
input so a change in the generator is caught.
"""

import hashlib

import numpy as np

CASES = {
    # 2D imaginary time, nonlinear, renormalised every step
    "g2d_imag_n64": dict(dim=2, n=64, box=10.0, g=100.0, gsteps=500, seed=11,
                         init="gauss", energy_every=100),
    # 2D imaginary time with the rotation gauge (imaginary-time gauge operators)
    "g2d_imag_gauge_n64": dict(dim=2, n=64, box=8.0, g=200.0, omega=0.5, gauge=True,
                               gsteps=400, seed=12, init="gauss", energy_every=100),
    # 2D real time with the rotation gauge, both gauge orders alternate
    "g2d_real_gauge_n64": dict(dim=2, n=64, box=8.0, g=200.0, omega=0.7, gauge=True,
                               dt=5e-5, esteps=400, seed=13, init="phase", energy_every=100),
    # 2D real time, linear Schroedinger, anisotropic trap
    "g2d_real_lin_n32": dict(dim=2, n=32, box=6.0, wy=1.3, gpe=False, dt=1e-4, esteps=300,
                             seed=14, init="phase", energy_every=100),
    # 3D imaginary time, anisotropic trap
    "g3d_imag_n16": dict(dim=3, n=16, box=6.0, wz=4.0, g=100.0, gsteps=200, seed=15,
                         init="gauss", energy_every=50),
    # 3D real time with the gauge (x,y,z then z,y,x orders)
    "g3d_real_gauge_n16": dict(dim=3, n=16, box=6.0, wz=2.0, g=50.0, omega=0.5, gauge=True,
                               dt=1e-4, esteps=200, seed=16, init="phase", energy_every=50),
    # 3D imaginary time with the gauge
    "g3d_imag_gauge_n32": dict(dim=3, n=32, box=6.0, wz=2.0, g=100.0, omega=0.3, gauge=True,
                               gsteps=100, seed=17, init="gauss", energy_every=50),
    # 2D imaginary time with GPUE's gauge ramp (-R 1 and -R 2): the gauge
    # factors raised to a cumulative power every step
    "g2d_imag_ramp1_n64": dict(dim=2, n=64, box=8.0, g=200.0, omega=0.5, gauge=True,
                               gdt=2e-4, gsteps=150, seed=18, init="gauss", energy_every=50,
                               ramp=True, ramp_type=1),
    "g2d_imag_ramp2_n64": dict(dim=2, n=64, box=8.0, g=150.0, omega=0.6, gauge=True,
                               gdt=2e-4, gsteps=120, seed=19, init="gauss", energy_every=40,
                               ramp=True, ramp_type=2),
    # the 256^2 imaginary-time workload: g=100, gdt=1e-4, 10000 steps
    "cfg1_256_imag": dict(dim=2, n=256, box=10.0, g=100.0, gsteps=10000, seed=1,
                          init="gauss", energy_every=1000),
}

# Full-size workloads timed on GPUE's own build (make_golden.py --timing): the
# 1024^2 rotating real-time case and the 256^3 ground state, with the step
# counts used for timing.
CASES.update({
    "cfg2_1024_real_gauge": dict(dim=2, n=1024, box=16.0, g=500.0, omega=0.7, gauge=True,
                                 dt=5e-5, esteps=20000, seed=2, init="phase"),
    "cfg3_256_imag": dict(dim=3, n=256, box=12.0, wz=4.0, g=1000.0, gsteps=5000, seed=3,
                          init="gauss"),
})
TIMING = [("cfg1_256_imag", 10000), ("cfg2_1024_real_gauge", 1000), ("cfg3_256_imag", 100)]
# Full-size runs kept as digests (make_golden.py --digest) with their step counts.
DIGESTS = {"cfg2_1024_real_gauge": 1000, "cfg3_256_imag": 100}
FIXTURES = [k for k in CASES if not k.startswith(("cfg2", "cfg3"))]

DEFAULTS = dict(wx=1.0, wy=1.0, wz=1.0, gamma=1.0, g=0.0, gpe=True, omega=0.0, gauge=False,
                gdt=1e-4, dt=1e-4, gsteps=0, esteps=0, energy_every=0, ramp=False, ramp_type=1)


def case(name):
    c = dict(DEFAULTS)
    c.update(CASES[name])
    return c


def coords(c):
    n, box = c["n"], c["box"]
    dx = box / (n >> 1)
    x = -box + dx * np.arange(n)
    return x, dx


def initial_psi(c):
    """complex128 array shaped (n, n) or (n, n, n) [z, y, x], normalised."""
    dim, n = c["dim"], c["n"]
    x, dx = coords(c)
    rng = np.random.Generator(np.random.PCG64(c["seed"]))
    grids = np.meshgrid(*([x] * dim), indexing="ij")
    r2 = sum(gi * gi for gi in grids)
    psi = np.exp(-r2 / 2.0) * (1.0 + 0.01 * rng.standard_normal(r2.shape))
    psi = psi.astype(np.complex128)
    if c["init"] == "phase":
        theta = 2 * np.pi * rng.random(r2.shape)
        k = 2 * np.pi * np.fft.fftfreq(n, d=dx)
        kg = np.meshgrid(*([k] * dim), indexing="ij")
        k2 = sum(ki * ki for ki in kg)
        sm = np.real(np.fft.ifftn(np.fft.fftn(theta) * np.exp(-0.5 * k2 * 0.25)))
        psi = psi * np.exp(1j * sm)
    dV = dx ** dim
    psi /= np.sqrt(np.sum(np.abs(psi) ** 2) * dV)
    return np.ascontiguousarray(psi)


def checksum(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def harness_args(c, psi0_path, out_prefix, data_dir):
    a = ["dim=%d" % c["dim"], "n=%d" % c["n"], "box=%r" % c["box"], "wx=%r" % c["wx"],
         "wy=%r" % c["wy"], "wz=%r" % c["wz"], "gamma=%r" % c["gamma"], "g=%r" % c["g"],
         "gpe=%d" % int(c["gpe"]), "omega=%r" % c["omega"], "gauge=%d" % int(c["gauge"]),
         "gdt=%r" % c["gdt"], "dt=%r" % c["dt"], "gsteps=%d" % c["gsteps"],
         "esteps=%d" % c["esteps"], "energy_every=%d" % c["energy_every"],
         "ramp=%d" % int(c["ramp"]), "ramp_type=%d" % c["ramp_type"],
         "psi0=" + psi0_path, "out=" + out_prefix, "data=" + data_dir]
    return a


# 2D states for the vortex finder (Tracker::findVortex): square n x n grids,
# x fastest, with GPUE's x grid.  "imprint" multiplies a Gaussian by
# (x - xk) + i qk (y - yk) factors at seeded positions (charges +-1; one of
# them sits exactly on a grid node, so psi is 0 there), plus 1% noise;
# "noise" is a random phase field whose plaquettes wind often and in
# neighbouring pairs, exercising the rule that skips the plaquette after a
# mark; "ring" puts the search radius through a ring of vortices.
VORTEX_CASES = {
    "vtx_imprint_n128": dict(n=128, box=8.0, radius=5.0, seed=31, kind="imprint", nv=14),
    "vtx_noise_n64": dict(n=64, box=6.0, radius=4.5, seed=32, kind="noise"),
    "vtx_ring_n96": dict(n=96, box=8.0, radius=3.0, seed=33, kind="ring", nv=10),
    "vtx_imprint_n256": dict(n=256, box=10.0, radius=9.0, seed=34, kind="imprint", nv=40),
}


def grid_x(n, box):
    """generate_p_space's x: -box + i dx on the first half, i dx on the second."""
    dx = box / (n >> 1)
    x = np.empty(n)
    h = n // 2
    x[:h] = -box + np.arange(h) * dx
    x[h:] = np.arange(h) * dx
    return x


def vortex_psi(v):
    """complex128 (n, n) [y, x] state of a VORTEX_CASES entry."""
    n, box = v["n"], v["box"]
    rng = np.random.Generator(np.random.PCG64(v["seed"]))
    x = grid_x(n, box)
    X, Y = np.meshgrid(x, x)
    if v["kind"] == "noise":
        amp = 0.5 + rng.random((n, n))
        return np.ascontiguousarray(amp * np.exp(2j * np.pi * rng.random((n, n))))
    psi = np.exp(-(X * X + Y * Y) / (0.5 * box) ** 2).astype(np.complex128)
    if v["kind"] == "ring":
        ang = 2 * np.pi * np.arange(v["nv"]) / v["nv"] + 0.1
        pos = np.stack([v["radius"] * np.cos(ang), v["radius"] * np.sin(ang)], 1)
        q = np.where(np.arange(v["nv"]) % 2 == 0, 1, -1)
    else:
        pos = (rng.random((v["nv"], 2)) - 0.5) * 1.4 * box
        pos[0] = (x[n // 2 + 3], x[n // 2 - 5])  # on a grid node
        q = rng.choice([-1, 1], v["nv"])
    for (xk, yk), qk in zip(pos, q):
        psi *= (X - xk) + 1j * qk * (Y - yk)
    psi *= 1.0 + 0.01 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    return np.ascontiguousarray(psi / np.abs(psi).max())


def vortex_harness_args(v, psi0_path, out_prefix):
    return ["mode=vortex", "n=%d" % v["n"], "box=%r" % v["box"], "radius=%r" % v["radius"],
            "psi0=" + psi0_path, "out=" + out_prefix]


# Equation-AST inputs pinned to GPUE's own parser (make_golden.py --ast runs
# the harness's host-only mode=ast on them and stores ast_gpue.json).  The
# doubles stand for Grid values the expressions may name.
AST_DOUBLES = {"omega": 0.7, "omegaX": 1.25, "omegaY": 0.8, "mass": 2.0, "xMax": 10.0,
               "fudge": 0.0, "rad": 10.0, "omegaR": 7071.0}

AST_CORPUS = [
    "(((3*x)+7)+(5-7)+cos(0)*1)+pow(120,2)",
    "x-y-z",
    "x-y+z",
    "2*x-3",
    "x/y*z",
    "x^2",
    "pow(x,3)+pow(y,2)",
    "exp(0-x)",
    "sqrt(x*x+y*y)",
    "cos(omega*t)*x",
    "0.5*mass*((omegaX*x)*(omegaX*x)+(omegaY*y)*(omegaY*y))",
    "rad*omegaR*x*y*z",
    "((x))",
    "(x+1)*(y-2)",
    "sin(x)*cos(y)+tan(z)",
    "jn(0,x)+yn(1,y)",
    "1.5+2.25*x",
    "[x+y]*2",
    "x*y*omega*omegaX*30000",
    "((3*x)+(y-(2*z)))/(1+t)",
    "k2n(2,x)",
    "exp(0-t)*sqrt(x)",
]
# Expressions GPUE's parse_eqn rejects (it prints "No value ... found!" and
# exits): a two-argument function nested inside another function's argument.
AST_REJECTED = ["sqrt(pow(x,2)+pow(y,2))", "sqrt(pow(x,2))"]

# Parameter-file texts: parse_param_file's line rules (continuations, the
# m|A|^2/2 suffix on V unless it is last, entries naming earlier entries).
AST_PARAM_TEXTS = {
    "rotation_gauge": "Ax = 0-y*omega\nAy = x*omega\nAz = 0\nV = 0.5*(x*x+y*y)\nK = 1\n",
    "continued_lines": ("Ax = 0\nAy = 0\nAz = 0\nV = 0.5*mass*\n(omegaX*omegaX*x*x\n"
                        "+omegaY*omegaY*y*y)\nK = cos(omega*t)\n"),
    "time_gauge": ("Ax = 0-y*omega*cos(omega*t)\nAy = x*omega\nAz = 0\n"
                   "V = 0.5*(x*x+y*y)\nK = 1\n"),
    "named_entries": "w = 2\nAx = 0\nAy = 0\nAz = 0\nV = w*w*x*x\nK = x\n",
}
# GPUE's own parameter files, read from the reference checkout when the
# fixture is made and stored in it with their parse.
AST_REFERENCE_FILES = ["src/example.cfg", "src/gauge.cfg"]
