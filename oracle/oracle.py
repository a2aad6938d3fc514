"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the CPU FP64 oracle.

Only tests/, the smoke check and the CPU-baseline leg of bench.py use this
module.  It wraps liboracle.so (built from gpe_oracle.cpp by this directory's
Makefile) and offers a numpy-level ``Problem`` that mirrors how GPUE sets a
run up (grids from generate_p_space, harmonic V and rotation gauge from
generate_fields) in hbar = m = 1 units.
"""

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class Node(C.Structure):
    _fields_ = [("val", C.c_double), ("is_dynamic", C.c_int32), ("var", C.c_int32),
                ("left", C.c_int32), ("right", C.c_int32), ("op_num", C.c_int32)]


class Cfg(C.Structure):
    _fields_ = [("dimnum", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("hbar", C.c_double), ("gN", C.c_double), ("gdt", C.c_double), ("dt", C.c_double),
                ("gpe", C.c_int32), ("corotating", C.c_int32), ("ramp", C.c_int32),
                ("ramp_type", C.c_int32), ("omega", C.c_double), ("threads", C.c_int32),
                ("energy_every", C.c_int32), ("threshold", C.c_double),
                ("threshold_abs", C.c_int32),
                ("ast_V", C.POINTER(Node)), ("ast_K", C.POINTER(Node)),
                ("ast_Ax", C.POINTER(Node)), ("ast_Ay", C.POINTER(Node)),
                ("ast_Az", C.POINTER(Node))]


class Result(C.Structure):
    _fields_ = [("steps_done", C.c_int32), ("early_stop", C.c_int32),
                ("n_energies", C.c_int32), ("energy", C.c_double)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
        L = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        L.orc_evolve.argtypes = [C.POINTER(Cfg)] + [dp] * 8 + [dp, C.c_int, C.c_int, dp,
                                                               C.POINTER(Result)]
        L.orc_evolve.restype = C.c_int
        L.orc_energy.argtypes = [C.POINTER(Cfg)] + [dp] * 6
        L.orc_energy.restype = C.c_double
        L.orc_fft1d.argtypes = [dp, C.c_int, C.c_int, C.c_long, C.c_long, C.c_int]
        L.orc_axis_grid.argtypes = [C.c_int, C.c_double, dp, dp]
        L.orc_fields.argtypes = ([C.c_int] * 4 + [dp] * 6 + [C.c_double] * 10 + [C.c_int]
                                 + [dp] * 5)
        L.orc_ast_eval.argtypes = [C.POINTER(Node)] + [C.c_double] * 4
        ip = C.POINTER(C.c_int)
        L.orc_find_vortex.argtypes = [dp, C.c_int, dp, C.c_double, ip, ip]
        L.orc_find_vortex.restype = C.c_int
        L.orc_ast_eval.restype = C.c_double
        L.orc_std_wfc.argtypes = [C.c_int] * 3 + [dp] * 3 + [C.c_double] * 5 + [dp]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def fft1d(data, sign, axis=-1):
    """Unnormalised DFT along one axis of a complex128 array (copy)."""
    a = np.ascontiguousarray(np.moveaxis(np.asarray(data, np.complex128), axis, -1)).copy()
    n = a.shape[-1]
    lib().orc_fft1d(_p(a.view(np.float64)), n, a.size // n, 1, n, sign)
    return np.moveaxis(a, -1, axis)


def axis_grid(n, xmax):
    x = np.zeros(n)
    p = np.zeros(n)
    lib().orc_axis_grid(n, xmax, _p(x), _p(p))
    return x, p


def nodes_array(arr):
    """ctypes array of Node from tree_to_array rows (val, dyn, var, l, r, op)."""
    out = (Node * len(arr))()
    for i, (v, d, var, l, r, op) in enumerate(arr):
        out[i] = Node(v, d, var, l, r, op)
    return out


class Problem:
    """A GPUE run in hbar = m = 1 units: grid, harmonic trap, rotation gauge."""

    def __init__(self, dim, n, box, wx=1.0, wy=1.0, wz=1.0, gamma=1.0, g=0.0, gpe=True,
                 omega=0.0, gauge=False, gdt=1e-4, dt=1e-4, hbar=1.0, mass=1.0,
                 energy_every=0, threshold=-1.0, threshold_abs=False, ramp=False,
                 ramp_type=1, threads=0, shifts=(0.0, 0.0, 0.0)):
        self.dim, self.n = dim, n
        self.nx = n
        self.ny = n if dim > 1 else 1
        self.nz = n if dim > 2 else 1
        self.box = box
        self.x, self.px = axis_grid(self.nx, box)
        if dim > 1:
            self.y, self.py = axis_grid(self.ny, box)
        else:
            self.y, self.py = np.zeros(1), np.zeros(1)
        if dim > 2:
            self.z, self.pz = axis_grid(self.nz, box)
        else:
            self.z, self.pz = np.zeros(1), np.zeros(1)
        self.dx = box / (n >> 1)
        self.dy = box / (n >> 1) if dim > 1 else 1.0
        self.dz = box / (n >> 1) if dim > 2 else 1.0
        N = self.nx * self.ny * self.nz
        self.V, self.K = np.zeros(N), np.zeros(N)
        self.Ax, self.Ay, self.Az = np.zeros(N), np.zeros(N), np.zeros(N)
        lib().orc_fields(dim, self.nx, self.ny, self.nz, _p(self.x), _p(self.y), _p(self.z),
                         _p(self.px), _p(self.py), _p(self.pz), hbar, mass, wx, wy, wz, gamma,
                         shifts[0], shifts[1], shifts[2], omega, 1 if gauge else 0,
                         _p(self.V), _p(self.K), _p(self.Ax), _p(self.Ay), _p(self.Az))
        self.cfg = Cfg(dim, self.nx, self.ny, self.nz, self.dx, self.dy, self.dz, hbar, g, gdt,
                       dt, 1 if gpe else 0, 1 if gauge else 0, 1 if ramp else 0, ramp_type,
                       omega, threads, energy_every, threshold, 1 if threshold_abs else 0,
                       None, None, None, None, None)
        self._ast_keep = []

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx) if self.dim == 3 else (self.ny, self.nx)

    def set_ast(self, name, rows):
        arr = nodes_array(rows)
        self._ast_keep.append(arr)
        setattr(self.cfg, "ast_" + name, C.cast(arr, C.POINTER(Node)))

    def evolve(self, psi, nsteps, gstate):
        """Returns (psi_out, result dict, energies)."""
        a = np.ascontiguousarray(psi, dtype=np.complex128).copy()
        cap = nsteps // max(self.cfg.energy_every, 1) + 2 if self.cfg.energy_every > 0 else 1
        en = np.zeros(cap)
        res = Result()
        lib().orc_evolve(C.byref(self.cfg), _p(self.V), _p(self.K), _p(self.Ax), _p(self.Ay),
                         _p(self.Az), _p(self.px), _p(self.py), _p(self.pz),
                         _p(a.view(np.float64)), nsteps, gstate, _p(en), C.byref(res))
        r = dict(steps_done=res.steps_done, early_stop=res.early_stop,
                 n_energies=res.n_energies, energy=res.energy)
        return a, r, en[:res.n_energies]

    def energy(self, psi):
        a = np.ascontiguousarray(psi, dtype=np.complex128)
        return lib().orc_energy(C.byref(self.cfg), _p(self.V), _p(self.K), _p(self.Ax),
                                _p(self.Ay), _p(self.Az), _p(a.view(np.float64)))


def find_vortex(psi, x, radius):
    """Tracker::findVortex (src/tracker.cu:102-166) on a complex128 (n, n)
    state [y, x] with grid x: (marker, winding, found), marker and winding
    int32 (n, n) arrays (winding: signed lround at the marks)."""
    a = np.ascontiguousarray(psi, dtype=np.complex128)
    n = a.shape[0]
    assert a.shape == (n, n)
    xs = np.ascontiguousarray(x, dtype=np.float64)
    marker = np.zeros((n, n), np.int32)
    winding = np.zeros((n, n), np.int32)
    ip = C.POINTER(C.c_int)
    found = lib().orc_find_vortex(_p(a.view(np.float64)), n, _p(xs), radius,
                                  marker.ctypes.data_as(ip), winding.ctypes.data_as(ip))
    return marker, winding, found

