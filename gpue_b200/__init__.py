"""gpue_b200: B200-native split-operator Gross-Pitaevskii step (GPUE's evolve()).

The product is the C-ABI shared library ``libgpue_b200.so`` built from
``gpue_b200/csrc`` (declared in ``include/gpue_b200.h``).  This module is a thin
ctypes mirror of that ABI for Python callers (tests, benchmarks).  Importing
it loads the library and raises if it has not been built: there is no
fallback implementation.
"""

import ctypes as C
import os

import numpy as np

__all__ = ["lib", "Params", "EvolveOpts", "EvolveResult", "Solver", "GpueError", "Batch",
           "BatchOpts", "BatchResult", "BatchStats", "Server", "ServerOpts", "Request",
           "ServerResult", "ServerStats", "PlanInfo",
           "PREC_FP64", "PREC_FP32", "C128", "C64", "MEM_HOST", "MEM_DEVICE",
           "GAUGE_ROTATION", "GAUGE_CONSTANT", "supported_length", "default_params"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgpue_b200.so")

PREC_FP64, PREC_FP32 = 0, 1
MEM_HOST, MEM_DEVICE = 0, 1
C128, C64 = 0, 1
GAUGE_ROTATION, GAUGE_CONSTANT = 0, 1

STATUS = {0: "GPUE_OK", 1: "GPUE_ERR_INVALID_ARG", 2: "GPUE_ERR_UNSUPPORTED",
          3: "GPUE_ERR_CUDA", 4: "GPUE_ERR_OUT_OF_MEMORY", 5: "GPUE_ERR_AST",
          6: "GPUE_ERR_STATE", 7: "GPUE_ERR_TIMEOUT", 8: "GPUE_ERR_CANCELLED"}


class GpueError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__("%s%s" % (STATUS.get(status, str(status)), (": " + msg) if msg else ""))


class Params(C.Structure):
    _fields_ = [("dimnum", C.c_int32), ("xDim", C.c_int32), ("yDim", C.c_int32),
                ("zDim", C.c_int32), ("xMax", C.c_double), ("yMax", C.c_double),
                ("zMax", C.c_double), ("hbar", C.c_double), ("mass", C.c_double),
                ("omegaX", C.c_double), ("omegaY", C.c_double), ("omegaZ", C.c_double),
                ("gammaY", C.c_double), ("x0_shift", C.c_double), ("y0_shift", C.c_double),
                ("z0_shift", C.c_double), ("omega", C.c_double), ("interaction", C.c_double),
                ("gDenConst", C.c_double), ("gdt", C.c_double), ("dt", C.c_double),
                ("gpe", C.c_int32), ("corotating", C.c_int32), ("gauge", C.c_int32),
                ("ramp", C.c_int32), ("ramp_type", C.c_int32), ("precision", C.c_int32),
                ("device", C.c_int32), ("reserved", C.c_int32 * 8)]


class EvolveOpts(C.Structure):
    _fields_ = [("energy_calc_steps", C.c_int32), ("energy_calc_threshold", C.c_double),
                ("threshold_abs", C.c_int32), ("polish_steps", C.c_int32),
                ("graph_chunk", C.c_int32), ("no_sync", C.c_int32),
                ("step_offset", C.c_int32), ("norm_guard", C.c_int32),
                ("norm_guard_period", C.c_int32), ("reserved", C.c_int32 * 3)]


class EvolveResult(C.Structure):
    _fields_ = [("steps_done", C.c_int32), ("early_stop", C.c_int32),
                ("n_energies", C.c_int32), ("reserved0", C.c_int32), ("energy", C.c_double),
                ("norm", C.c_double), ("device_ms", C.c_double),
                ("kernel_launches", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


class BatchOpts(C.Structure):
    _fields_ = [("energy_calc_steps", C.c_int32), ("energy_calc_threshold", C.c_double),
                ("threshold_abs", C.c_int32), ("max_steps", C.c_int32),
                ("norm_guard", C.c_int32), ("segments_per_launch", C.c_int32),
                ("autotune", C.c_int32), ("reserved", C.c_int32 * 5)]


class BatchResult(C.Structure):
    _fields_ = [("steps_done", C.c_int32), ("early_stop", C.c_int32), ("energy", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchStats(C.Structure):
    _fields_ = [("device_ms", C.c_double), ("kernel_launches", C.c_int64),
                ("graph_launches", C.c_int64), ("point_steps", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PlanInfo(C.Structure):
    _fields_ = [("n", C.c_int32), ("ra", C.c_int32), ("rb", C.c_int32), ("rc", C.c_int32),
                ("threads_per_line", C.c_int32), ("lines_per_cta", C.c_int32),
                ("threads", C.c_int32), ("blocks", C.c_int32), ("tuned", C.c_int32),
                ("us", C.c_float), ("default_us", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Observables(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("norm", "energy", "e_kinetic", "e_potential",
                                          "e_interaction", "e_rotation", "x", "y", "z",
                                          "r2", "q", "lz")] + [("reserved", C.c_double * 4)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class Vortex(C.Structure):
    _fields_ = [("i", C.c_int32), ("j", C.c_int32), ("marker", C.c_int32),
                ("winding", C.c_int32)]


VORTEX_DTYPE = np.dtype([("i", np.int32), ("j", np.int32), ("marker", np.int32),
                         ("winding", np.int32)])


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("precision", C.c_int32),
                ("hbm_budget_bytes", C.c_int64), ("check_steps", C.c_int32),
                ("max_active", C.c_int32), ("threshold", C.c_double),
                ("threshold_abs", C.c_int32), ("autotune", C.c_int32),
                ("reserved", C.c_int32 * 6)]


class Request(C.Structure):
    _fields_ = [("params", Params), ("gstate", C.c_int32), ("max_steps", C.c_int32),
                ("psi0", C.c_void_p), ("psi_out", C.c_void_p), ("tag", C.c_int64),
                ("deadline_s", C.c_double)]


class ServerResult(C.Structure):
    _fields_ = [("tag", C.c_int64), ("status", C.c_int32), ("steps_done", C.c_int32),
                ("early_stop", C.c_int32), ("reserved0", C.c_int32), ("energy", C.c_double),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64),
                ("failed", C.c_int64), ("active", C.c_int32), ("queued", C.c_int32),
                ("bytes_resident", C.c_int64), ("bytes_peak", C.c_int64),
                ("bytes_budget", C.c_int64), ("ticks", C.c_int64),
                ("kernel_launches", C.c_int64), ("point_steps", C.c_double),
                ("busy_s", C.c_double), ("admit_s", C.c_double), ("issue_s", C.c_double),
                ("finish_s", C.c_double), ("admitted_in_tick", C.c_int64),
                ("timed_out", C.c_int64), ("cancelled", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib():
    """The loaded libgpue_b200.so (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libgpue_b200.so is not built; run `make -C gpue_b200` "
                              "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        vp, i32 = C.c_void_p, C.c_int32
        L.gpue_abi_version.restype = C.c_int
        L.gpue_default_params.argtypes = [C.POINTER(Params)]
        L.gpue_ctx_create.argtypes = [C.POINTER(Params), C.POINTER(vp)]
        L.gpue_ctx_destroy.argtypes = [vp]
        L.gpue_last_error.argtypes = [vp]
        L.gpue_last_error.restype = C.c_char_p
        L.gpue_supported_length.argtypes = [i32, i32]
        L.gpue_set_operators.argtypes = [vp, i32]
        L.gpue_set_wfc.argtypes = [vp, vp, i32, i32]
        L.gpue_get_wfc.argtypes = [vp, vp, i32, i32]
        L.gpue_evolve.argtypes = [vp, i32, i32, C.POINTER(EvolveOpts), C.POINTER(EvolveResult)]
        L.gpue_energy.argtypes = [vp, C.POINTER(C.c_double)]
        L.gpue_norm.argtypes = [vp, C.POINTER(C.c_double)]
        L.gpue_observables_get.argtypes = [vp, C.POINTER(Observables)]
        L.gpue_set_check_observables.argtypes = [vp, C.POINTER(Observables), i32]
        L.gpue_find_vortices.argtypes = [vp, C.c_double, vp, i32, vp, i32, C.POINTER(i32)]
        L.gpue_ctx_stream.argtypes = [vp, C.POINTER(vp)]
        L.gpue_ctx_wfc_device.argtypes = [vp, C.POINTER(vp), C.POINTER(i32)]
        L.gpue_norm_noalloc.argtypes = [vp, i32, C.c_int64, C.c_double, vp, vp]
        L.gpue_norm_noalloc.restype = C.c_int
        L.gpue_load_param_text.argtypes = [vp, C.c_char_p, i32, C.POINTER(C.c_char_p),
                                           C.POINTER(C.c_double), i32]
        L.gpue_ast_parse.argtypes = [C.c_char_p, C.POINTER(C.c_char_p), C.POINTER(C.c_double),
                                     i32, vp, i32, C.POINTER(i32)]
        L.gpue_ast_parse_file.argtypes = [C.c_char_p, C.POINTER(C.c_char_p),
                                          C.POINTER(C.c_double), i32, i32, C.c_char_p, i32,
                                          C.POINTER(i32), vp, i32, C.POINTER(i32),
                                          C.POINTER(i32)]
        L.gpue_batch_create.argtypes = [C.POINTER(vp), i32, C.POINTER(vp)]
        L.gpue_batch_destroy.argtypes = [vp]
        L.gpue_batch_last_error.argtypes = [vp]
        L.gpue_batch_last_error.restype = C.c_char_p
        L.gpue_batch_evolve.argtypes = [vp, i32, C.POINTER(BatchOpts), C.POINTER(BatchResult),
                                        C.POINTER(BatchStats)]
        L.gpue_set_gauge_tables.argtypes = [vp, vp, vp, vp]
        L.gpue_set_potential_table.argtypes = [vp, vp]
        L.gpue_snapshot_save.argtypes = [vp, C.c_char_p, i32, C.c_int64]
        L.gpue_snapshot_load.argtypes = [vp, C.c_char_p, C.POINTER(i32), C.POINTER(C.c_int64)]
        L.gpue_autotune.argtypes = [vp, i32]
        L.gpue_get_plan.argtypes = [vp, i32, C.POINTER(PlanInfo)]
        L.gpue_list_plans.argtypes = [i32, i32, C.POINTER(PlanInfo), i32, C.POINTER(i32)]
        L.gpue_set_plan.argtypes = [vp, i32, i32, i32, i32, i32, i32]
        L.gpue_time_passes.argtypes = [vp, i32, i32, C.POINTER(C.c_float), C.POINTER(i32), i32,
                                       C.POINTER(i32)]
        L.gpue_server_create.argtypes = [C.POINTER(ServerOpts), C.POINTER(vp)]
        L.gpue_server_destroy.argtypes = [vp]
        L.gpue_server_last_error.argtypes = [vp]
        L.gpue_server_last_error.restype = C.c_char_p
        L.gpue_server_submit.argtypes = [vp, C.POINTER(Request)]
        L.gpue_server_poll.argtypes = [vp, C.POINTER(ServerResult), i32, C.POINTER(i32),
                                       C.c_double]
        L.gpue_server_get_stats.argtypes = [vp, C.POINTER(ServerStats)]
        L.gpue_server_cancel.argtypes = [vp, C.c_int64]
        L.gpue_server_clock.argtypes = [vp]
        L.gpue_server_clock.restype = C.c_double
        for name in ("gpue_server_create", "gpue_server_destroy", "gpue_server_submit",
                     "gpue_server_poll", "gpue_server_get_stats", "gpue_server_cancel"):
            getattr(L, name).restype = C.c_int
        for name in ("gpue_default_params", "gpue_ctx_create", "gpue_ctx_destroy",
                     "gpue_set_operators", "gpue_set_wfc", "gpue_get_wfc", "gpue_evolve",
                     "gpue_energy", "gpue_norm", "gpue_ctx_stream", "gpue_ctx_wfc_device",
                     "gpue_load_param_text", "gpue_ast_parse", "gpue_ast_parse_file",
                     "gpue_batch_create",
                     "gpue_batch_destroy", "gpue_batch_evolve", "gpue_autotune",
                     "gpue_get_plan", "gpue_set_gauge_tables", "gpue_observables_get",
                     "gpue_find_vortices", "gpue_set_potential_table", "gpue_snapshot_save",
                     "gpue_snapshot_load", "gpue_list_plans", "gpue_set_plan",
                     "gpue_set_check_observables", "gpue_time_passes"):
            getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def supported_length(n, precision=PREC_FP64):
    return bool(lib().gpue_supported_length(precision, n))


def list_plans(n, precision=PREC_FP64):
    """The compiled FFT plans of length n (gpue_list_plans), default first."""
    cnt = C.c_int32()
    _check(lib().gpue_list_plans(precision, n, None, 0, C.byref(cnt)))
    out = (PlanInfo * max(cnt.value, 1))()
    _check(lib().gpue_list_plans(precision, n, out, cnt.value, C.byref(cnt)))
    return [{k: out[i].as_dict()[k] for k in ("n", "ra", "rb", "rc", "threads_per_line")}
            for i in range(cnt.value)]


def default_params():
    p = Params()
    _check(lib().gpue_default_params(C.byref(p)))
    return p


def _check(st, ctx=None):
    if st != 0:
        msg = lib().gpue_last_error(ctx).decode() if ctx else ""
        raise GpueError(st, msg)


def make_params(dim, n, box, hbar=1.0, mass=1.0, wx=1.0, wy=1.0, wz=1.0, gamma=1.0, g=0.0,
                gpe=True, omega=0.0, gauge=False, gdt=1e-4, dt=1e-4, precision=PREC_FP64,
                ramp=False, ramp_type=1, device=0, shifts=(0.0, 0.0, 0.0)):
    """Params for a square/cubic run with gN = g (interaction = g, gDenConst = 1)."""
    p = Params()
    p.dimnum = dim
    p.xDim = p.yDim = n
    p.zDim = n if dim == 3 else 1
    p.xMax = p.yMax = p.zMax = box
    p.hbar, p.mass = hbar, mass
    p.omegaX, p.omegaY, p.omegaZ, p.gammaY = wx, wy, wz, gamma
    p.x0_shift, p.y0_shift, p.z0_shift = shifts
    p.omega = omega
    p.interaction, p.gDenConst = g, 1.0
    p.gdt, p.dt = gdt, dt
    p.gpe = 1 if gpe else 0
    p.corotating = 1 if gauge else 0
    p.gauge = GAUGE_ROTATION
    p.ramp, p.ramp_type = (1 if ramp else 0), ramp_type
    p.precision = precision
    p.device = device
    return p


class Solver:
    """One context of the C ABI: resident wavefunction plus operators."""

    def __init__(self, params):
        self.params = params
        h = C.c_void_p()
        _check(lib().gpue_ctx_create(C.byref(params), C.byref(h)))
        self._h = h
        d = params.dimnum
        # [z, y, x], x fastest
        self.shape = ((params.zDim, params.yDim, params.xDim) if d == 3
                      else (params.yDim, params.xDim))
        self.precision = params.precision

    def close(self):
        if self._h:
            lib().gpue_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, st):
        _check(st, self._h)

    def set_operators(self, ev_type):
        self._ck(lib().gpue_set_operators(self._h, ev_type))

    def set_wfc(self, psi):
        a = np.ascontiguousarray(psi)
        if a.dtype == np.complex128:
            dt = C128
        elif a.dtype == np.complex64:
            dt = C64
        else:
            raise TypeError("psi must be complex64 or complex128")
        if a.size != int(np.prod(self.shape)):
            raise ValueError("psi has %d points, grid has %d" % (a.size, np.prod(self.shape)))
        self._ck(lib().gpue_set_wfc(self._h, a.ctypes.data_as(C.c_void_p), MEM_HOST, dt))

    def get_wfc(self, dtype=np.complex128):
        out = np.empty(self.shape, dtype=dtype)
        dt = C128 if out.dtype == np.complex128 else C64
        self._ck(lib().gpue_get_wfc(self._h, out.ctypes.data_as(C.c_void_p), MEM_HOST, dt))
        return out

    def set_wfc_device(self, ptr, dtype):
        self._ck(lib().gpue_set_wfc(self._h, C.c_void_p(ptr), MEM_DEVICE, dtype))

    def get_wfc_device(self, ptr, dtype):
        self._ck(lib().gpue_get_wfc(self._h, C.c_void_p(ptr), MEM_DEVICE, dtype))

    def evolve(self, nsteps, gstate, energy_every=0, threshold=-1.0, threshold_abs=False,
               polish_steps=0, graph_chunk=0, no_sync=False, step_offset=0, norm_guard=-1,
               norm_guard_period=0):
        o = EvolveOpts()
        o.norm_guard = norm_guard
        o.norm_guard_period = norm_guard_period
        o.no_sync = 1 if no_sync else 0
        o.step_offset = step_offset
        o.energy_calc_steps = energy_every
        o.energy_calc_threshold = threshold
        o.threshold_abs = 1 if threshold_abs else 0
        o.polish_steps = polish_steps
        o.graph_chunk = graph_chunk
        r = EvolveResult()
        self._ck(lib().gpue_evolve(self._h, nsteps, gstate, C.byref(o), C.byref(r)))
        return r.as_dict()

    def energy(self):
        e = C.c_double()
        self._ck(lib().gpue_energy(self._h, C.byref(e)))
        return e.value

    def norm(self):
        e = C.c_double()
        self._ck(lib().gpue_norm(self._h, C.byref(e)))
        return e.value

    def find_vortices(self, radius, cap=None):
        """Tracker::findVortex on the resident 2D state (gpue_find_vortices):
        (marker int32 (n, n), list of marks as a VORTEX_DTYPE array, found)."""
        n = self.params.xDim
        marker = np.zeros((n, n), np.int32)
        cap = n * n // 2 + 1 if cap is None else int(cap)
        lst = np.zeros(max(cap, 1), VORTEX_DTYPE)
        found = C.c_int32()
        vp = C.c_void_p
        self._ck(lib().gpue_find_vortices(self._h, float(radius), marker.ctypes.data_as(vp),
                                          MEM_HOST, lst.ctypes.data_as(vp) if cap else None,
                                          cap, C.byref(found)))
        return marker, lst[:min(found.value, cap)], found.value

    def record_check_observables(self, cap):
        """Record observables at every energy check of later evolve calls
        (gpue_set_check_observables); cap = 0 turns it off."""
        self._obs_buf = (Observables * max(int(cap), 1))() if cap else None
        self._ck(lib().gpue_set_check_observables(self._h, self._obs_buf, int(cap)))

    def check_observables(self, n):
        """The observables of the first n checks of the latest evolve call."""
        return [self._obs_buf[k].as_dict() for k in range(n)]

    def observables(self):
        """Energy terms, trapezoid density moments and <L_z> of the current
        state (gpue_observables_get), as a dict."""
        o = Observables()
        self._ck(lib().gpue_observables_get(self._h, C.byref(o)))
        return o.as_dict()

    def stream(self):
        s = C.c_void_p()
        self._ck(lib().gpue_ctx_stream(self._h, C.byref(s)))
        return s.value or 0

    def wfc_device(self):
        p, d = C.c_void_p(), C.c_int32()
        self._ck(lib().gpue_ctx_wfc_device(self._h, C.byref(p), C.byref(d)))
        return p.value, d.value

    def autotune(self, force=False):
        """Time the compiled plans and lines-per-CTA choices; keep the fastest."""
        self._ck(lib().gpue_autotune(self._h, 1 if force else 0))
        return [self.plan(a) for a in range(len(self.shape))]

    def set_plan(self, axis, ra, rb, rc, threads_per_line, lines_per_cta=0):
        """Use one compiled plan on one axis (gpue_set_plan)."""
        self._ck(lib().gpue_set_plan(self._h, axis, ra, rb, rc, threads_per_line,
                                     lines_per_cta))

    def time_passes(self, gstate=0, nsteps=8):
        """Mean device time (us) of each pass of a time step (gpue_time_passes),
        as a list of (kind, us): kind 0/1/2 a line pass along x/y/z (2 also the
        3D complex64 z tile pass), 3/4 the forward/inverse XY pass."""
        cap = 16
        us = (C.c_float * cap)()
        kinds = (C.c_int32 * cap)()
        n = C.c_int32(0)
        self._ck(lib().gpue_time_passes(self._h, gstate, nsteps, us, kinds, cap, C.byref(n)))
        return [(int(kinds[i]), float(us[i])) for i in range(min(n.value, cap))]

    def plan(self, axis):
        out = PlanInfo()
        self._ck(lib().gpue_get_plan(self._h, axis, C.byref(out)))
        return out.as_dict()

    def set_gauge_tables(self, Ax=None, Ay=None, Az=None):
        """Full-field gauge components (GPUE's -A file), x fastest."""
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).ravel()
                for a in (Ax, Ay, Az)]
        for a in keep:
            if a is not None and a.size != int(np.prod(self.shape)):
                raise ValueError("gauge table has %d points, grid has %d"
                                 % (a.size, np.prod(self.shape)))
        ptr = [None if a is None else a.ctypes.data for a in keep]
        self._ck(lib().gpue_set_gauge_tables(self._h, *ptr))

    def save_snapshot(self, path, gstate=0, step=0):
        """Binary snapshot of the state for checkpoint/resume (gpue_snapshot_save)."""
        self._ck(lib().gpue_snapshot_save(self._h, os.fsencode(path), int(gstate), int(step)))

    def load_snapshot(self, path):
        """Load a snapshot (gpue_snapshot_load); returns (gstate, step)."""
        g, st = C.c_int32(), C.c_int64()
        self._ck(lib().gpue_snapshot_load(self._h, os.fsencode(path), C.byref(g), C.byref(st)))
        return g.value, st.value

    def set_potential_table(self, V):
        """Full-field potential V (GPUE's V_gpu, e.g. -v torus), x fastest."""
        v = np.ascontiguousarray(V, dtype=np.float64).ravel()
        if v.size != int(np.prod(self.shape)):
            raise ValueError("potential table has %d points, grid has %d"
                             % (v.size, np.prod(self.shape)))
        self._ck(lib().gpue_set_potential_table(self._h, v.ctypes.data))

    def load_param_text(self, text, time_mode=0, doubles=None):
        """Parameter-file fields (GPUE's -I file) from "name = expr" lines."""
        doubles = doubles or {}
        names = (C.c_char_p * max(1, len(doubles)))(*[k.encode() for k in doubles])
        vals = (C.c_double * max(1, len(doubles)))(*doubles.values())
        self._ck(lib().gpue_load_param_text(self._h, text.encode(), time_mode, names, vals,
                                            len(doubles)))


class Batch:
    """Independent solves stepped together (gpue_batch_*); holds the Solvers."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s._h.value for s in self.solvers])
        h = C.c_void_p()
        st = lib().gpue_batch_create(arr, len(self.solvers), C.byref(h))
        if st != 0:
            raise GpueError(st, "gpue_batch_create")
        self._h = h

    def close(self):
        if self._h:
            lib().gpue_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def evolve(self, gstate, max_steps, energy_every=0, threshold=-1.0, threshold_abs=False,
               norm_guard=-1, segments_per_launch=0, autotune=False):
        """Returns (per-solve result dicts, stats dict)."""
        o = BatchOpts()
        o.autotune = 1 if autotune else 0
        o.energy_calc_steps = energy_every
        o.energy_calc_threshold = threshold
        o.threshold_abs = 1 if threshold_abs else 0
        o.max_steps = max_steps
        o.norm_guard = norm_guard
        o.segments_per_launch = segments_per_launch
        res = (BatchResult * len(self.solvers))()
        stats = BatchStats()
        st = lib().gpue_batch_evolve(self._h, gstate, C.byref(o), res, C.byref(stats))
        if st != 0:
            raise GpueError(st, lib().gpue_batch_last_error(self._h).decode())
        return [r.as_dict() for r in res], stats.as_dict()


class Server:
    """The serving loop (gpue_server_*): submit solves, poll finished ones.

    Each request's initial state (complex128) and, when asked for, its output
    buffer are kept referenced here until its result has been polled."""

    def __init__(self, precision=PREC_FP32, check_steps=100, threshold=1e-10,
                 threshold_abs=True, hbm_budget=0, max_active=0, device=0, autotune=False):
        o = ServerOpts()
        o.autotune = 1 if autotune else 0
        o.device = device
        o.precision = precision
        o.hbm_budget_bytes = int(hbm_budget)
        o.check_steps = check_steps
        o.max_active = max_active
        o.threshold = threshold
        o.threshold_abs = 1 if threshold_abs else 0
        h = C.c_void_p()
        st = lib().gpue_server_create(C.byref(o), C.byref(h))
        if st != 0:
            raise GpueError(st, "gpue_server_create")
        self._h = h
        self._live = {}

    def close(self):
        if self._h:
            lib().gpue_server_destroy(self._h)
            self._h = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, params, gstate, max_steps, psi0, tag, want_psi=True, deadline=0.0):
        """Queues a solve; deadline (seconds after submission, 0 for none)
        makes it fail with GPUE_ERR_TIMEOUT when it has not finished by then."""
        a = np.ascontiguousarray(psi0, dtype=np.complex128)
        out = np.empty_like(a) if want_psi else None
        q = Request()
        q.params = params
        q.gstate = gstate
        q.max_steps = max_steps
        q.psi0 = a.ctypes.data
        q.psi_out = out.ctypes.data if out is not None else None
        q.tag = tag
        q.deadline_s = float(deadline)
        self._live[tag] = (a, out)
        st = lib().gpue_server_submit(self._h, C.byref(q))
        if st != 0:
            del self._live[tag]
            raise GpueError(st, lib().gpue_server_last_error(self._h).decode())

    def cancel(self, tag):
        """Cancels the queued or resident requests with this tag (their
        results come back with GPUE_ERR_CANCELLED)."""
        st = lib().gpue_server_cancel(self._h, C.c_int64(tag))
        if st != 0:
            raise GpueError(st, "no queued or resident request with tag %d" % tag)

    def poll(self, timeout=0.0, cap=256):
        """Finished results as dicts (with "psi" when the output was kept)."""
        buf = (ServerResult * cap)()
        n = C.c_int32()
        _check(lib().gpue_server_poll(self._h, buf, cap, C.byref(n), float(timeout)))
        out = []
        for i in range(n.value):
            d = buf[i].as_dict()
            a, psi = self._live.pop(d["tag"], (None, None))
            d["psi"] = psi
            out.append(d)
        return out

    def stats(self):
        s = ServerStats()
        lib().gpue_server_get_stats(self._h, C.byref(s))
        return s.as_dict()

    def clock(self):
        return lib().gpue_server_clock(self._h)

    def last_error(self):
        return lib().gpue_server_last_error(self._h).decode()
