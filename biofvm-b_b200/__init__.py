"""Python binding of the B200 BioFVM-B diffusion-decay library (C ABI over ctypes).

The product is the C ABI in include/biofvm_b200.h, implemented by
lib/libbiofvm_b200.so (CUDA, sm_100a). This module only loads that library
and wraps its calls; there is no CPU fallback: if the library is missing or
no CUDA device is present, every call raises.

The package directory is named ``biofvm-b_b200`` and is imported by path:

    import importlib.util, sys
    spec = importlib.util.spec_from_file_location(
        "biofvm_b_b200", "biofvm-b_b200/__init__.py",
        submodule_search_locations=["biofvm-b_b200"])
    bfb = importlib.util.module_from_spec(spec); sys.modules["biofvm_b_b200"] = bfb
    spec.loader.exec_module(bfb)
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libbiofvm_b200.so"

FP64 = 0
FP32 = 1
STEP_BULK = 1
STEP_DIFFUSION = 2
STEP_CELLS = 4
OPT_FREEZE_FACTORS = 1
OPT_USE_GRAPHS = 2
OPT_USE_TMA = 3
BATCH_OPT_WARPS_PER_CTA = 1
BATCH_OPT_TILES_PER_ITEM = 2
BATCH_OPT_MODE = 3
BATCH_MODE_PERSISTENT = 0
BATCH_MODE_STAGED = 1
BATCH_MODE_GRAPH = 2

ERRORS = {
    -1: "BFB_ERR_INVALID_ARG",
    -2: "BFB_ERR_SIZE",
    -3: "BFB_ERR_OOM",
    -4: "BFB_ERR_CUDA",
    -5: "BFB_ERR_STATE",
    -6: "BFB_ERR_WATCHDOG",
    -7: "BFB_ERR_UNSUPPORTED",
}

# Every symbol declared in include/biofvm_b200.h (checked by the CPU tests).
EXPORTS = [
    "bfb_last_error", "bfb_version", "bfb_create", "bfb_create_domain", "bfb_destroy", "bfb_get_shape",
    "bfb_set_stream", "bfb_set_option", "bfb_synchronize", "bfb_set_coefficients", "bfb_set_field",
    "bfb_get_field", "bfb_set_field_raw", "bfb_get_field_raw", "bfb_set_field_device", "bfb_get_field_device",
    "bfb_compare_fields", "bfb_field_device_ptr", "bfb_field_pitch", "bfb_set_dirichlet",
    "bfb_set_dirichlet_uniform", "bfb_apply_dirichlet", "bfb_diffusion_step", "bfb_set_bulk", "bfb_bulk_step",
    "bfb_set_agents", "bfb_set_agent_constants", "bfb_agent_voxels", "bfb_cells_step", "bfb_simulate", "bfb_step_host", "bfb_profile_steps",
    "bfb_checksum", "bfb_compute_gradients", "bfb_get_gradients", "bfb_write_matlab", "bfb_set_tuning", "bfb_get_tuning", "bfb_autotune", "bfb_batch_create", "bfb_batch_destroy", "bfb_batch_set_option", "bfb_batch_get_option", "bfb_batch_simulate",
    "bfb_batch_simulate_loop", "bfb_batch_synchronize", "bfb_batch_autotune", "bfb_adjoint_run",
    "bfb_checksum_noalloc", "bfb_watchdog_selftest", "bfb_host_register", "bfb_host_unregister",
    "bfb_batch_set_stream", "bfb_create_slab", "bfb_slab_info", "bfb_slab_x_forward", "bfb_slab_x_backward",
    "bfb_slab_yz",
]


class BFBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_up = ctypes.POINTER(ctypes.c_uint8)


def load_library(path: Path = LIB_PATH) -> ctypes.CDLL:
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not path.exists():
        raise FileNotFoundError(f"{path} is missing: build it with `python biofvm-b_b200/build.py`")
    L = ctypes.CDLL(str(path))
    L.bfb_last_error.restype = ctypes.c_char_p
    sig = {
        "bfb_create": [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                       ctypes.c_int, ctypes.c_int],
        "bfb_create_domain": [ctypes.POINTER(_vp)] + [ctypes.c_double] * 7 + [ctypes.c_int] * 3,
        "bfb_destroy": [_vp],
        "bfb_get_shape": [_vp, _ip, _ip, _ip, _ip],
        "bfb_set_stream": [_vp, _vp],
        "bfb_set_option": [_vp, ctypes.c_int, ctypes.c_int],
        "bfb_synchronize": [_vp],
        "bfb_watchdog_selftest": [_vp, ctypes.c_int],
        "bfb_host_register": [_vp, ctypes.c_size_t],
        "bfb_host_unregister": [_vp],
        "bfb_set_coefficients": [_vp, _dp, _dp],
        "bfb_set_field": [_vp, _vp],
        "bfb_get_field": [_vp, _vp],
        "bfb_set_field_raw": [_vp, _vp],
        "bfb_get_field_raw": [_vp, _vp],
        "bfb_set_field_device": [_vp, _vp, ctypes.c_int],
        "bfb_get_field_device": [_vp, _vp, ctypes.c_int],
        "bfb_compare_fields": [_vp, _vp, _dp],
        "bfb_field_device_ptr": [_vp, ctypes.POINTER(_vp)],
        "bfb_field_pitch": [_vp, ctypes.POINTER(ctypes.c_int)],
        "bfb_set_dirichlet": [_vp, _vp, _vp, _vp],
        "bfb_set_dirichlet_uniform": [_vp, _vp, _vp, _vp],
        "bfb_apply_dirichlet": [_vp],
        "bfb_diffusion_step": [_vp, ctypes.c_double, ctypes.c_int],
        "bfb_set_bulk": [_vp, _vp, _vp, _vp],
        "bfb_bulk_step": [_vp, ctypes.c_double],
        "bfb_set_agents": [_vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_double],
        "bfb_set_agent_constants": [_vp, ctypes.c_int, _vp, _vp, _vp, _vp],
        "bfb_agent_voxels": [_vp, _vp],
        "bfb_cells_step": [_vp, ctypes.c_double],
        "bfb_simulate": [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_int],
        "bfb_step_host": [_vp, _vp, ctypes.c_double, ctypes.c_int],
        "bfb_profile_steps": [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp],
        "bfb_checksum": [_vp, _dp],
        "bfb_compute_gradients": [_vp, _vp],
        "bfb_get_gradients": [_vp, _dp],
        "bfb_write_matlab": [_vp, ctypes.c_char_p],
        "bfb_set_tuning": [_vp, _ip],
        "bfb_get_tuning": [_vp, _ip],
        "bfb_autotune": [_vp, ctypes.c_double, ctypes.c_int, _ip, _dp],
        "bfb_checksum_noalloc": [_vp, ctypes.c_int, ctypes.c_longlong, ctypes.c_int, _vp, _vp],
        "bfb_batch_create": [ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(_vp)],
        "bfb_batch_destroy": [_vp],
        "bfb_batch_set_option": [_vp, ctypes.c_int, ctypes.c_int],
        "bfb_batch_get_option": [_vp, ctypes.c_int, _ip],
        "bfb_batch_simulate": [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_int],
        "bfb_batch_simulate_loop": [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_int],
        "bfb_batch_synchronize": [_vp],
        "bfb_batch_set_stream": [_vp, _vp],
        "bfb_batch_autotune": [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, _ip, _dp],
        "bfb_adjoint_run": [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _dp, _dp,
                            _dp, _dp, _dp],
        "bfb_create_slab": [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                            ctypes.c_int, ctypes.c_double, ctypes.c_int],
        "bfb_slab_info": [_vp, _ip, _ip, ctypes.POINTER(ctypes.c_longlong)],
        "bfb_slab_x_forward": [_vp, ctypes.c_double, _vp, _vp, ctypes.c_longlong, ctypes.c_longlong],
        "bfb_slab_x_backward": [_vp, ctypes.c_double, _vp, _vp, ctypes.c_longlong, ctypes.c_longlong],
        "bfb_slab_yz": [_vp, ctypes.c_double],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    _lib = L
    return L


def _check(code: int):
    if code != 0:
        raise BFBError(code, _lib.bfb_last_error().decode())


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _u8(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint8)


def host_register(a: np.ndarray):
    """Page-lock a host array (bfb_host_register) so that field copies from and
    to it run at pinned-memory speed; undo with host_unregister before the
    array is freed."""
    L = load_library()
    _check(L.bfb_host_register(ctypes.c_void_p(a.ctypes.data), a.nbytes))


def host_unregister(a: np.ndarray):
    L = load_library()
    _check(L.bfb_host_unregister(ctypes.c_void_p(a.ctypes.data)))


class Env:
    """One device-resident microenvironment (a ``bfb_env``)."""

    def __init__(self, shape, n_substrates, dx=20.0, precision=FP64, device=0, domain=None):
        L = load_library()
        h = _vp()
        if domain is not None:
            x0, x1, y0, y1, z0, z1 = domain
            _check(L.bfb_create_domain(ctypes.byref(h), x0, x1, y0, y1, z0, z1, dx, n_substrates, precision, device))
        else:
            nx, ny, nz = shape
            _check(L.bfb_create(ctypes.byref(h), nx, ny, nz, n_substrates, dx, precision, device))
        self.h = h
        self.L = L
        a = [ctypes.c_int() for _ in range(4)]
        _check(L.bfb_get_shape(h, *[ctypes.byref(x) for x in a]))
        self.nx, self.ny, self.nz, self.S = (x.value for x in a)
        self.precision = precision
        self.dx = dx

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz, self.S)

    def close(self):
        if getattr(self, "h", None):
            self.L.bfb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- configuration --------------------------------------------------
    def set_stream(self, stream_handle: int):
        _check(self.L.bfb_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def set_option(self, opt, value):
        _check(self.L.bfb_set_option(self.h, opt, int(value)))

    def set_coefficients(self, D, lam):
        D, lam = _f64(D), _f64(lam)
        assert D.size == self.S and lam.size == self.S
        _check(self.L.bfb_set_coefficients(self.h, D.ctypes.data_as(_dp), lam.ctypes.data_as(_dp)))

    def set_dirichlet(self, activation, values=None, face_mask=None):
        act = _u8(activation)
        v = None if values is None else _f64(values)
        if v is not None:
            assert v.size == self.nx * self.ny * self.nz * self.S
        fm = _u8(face_mask)
        _check(self.L.bfb_set_dirichlet(self.h, _ptr(v), _ptr(act), _ptr(fm)))

    def set_dirichlet_uniform(self, activation, value_per_substrate, face_mask=None):
        _check(self.L.bfb_set_dirichlet_uniform(self.h, _ptr(_f64(value_per_substrate)), _ptr(_u8(activation)),
                                                _ptr(_u8(face_mask))))

    def apply_dirichlet(self):
        _check(self.L.bfb_apply_dirichlet(self.h))

    def set_bulk(self, S_rate=None, T_target=None, U_rate=None):
        if S_rate is None:
            _check(self.L.bfb_set_bulk(self.h, None, None, None))
            return
        a, b, c = _f64(S_rate), _f64(T_target), _f64(U_rate)
        _check(self.L.bfb_set_bulk(self.h, _ptr(a), _ptr(b), _ptr(c)))

    def set_agents(self, pos, volume, secretion, uptake, saturation, dt, active=None):
        pos, volume = _f64(pos), _f64(volume)
        sec, upt, sat = _f64(secretion), _f64(uptake), _f64(saturation)
        n = pos.shape[0]
        _check(self.L.bfb_set_agents(self.h, n, _ptr(pos), _ptr(volume), _ptr(sec), _ptr(upt), _ptr(sat),
                                     _ptr(_u8(active)), dt))
        self.n_agents = n

    def set_agent_constants(self, voxel, temp1, temp2, active=None):
        vox = np.ascontiguousarray(voxel, dtype=np.int32)
        t1, t2 = _f64(temp1), _f64(temp2)
        _check(self.L.bfb_set_agent_constants(self.h, vox.size, _ptr(vox), _ptr(t1), _ptr(t2), _ptr(_u8(active))))
        self.n_agents = vox.size

    def agent_voxels(self):
        out = np.zeros(getattr(self, "n_agents", 0), dtype=np.int32)
        _check(self.L.bfb_agent_voxels(self.h, _ptr(out)))
        return out

    # -- data -----------------------------------------------------------
    def set_field(self, rho):
        rho = _f64(rho)
        assert rho.size == self.nx * self.ny * self.nz * self.S
        _check(self.L.bfb_set_field(self.h, _ptr(rho)))

    def get_field(self):
        out = np.empty(self.shape, dtype=np.float64)
        _check(self.L.bfb_get_field(self.h, _ptr(out)))
        return out

    def set_field_raw(self, rho):
        dt = np.float64 if self.precision == FP64 else np.float32
        rho = np.ascontiguousarray(rho, dtype=dt)
        _check(self.L.bfb_set_field_raw(self.h, _ptr(rho)))

    def get_field_raw(self):
        dt = np.float64 if self.precision == FP64 else np.float32
        out = np.empty(self.shape, dtype=dt)
        _check(self.L.bfb_get_field_raw(self.h, _ptr(out)))
        return out

    def set_field_device(self, ptr: int, precision: int):
        _check(self.L.bfb_set_field_device(self.h, ctypes.c_void_p(ptr), precision))

    def get_field_device(self, ptr: int, precision: int):
        _check(self.L.bfb_get_field_device(self.h, ctypes.c_void_p(ptr), precision))

    def compare(self, ref: "Env"):
        """Relative L-inf and L2 of this field against ref's, computed on the device."""
        out = np.zeros(4)
        _check(self.L.bfb_compare_fields(self.h, ref.h, out.ctypes.data_as(_dp)))
        return out[0] / max(out[1], 1e-300), float(np.sqrt(out[2] / max(out[3], 1e-300)))

    def field_device_ptr(self) -> int:
        """The device field: rows (i, j) of nz*S values, field_pitch() elements apart."""
        p = _vp()
        _check(self.L.bfb_field_device_ptr(self.h, ctypes.byref(p)))
        return p.value

    def field_pitch(self) -> int:
        """Elements between the device field's (i, j) rows: nz*S, or that padded to 16 bytes."""
        n = ctypes.c_int()
        _check(self.L.bfb_field_pitch(self.h, ctypes.byref(n)))
        return n.value

    # -- stepping -------------------------------------------------------
    def diffusion_step(self, dt, n=1):
        _check(self.L.bfb_diffusion_step(self.h, dt, n))

    def bulk_step(self, dt):
        _check(self.L.bfb_bulk_step(self.h, dt))

    def cells_step(self, dt):
        _check(self.L.bfb_cells_step(self.h, dt))

    def simulate(self, dt, n, flags=STEP_DIFFUSION):
        _check(self.L.bfb_simulate(self.h, dt, n, flags))

    def step_host_ptr(self, host_ptr: int, dt, n=1):
        _check(self.L.bfb_step_host(self.h, ctypes.c_void_p(host_ptr), dt, n))

    def synchronize(self):
        _check(self.L.bfb_synchronize(self.h))

    def watchdog_selftest(self, polls=64):
        """Queue one bounded wait that runs out (bfb_watchdog_selftest): the
        env's error flag is set as a stalled copy would set it."""
        _check(self.L.bfb_watchdog_selftest(self.h, polls))

    def profile_steps(self, dt, n, flags=STEP_DIFFUSION):
        """Milliseconds per phase over n steps: x, y, z, bulk, cells."""
        out = np.zeros(5)
        _check(self.L.bfb_profile_steps(self.h, dt, n, flags, out.ctypes.data_as(_dp)))
        return out

    def checksum(self):
        out = np.zeros(self.S)
        _check(self.L.bfb_checksum(self.h, out.ctypes.data_as(_dp)))
        return out

    def gradients(self):
        """(nx, ny, nz, S, 3) gradient vectors as host doubles (bfb_get_gradients)."""
        out = np.empty((*self.shape, 3), dtype=np.float64)
        _check(self.L.bfb_get_gradients(self.h, out.ctypes.data_as(_dp)))
        return out

    def write_matlab(self, filename):
        """The reference's MATLAB v4 snapshot of the field (bfb_write_matlab)."""
        _check(self.L.bfb_write_matlab(self.h, str(filename).encode()))

    def compute_gradients_device(self, ptr: int):
        """Gradient vectors into a device array of 3*V*S env-precision elements."""
        _check(self.L.bfb_compute_gradients(self.h, ctypes.c_void_p(ptr)))

    # -- launch shape ---------------------------------------------------
    def get_tuning(self):
        """[(tma, warps, chunks) for x, y, z]"""
        v = (ctypes.c_int * 9)()
        _check(self.L.bfb_get_tuning(self.h, v))
        return [tuple(v[3 * a:3 * a + 3]) for a in range(3)]

    def set_tuning(self, shape):
        flat = [int(x) for axis in shape for x in axis]
        v = (ctypes.c_int * 9)(*flat)
        _check(self.L.bfb_set_tuning(self.h, v))

    def autotune(self, dt, trials=5):
        """Times every launch shape of each sweep; keeps and returns the fastest
        as ([(tma, warps, chunks)] * 3, [ms per launch] * 3)."""
        v = (ctypes.c_int * 9)()
        ms = np.zeros(3)
        _check(self.L.bfb_autotune(self.h, dt, trials, v, ms.ctypes.data_as(_dp)))
        return [tuple(v[3 * a:3 * a + 3]) for a in range(3)], ms

    def adjoint_run(self, dt, n_steps, dL_dfinal_ptr: int, flags=STEP_DIFFUSION, checkpoint_every=None,
                    dL_dinitial_ptr: int = None, final_ptr: int = None, agent_grads=False, coef_grads=True):
        """Reverse mode of n_steps steps from the current field (bfb_adjoint_run).

        The pointers are device arrays of the env precision in the field layout.
        Returns a dict of host gradients: D and lambda (unless coef_grads is
        False, which skips the sums they need) and, with agent_grads,
        secretion / uptake / saturation as [n_agents, S] arrays."""
        K = checkpoint_every or max(1, int(round(n_steps ** 0.5)))
        gD, gL = (np.zeros(self.S), np.zeros(self.S)) if coef_grads else (None, None)
        na = getattr(self, "n_agents", 0)
        ga = [np.zeros((na, self.S)) for _ in range(3)] if agent_grads else [None] * 3
        ap = [None if g is None else g.ctypes.data_as(_dp) for g in ga]
        _check(self.L.bfb_adjoint_run(self.h, dt, n_steps, flags, K, ctypes.c_void_p(dL_dfinal_ptr),
                                      None if dL_dinitial_ptr is None else ctypes.c_void_p(dL_dinitial_ptr),
                                      None if final_ptr is None else ctypes.c_void_p(final_ptr),
                                      None if gD is None else gD.ctypes.data_as(_dp),
                                      None if gL is None else gL.ctypes.data_as(_dp), *ap))
        out = {"D": gD, "lambda": gL} if coef_grads else {}
        if agent_grads:
            out.update(secretion=ga[0], uptake=ga[1], saturation=ga[2])
        return out


class SlabEnv(Env):
    """Planes [x0, x0 + nx_local) of a grid of nx_global x planes, FP64: one
    rank's share of an x-slab decomposition (``bfb_create_slab``; the reference
    splits x over MPI ranks, BioFVM_parallel.cpp:108-144). Its x lines continue
    in the neighbouring slabs; ``slabs.step`` runs the pipelined exchange."""

    def __init__(self, nx_global, x0, nx_local, ny, nz, n_substrates, dx=20.0, device=0):
        L = load_library()
        h = _vp()
        _check(L.bfb_create_slab(ctypes.byref(h), nx_global, x0, nx_local, ny, nz, n_substrates, dx, device))
        self.h = h
        self.L = L
        self.nx, self.ny, self.nz, self.S = nx_local, ny, nz, n_substrates
        self.precision = FP64
        self.dx = dx
        g, x, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        _check(L.bfb_slab_info(h, ctypes.byref(g), ctypes.byref(x), ctypes.byref(n)))
        self.nx_global, self.x0, self.lines = g.value, x.value, n.value

    @property
    def first(self):
        return self.x0 == 0

    @property
    def last(self):
        return self.x0 + self.nx == self.nx_global

    def x_forward(self, dt, prev_in_ptr: int, prev_out_ptr: int, line0=0, line1=None):
        """Forward half of the x sweep over lines [line0, line1): device arrays of
        ``lines`` doubles (0 for none)."""
        line1 = self.lines if line1 is None else line1
        _check(self.L.bfb_slab_x_forward(self.h, dt, ctypes.c_void_p(prev_in_ptr or None),
                                         ctypes.c_void_p(prev_out_ptr or None), line0, line1))

    def x_backward(self, dt, next_in_ptr: int, next_out_ptr: int, line0=0, line1=None):
        line1 = self.lines if line1 is None else line1
        _check(self.L.bfb_slab_x_backward(self.h, dt, ctypes.c_void_p(next_in_ptr or None),
                                          ctypes.c_void_p(next_out_ptr or None), line0, line1))

    def yz(self, dt):
        _check(self.L.bfb_slab_yz(self.h, dt))


class Batch:
    """Many envs stepped together (a ``bfb_batch``): one launch per stage over
    every env's tiles (``BATCH_MODE_STAGED``, the default), one persistent
    launch per step (``BATCH_MODE_PERSISTENT``), or every env's own kernels as
    independent branches of one graph (``BATCH_MODE_GRAPH``)."""

    def __init__(self, envs):
        self.L = load_library()
        self.envs = list(envs)  # kept alive: the batch references them
        arr = (_vp * len(self.envs))(*[e.h for e in self.envs])
        h = _vp()
        _check(self.L.bfb_batch_create(ctypes.byref(h), len(self.envs), arr))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.bfb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_warps(self, w):
        _check(self.L.bfb_batch_set_option(self.h, BATCH_OPT_WARPS_PER_CTA, w))

    def set_tiles_per_item(self, t):
        _check(self.L.bfb_batch_set_option(self.h, BATCH_OPT_TILES_PER_ITEM, t))

    def set_mode(self, m):
        _check(self.L.bfb_batch_set_option(self.h, BATCH_OPT_MODE, m))

    def get_option(self, option):
        v = ctypes.c_int()
        _check(self.L.bfb_batch_get_option(self.h, option, ctypes.byref(v)))
        return v.value

    @property
    def mode(self):
        return self.get_option(BATCH_OPT_MODE)

    def autotune(self, dt, flags=STEP_DIFFUSION, trials=3):
        """Picks the mode, warps per CTA and tiles per item; returns ((warps, tiles), ms per step).
        The chosen mode is ``self.mode`` afterwards."""
        v = (ctypes.c_int * 2)()
        ms = ctypes.c_double()
        _check(self.L.bfb_batch_autotune(self.h, dt, flags, trials, v, ctypes.byref(ms)))
        return (v[0], v[1]), ms.value

    def simulate(self, dt, n, flags=STEP_DIFFUSION):
        _check(self.L.bfb_batch_simulate(self.h, dt, n, flags))

    def simulate_loop(self, dt, n, flags=STEP_DIFFUSION):
        _check(self.L.bfb_batch_simulate_loop(self.h, dt, n, flags))

    def synchronize(self):
        _check(self.L.bfb_batch_synchronize(self.h))

    def set_stream(self, stream_handle: int):
        """Issue the batch's steps on a caller's CUDA stream (0: its own)."""
        _check(self.L.bfb_batch_set_stream(self.h, ctypes.c_void_p(stream_handle or None)))
