"""ctypes front-end for the test oracle.

TEST INFRASTRUCTURE ONLY. Two CPU checkers live under oracle/:

* ``Oracle``  -- our C restatement (lod_oracle.c -> _build/liboracle.so), which
  travels with the repository and is what GPU tests compare against.
* ``RefLib``  -- the reference BioFVM-B library compiled from its own sources
  (oracle/Makefile ``ref`` target -> _ref/libbiofvm_ref.so), used to pin the
  restatement (bit-exact) and as the CPU baseline in bench.py.

Only tests/, __graft_entry__.smoke() and bench.py import this module.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libbiofvm_ref.so"

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_up = ctypes.POINTER(ctypes.c_uint8)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _u(a):
    return a.ctypes.data_as(_up)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def face_mask_all(activation):
    """The reference's Dirichlet mask: all six faces follow the per-substrate
    activation flag (BioFVM_microenvironment.cpp:381-484)."""
    act = np.asarray(activation, dtype=np.uint8)
    return np.ascontiguousarray(np.tile(act, (6, 1)), dtype=np.uint8)


class Oracle:
    """Our C restatement of the hot path (see lod_oracle.h)."""

    def __init__(self, path: Path = ORACLE_SO):
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run `make -C oracle liboracle`")
        self.lib = ctypes.CDLL(str(path))
        L = self.lib
        L.orc_factors.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp]
        L.orc_constant1.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp]
        L.orc_dirichlet.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _up]
        L.orc_lod_step.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _up]
        L.orc_bulk_step.argtypes = [_dp, ctypes.c_int64, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp]
        L.orc_bin_agents.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip]
        L.orc_agent_constants.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_cells_step.argtypes = [_dp, ctypes.c_int, ctypes.c_int, _ip, _dp, _dp, _up]
        L.orc_checksum.argtypes = [_dp, ctypes.c_int64, ctypes.c_int, _dp]
        L.orc_gradients.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp]
        L.orc_lod_step_adjoint.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _up, _dp, _dp]
        L.orc_lod_steps_f32.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp, ctypes.c_int,
                                        _dp, _up]
        _fp = ctypes.POINTER(ctypes.c_float)
        L.orc_bulk_step_f32.argtypes = [_fp, ctypes.c_int64, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp]
        L.orc_cells_step_f32.argtypes = [_fp, ctypes.c_int, ctypes.c_int, _ip, _dp, _dp, _up]

    def factors(self, n, dt, dx, D, lam):
        D, lam = f64(D), f64(lam)
        S = D.size
        den = np.zeros((n, S))
        c = np.zeros((n, S))
        self.lib.orc_factors(n, S, dt, dx, _d(D), _d(lam), _d(den), _d(c))
        return den, c

    def constant1(self, dt, dx, D):
        D = f64(D)
        out = np.zeros(D.size)
        self.lib.orc_constant1(D.size, dt, dx, _d(D), _d(out))
        return out

    def dirichlet(self, rho, values, face_mask):
        rho = f64(rho).copy()
        nx, ny, nz, S = rho.shape
        values = f64(values)
        fm = np.ascontiguousarray(face_mask, dtype=np.uint8)
        self.lib.orc_dirichlet(_d(rho), nx, ny, nz, S, _d(values), _u(fm))
        return rho

    def lod_steps(self, rho, dt, dx, D, lam, n_steps=1, dir_values=None, face_mask=None):
        """n LOD diffusion-decay steps; rho is (nx, ny, nz, S)."""
        rho = f64(rho).copy()
        nx, ny, nz, S = rho.shape
        if dir_values is None:
            dir_values = np.zeros_like(rho)
        if face_mask is None:
            face_mask = np.zeros((6, S), np.uint8)
        dv = f64(dir_values)
        fm = np.ascontiguousarray(face_mask, dtype=np.uint8)
        fx = self.factors(nx, dt, dx, D, lam)
        fy = self.factors(ny, dt, dx, D, lam)
        fz = self.factors(nz, dt, dx, D, lam)
        c1 = self.constant1(dt, dx, D)
        for _ in range(n_steps):
            self.lib.orc_lod_step(_d(rho), nx, ny, nz, S, _d(fx[0]), _d(fx[1]), _d(fy[0]), _d(fy[1]),
                                  _d(fz[0]), _d(fz[1]), _d(c1), _d(dv), _u(fm))
        return rho

    def lod_steps_f32(self, rho, dt, dx, D, lam, n_steps=1, dir_values=None, face_mask=None):
        """The product's FP32 path restated (orc_lod_steps_f32): n LOD steps on
        an FP32 field; rho (nx, ny, nz, S) is rounded to FP32 first, as the
        device upload does. Returns float32."""
        rho = np.ascontiguousarray(rho, dtype=np.float32).copy()
        nx, ny, nz, S = rho.shape
        D, lam = f64(D), f64(lam)
        dv = None if dir_values is None else f64(np.broadcast_to(dir_values, rho.shape))
        fm = None if face_mask is None else np.ascontiguousarray(face_mask, dtype=np.uint8)
        if (dv is None) != (fm is None):
            raise ValueError("dir_values and face_mask go together")
        self.lib.orc_lod_steps_f32(rho.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), nx, ny, nz, S, dt, dx,
                                   _d(D), _d(lam), n_steps, None if dv is None else _d(dv),
                                   None if fm is None else _u(fm))
        return rho

    def bulk_step_f32(self, rho, dt, S_rate, T_target, U_rate):
        """The FP32 path's bulk update (orc_bulk_step_f32) on a float32 field."""
        rho = np.ascontiguousarray(rho, dtype=np.float32).copy()
        S = rho.shape[-1]
        Sr, Tt, Ur = f64(S_rate), f64(T_target), f64(U_rate)
        self.lib.orc_bulk_step_f32(rho.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), rho.size // S, S, dt,
                                   _d(Sr), _d(Tt), _d(Ur))
        return rho

    def cells_step_f32(self, rho, voxel, t1, t2, active=None):
        """The FP32 path's agent update (orc_cells_step_f32) on a float32 field."""
        rho = np.ascontiguousarray(rho, dtype=np.float32).copy()
        S = rho.shape[-1]
        voxel = np.ascontiguousarray(voxel, dtype=np.int32)
        act = None if active is None else np.ascontiguousarray(active, dtype=np.uint8)
        self.lib.orc_cells_step_f32(rho.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), S, voxel.size, _i(voxel),
                                    _d(f64(t1)), _d(f64(t2)), _u(act) if act is not None else ctypes.cast(None, _up))
        return rho

    def bulk_step(self, rho, dt, S_rate, T_target, U_rate):
        rho = f64(rho).copy()
        S = rho.shape[-1]
        V = rho.size // S
        Sr, Tt, Ur = f64(S_rate), f64(T_target), f64(U_rate)
        self.lib.orc_bulk_step(_d(rho), V, S, dt, _d(Sr), _d(Tt), _d(Ur))
        return rho

    def bin_agents(self, pos, bbox, dx, shape):
        pos = f64(pos)
        n = pos.shape[0]
        out = np.zeros(n, dtype=np.int32)
        bb = f64(bbox)
        self.lib.orc_bin_agents(n, _d(pos), _d(bb), dx, dx, dx, shape[0], shape[1], shape[2], _i(out))
        return out

    def agent_constants(self, dt, dx, volume, sec, upt, sat):
        sec, upt, sat, volume = f64(sec), f64(upt), f64(sat), f64(volume)
        n, S = sec.shape
        t1 = np.zeros((n, S))
        t2 = np.zeros((n, S))
        self.lib.orc_agent_constants(n, S, dt, dx, dx, dx, _d(volume), _d(sec), _d(upt), _d(sat), _d(t1), _d(t2))
        return t1, t2

    def cells_step(self, rho, voxel, t1, t2, active=None):
        rho = f64(rho).copy()
        S = rho.shape[-1]
        voxel = np.ascontiguousarray(voxel, dtype=np.int32)
        n = voxel.size
        act = None if active is None else np.ascontiguousarray(active, dtype=np.uint8)
        self.lib.orc_cells_step(_d(rho), S, n, _i(voxel), _d(f64(t1)), _d(f64(t2)),
                                _u(act) if act is not None else ctypes.cast(None, _up))
        return rho

    def checksum(self, rho):
        rho = f64(rho)
        S = rho.shape[-1]
        out = np.zeros(S)
        self.lib.orc_checksum(_d(rho), rho.size // S, S, _d(out))
        return out

    def gradients(self, rho, dx):
        """(nx, ny, nz, S, 3) gradient vectors (orc_gradients)."""
        rho = f64(rho)
        nx, ny, nz, S = rho.shape
        out = np.zeros((nx, ny, nz, S, 3))
        self.lib.orc_gradients(_d(rho), nx, ny, nz, S, dx, _d(out))
        return out

    def lod_step_adjoint(self, rho_in, lam_out, dt, dx, D, lam_rates, dir_values=None, face_mask=None):
        rho_in = f64(rho_in)
        nx, ny, nz, S = rho_in.shape
        lam = f64(lam_out).copy()
        if dir_values is None:
            dir_values = np.zeros_like(rho_in)
        if face_mask is None:
            face_mask = np.zeros((6, S), np.uint8)
        gD = np.zeros(S)
        gL = np.zeros(S)
        self.lib.orc_lod_step_adjoint(_d(rho_in), _d(lam), nx, ny, nz, S, dt, dx, _d(f64(D)), _d(f64(lam_rates)),
                                      _d(f64(dir_values)), _u(np.ascontiguousarray(face_mask, np.uint8)),
                                      _d(gD), _d(gL))
        return lam, gD, gL


class RefLib:
    """The reference BioFVM-B library compiled from its own sources."""

    available = REF_SO.exists()

    def __init__(self, path: Path = REF_SO):
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference is mounted")
        self.lib = ctypes.CDLL(str(path))
        L = self.lib
        L.ref_create.restype = ctypes.c_void_p
        L.ref_create.argtypes = [ctypes.c_double] * 7 + [ctypes.c_int, _dp, _dp]
        L.ref_destroy.argtypes = [ctypes.c_void_p]
        L.ref_sizes.argtypes = [ctypes.c_void_p, _ip]
        L.ref_set_solver.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_set_field.argtypes = [ctypes.c_void_p, _dp]
        L.ref_get_field.argtypes = [ctypes.c_void_p, _dp]
        L.ref_set_dirichlet_activation.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.ref_set_dirichlet_value.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.ref_set_dirichlet_face_values.argtypes = [ctypes.c_void_p, _dp]
        L.ref_apply_dirichlet.argtypes = [ctypes.c_void_p]
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_max_threads.restype = ctypes.c_int
        L.ref_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.ref_set_bulk.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.ref_bulk_step.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.ref_add_agents.restype = ctypes.c_int
        L.ref_add_agents.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, ctypes.c_double]
        L.ref_agent_voxels.argtypes = [ctypes.c_void_p, _ip]
        L.ref_cells_step.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.ref_gradients.argtypes = [ctypes.c_void_p, _dp]
        L.ref_write_matlab.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.ref_print_densities.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.ref_gradients_per_voxel.argtypes = [ctypes.c_void_p, _dp]


class RefEnv:
    """One reference Microenvironment (see ref_driver.cpp)."""

    def __init__(self, ref: RefLib, bbox, dx, D, lam):
        self.ref = ref
        D, lam = f64(D), f64(lam)
        x0, y0, z0, x1, y1, z1 = bbox
        self.h = ref.lib.ref_create(x0, x1, y0, y1, z0, z1, dx, D.size, _d(D), _d(lam))
        s = np.zeros(4, dtype=np.int32)
        ref.lib.ref_sizes(self.h, _i(s))
        self.shape = tuple(int(v) for v in s)
        self.n_agents = 0

    def close(self):
        if self.h:
            self.ref.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_solver(self, which):
        self.ref.lib.ref_set_solver(self.h, which)

    def set_field(self, rho):
        rho = f64(rho)
        assert rho.size == int(np.prod(self.shape))
        self.ref.lib.ref_set_field(self.h, _d(rho))

    def field(self):
        out = np.zeros(self.shape)
        self.ref.lib.ref_get_field(self.h, _d(out))
        return out

    def set_dirichlet(self, activation, value=None, face_values=None):
        for d, a in enumerate(activation):
            self.ref.lib.ref_set_dirichlet_activation(self.h, d, int(bool(a)))
        if value is not None:
            for d, v in enumerate(value):
                self.ref.lib.ref_set_dirichlet_value(self.h, d, float(v))
        if face_values is not None:
            self.ref.lib.ref_set_dirichlet_face_values(self.h, _d(f64(face_values)))

    def apply_dirichlet(self):
        self.ref.lib.ref_apply_dirichlet(self.h)

    def step(self, dt, n=1):
        self.ref.lib.ref_step(self.h, dt, n)

    def set_bulk(self, S_rate, T_target, U_rate):
        self.ref.lib.ref_set_bulk(self.h, _d(f64(S_rate)), _d(f64(T_target)), _d(f64(U_rate)))

    def bulk_step(self, dt):
        self.ref.lib.ref_bulk_step(self.h, dt)

    def add_agents(self, pos, volume, sec, upt, sat, dt):
        pos, volume, sec, upt, sat = f64(pos), f64(volume), f64(sec), f64(upt), f64(sat)
        n = pos.shape[0]
        acc = self.ref.lib.ref_add_agents(self.h, n, _d(pos), _d(volume), _d(sec), _d(upt), _d(sat), dt)
        self.n_agents += n
        return acc

    def agent_voxels(self):
        out = np.zeros(self.n_agents, dtype=np.int32)
        self.ref.lib.ref_agent_voxels(self.h, _i(out))
        return out

    def cells_step(self, dt):
        self.ref.lib.ref_cells_step(self.h, dt)

    def write_matlab(self, filename):
        self.ref.lib.ref_write_matlab(self.h, str(filename).encode())

    def print_densities(self, filename):
        """The text dump of print_result / print_voxels_densities (appends)."""
        self.ref.lib.ref_print_densities(self.h, str(filename).encode())

    def gradients(self, per_voxel=False):
        """(nx, ny, nz, S, 3) gradient vectors from compute_all_gradient_vectors,
        or from the per-voxel accessor path."""
        out = np.zeros((*self.shape, 3))
        fn = self.ref.lib.ref_gradients_per_voxel if per_voxel else self.ref.lib.ref_gradients
        fn(self.h, _d(out))
        return out


def set_threads(ref: RefLib, n: int):
    os.environ.setdefault("OMP_PROC_BIND", "close")
    ref.lib.ref_set_threads(n)
