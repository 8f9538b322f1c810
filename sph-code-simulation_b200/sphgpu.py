"""Python binding of the C ABI in include/sphgpu.h (ctypes).

Mirrors the reference's module surface over a GPU context:

    sim = Simulation(params)            # Simulation(param) + BHTree::initialize
    sim.upload(fields)                  # particle arrays, caller order
    sim.initialize()                    # tail of Solver::initialize
    sim.integrate()                     # Solver::integrate + update_time
    sim.tree_make(); sim.pre_interaction(); sim.fluid_force(); ...

Errors from the library raise :class:`SPHException` (the reference's
THROW_ERROR -> sph::SPHException convention, include/exception.hpp:9-14).
There is no CPU fallback: loading fails loudly when libsphgpu.so is absent,
and compute calls fail when no sm_100 device is present.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsphgpu.so")

# enums, field names and the parameter struct live in sphparams (no library load)
from sphparams import (CUBIC_SPLINE, DISPH, FIELD_INDEX, FIELDS, FP64, GAUSSIAN, GDISPH, GSPH,  # noqa: F401
                       GUESS_MLP, GUESS_NONE, MIXED, NFIELDS, RIEMANN_HLL, RIEMANN_ITERATIVE, SRGSPH, SSPH,
                       WENDLAND, Params, config_params)
STAGES = ["timestep", "predict", "tree", "gather_walk", "pre", "set_kernel", "pair_walk",
          "force", "gravity", "correct", "recheck"]


class SPHException(RuntimeError):
    """Raised for fatal (<0) status codes of the C ABI."""


class LaneEmden(C.Structure):
    """A tabulated Lane-Emden solution and its scaling (sphgpu_lane_emden)."""
    _fields_ = [("alpha_scaling", C.c_double), ("K", C.c_double), ("xi_1", C.c_double),
                ("xi", C.POINTER(C.c_double)), ("theta", C.POINTER(C.c_double)),
                ("dtheta", C.POINTER(C.c_double)), ("npts", C.c_int64)]


class CsvMeta(C.Structure):
    """Header values of a CSV v1 snapshot (sphgpu_csv_meta)."""
    _fields_ = [("step", C.c_int), ("time", C.c_double), ("sph_type", C.c_int), ("kernel", C.c_int),
                ("gamma", C.c_double), ("g_constant", C.c_double), ("neighbor_number", C.c_int),
                ("use_gravity", C.c_int), ("use_balsara", C.c_int), ("use_time_dependent_av", C.c_int),
                ("kinetic", C.c_double), ("thermal", C.c_double), ("potential", C.c_double),
                ("precision", C.c_int), ("timestamp", C.c_char_p)]


CSV_FIELDS = ["pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "acc_x", "acc_y", "acc_z", "mass", "dens",
              "pres", "ene", "sml", "sound", "alpha", "balsara", "gradh", "phi", "neighbor"]


def csv_write(path: str, fields: Dict[str, np.ndarray], meta: "CsvMeta", ids=None):
    """Write host arrays as a CSV v1 snapshot (no device needed)."""
    n = len(next(iter(fields.values()))) if fields else 0
    ptrs, keep = _field_ptrs({k: v for k, v in fields.items() if k in FIELD_INDEX}, n, False)
    idp = None
    if ids is not None:
        ids = np.ascontiguousarray(ids, dtype=np.int64)
        idp = ids.ctypes.data_as(C.POINTER(C.c_int64))
    rc = lib().sphgpu_csv_write_host(path.encode(), n, ptrs, idp, C.byref(meta))
    if rc < 0:
        raise SPHException(f"csv_write failed ({rc}) for {path}")


def csv_read(path: str):
    """(fields, ids, meta) of a CSV v1 snapshot."""
    n = C.c_int64()
    meta = CsvMeta()
    if lib().sphgpu_csv_read_host(path.encode(), C.byref(n), 0, None, None, None) < 0:
        raise SPHException(f"csv_read failed for {path}")
    out = {f: np.zeros(n.value) for f in CSV_FIELDS}
    ids = np.zeros(n.value, dtype=np.int64)
    ptrs, _ = _field_ptrs(out, n.value, True)
    rc = lib().sphgpu_csv_read_host(path.encode(), C.byref(n), n.value, ptrs,
                                    ids.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(meta))
    if rc < 0:
        raise SPHException(f"csv_read failed ({rc}) for {path}")
    return out, ids, meta


class Counters(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "newton_nonconverged", "riemann_solves", "riemann_iterations", "riemann_fallbacks",
        "gather_capacity", "max_gather", "max_pair", "node_count", "retries", "walk_group_warps",
        "walk_split_warps", "walk_fallbacks", "mlp_guesses", "force_list_builds", "pre_candidates",
        "pre_newton_pairs", "pre_pairs", "pre_list_entries", "force_candidates", "force_pairs", "gravity_nodes",
        "gravity_monopoles", "gravity_leaf_pairs", "mixed_rechecks", "skin_builds",
        "skin_reuses")]


_lib = None


def lib() -> C.CDLL:
    """Load libsphgpu.so (built in-tree by build.py); raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() first")
    L = C.CDLL(LIB_PATH)
    vp, i64, i32p, i64p, dp = C.c_void_p, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_double)
    dpp = C.POINTER(C.POINTER(C.c_double))
    sig = {
        "sphgpu_default_params": (None, [C.POINTER(Params)]),
        "sphgpu_create": (C.c_int, [C.POINTER(Params), C.POINTER(vp)]),
        "sphgpu_destroy": (C.c_int, [vp]),
        "sphgpu_last_error": (C.c_char_p, [vp]),
        "sphgpu_device_ok": (C.c_int, []),
        "sphgpu_upload": (C.c_int, [vp, i64, dpp]),
        "sphgpu_download": (C.c_int, [vp, dpp]),
        "sphgpu_particle_num": (i64, [vp]),
        "sphgpu_get_time": (C.c_int, [vp, dp, dp]),
        "sphgpu_set_dt": (C.c_int, [vp, C.c_double]),
        "sphgpu_get_h_per_v_sig": (C.c_int, [vp, dp]),
        "sphgpu_tree_make": (C.c_int, [vp]),
        "sphgpu_tree_set_kernel": (C.c_int, [vp]),
        "sphgpu_neighbor_search": (C.c_int, [vp, C.c_int, i64p, i32p, i64]),
        "sphgpu_force_pairs": (C.c_int, [vp, i64p, i32p, i64]),
        "sphgpu_exhaustive_search": (C.c_int, [vp, C.c_int, i64p, i32p, i64]),
        "sphgpu_pre_interaction": (C.c_int, [vp]),
        "sphgpu_fluid_force": (C.c_int, [vp]),
        "sphgpu_gravity_force": (C.c_int, [vp]),
        "sphgpu_gravity_direct": (C.c_int, [vp]),
        "sphgpu_timestep": (C.c_int, [vp, dp]),
        "sphgpu_predict": (C.c_int, [vp]),
        "sphgpu_correct": (C.c_int, [vp]),
        "sphgpu_initialize": (C.c_int, [vp]),
        "sphgpu_integrate": (C.c_int, [vp]),
        "sphgpu_integrate_host": (C.c_int, [vp, dpp, dpp]),
        "sphgpu_energies": (C.c_int, [vp, dp, dp, dp, dp]),
        "sphgpu_write_csv": (C.c_int, [vp, C.c_char_p, C.c_int, C.c_int]),
        "sphgpu_relax_step": (C.c_int, [vp, C.POINTER(LaneEmden), C.c_int, dp]),
        "sphgpu_read_csv": (C.c_int, [vp, C.c_char_p, C.POINTER(C.c_int)]),
        "sphgpu_csv_write_host": (C.c_int, [C.c_char_p, i64, dpp, i64p, C.POINTER(CsvMeta)]),
        "sphgpu_csv_read_host": (C.c_int, [C.c_char_p, i64p, i64, dpp, i64p, C.POINTER(CsvMeta)]),
        "sphgpu_get_counters": (C.c_int, [vp, C.POINTER(Counters)]),
        "sphgpu_reset_counters": (C.c_int, [vp]),
        "sphgpu_enable_timing": (C.c_int, [vp, C.c_int]),
        "sphgpu_get_stage_times": (C.c_int, [vp, dp, i64p]),
        "sphgpu_synchronize": (C.c_int, [vp]),
        "sphgpu_test_flag_pass_guard": (C.c_int, [vp, C.c_int]),
        "sphgpu_set_initial_smoothing": (C.c_int, [vp, C.c_int]),
        "sphgpu_set_walk_mode": (C.c_int, [vp, C.c_int]),
        "sphgpu_timer_start": (C.c_int, [vp]),
        "sphgpu_timer_stop": (C.c_int, [vp, dp]),
        "sphgpu_launch_count": (i64, [vp]),
        "sphgpu_tree_nodes": (i64, [vp, i32p, dp, i64]),
        "sphgpu_mlp_param_count": (i64, []),
        "sphgpu_mlp_set_params": (C.c_int, [vp, C.POINTER(C.c_float)]),
        "sphgpu_mlp_get_params": (C.c_int, [vp, C.POINTER(C.c_float)]),
        "sphgpu_mlp_init": (C.c_int, [vp, C.c_uint64]),
        "sphgpu_mlp_predict": (C.c_int, [vp, dp, i64, C.POINTER(C.c_float)]),
        "sphgpu_mlp_train": (C.c_int, [vp, dp, dp, i64, C.c_int, C.c_int, C.c_float, C.c_uint64,
                                       C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "sphgpu_riemann_batch": (C.c_int, [vp, dp, i64, C.c_int, dp, dp, i32p, i32p]),
        "sphgpu_harvest_begin": (C.c_int, [vp, i64, C.c_uint32]),
        "sphgpu_harvest_end": (C.c_int, [vp, dp, i64, i64p]),
        "sphgpu_sample_evrard": (i64, [C.c_int, C.c_double, C.c_double, dpp]),
        "sphgpu_sample_shear_layer": (i64, [C.c_double, C.c_double, C.c_double, dpp]),
        "sphgpu_sample_shock_tube": (i64, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, dpp]),
        "sphgpu_sample_sr_shock_tube": (i64, [C.c_double, C.c_double, C.c_double, C.c_double, dpp]),
        "sphgpu_timestep_noalloc": (C.c_int, [vp, vp, i64, C.c_double, C.c_double, C.c_double, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def default_params(**kw) -> Params:
    p = Params()
    lib().sphgpu_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        if k.startswith("range_"):
            setattr(p, k, (C.c_double * 3)(*v))
        else:
            setattr(p, k, v)
    return p


def device_ok() -> bool:
    return bool(lib().sphgpu_device_ok())


def _field_ptrs(arrays: Dict[str, np.ndarray], n: int, writable: bool):
    ptrs = (C.POINTER(C.c_double) * NFIELDS)()
    keep = []
    for name, arr in arrays.items():
        k = FIELD_INDEX[name]
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != (n,):
            raise ValueError(f"field {name}: shape {a.shape} != ({n},)")
        if writable and a is not arr:
            raise ValueError(f"field {name} must be a contiguous float64 array")
        keep.append(a)
        ptrs[k] = a.ctypes.data_as(C.POINTER(C.c_double))
    return ptrs, keep


def _sample(fn, *args) -> Dict[str, np.ndarray]:
    n = fn(*args, None)
    out = {f: np.zeros(n) for f in FIELDS}
    ptrs, _ = _field_ptrs(out, n, True)
    fn(*args, ptrs)
    return out


def sample_evrard(N: int, G: float = 1.0, gamma: float = 5.0 / 3.0) -> Dict[str, np.ndarray]:
    """Evrard sphere on an N^3 lattice (Solver::make_evrard, src/sample/evrard.cpp:13-87)."""
    return _sample(lib().sphgpu_sample_evrard, C.c_int(N), C.c_double(G), C.c_double(gamma))


def sample_shear_layer(dx: float, lz: float = 0.125, gamma: float = 5.0 / 3.0) -> Dict[str, np.ndarray]:
    """3-D periodic shear layer (Kelvin-Helmholtz set-up of src/sample/khi.cpp:12-73, extruded)."""
    return _sample(lib().sphgpu_sample_shear_layer, C.c_double(dx), C.c_double(lz), C.c_double(gamma))


def sample_shock_tube(dx: float, ly: float = 0.05, p_left: float = 1000.0, p_right: float = 0.01,
                      gamma: float = 1.4) -> Dict[str, np.ndarray]:
    """3-D shock tube along x in [-0.5, 0.5] x [0, ly]^2."""
    return _sample(lib().sphgpu_sample_shock_tube, C.c_double(dx), C.c_double(ly), C.c_double(p_left),
                   C.c_double(p_right), C.c_double(gamma))


def sample_sr_shock_tube(dx: float, ly: float = 0.05, gamma: float = 5.0 / 3.0,
                         c_speed: float = 1.0) -> Dict[str, np.ndarray]:
    """Special-relativistic Sod tube in 3-D (left n = 1, P = 1; right n = 0.125, P = 0.1)."""
    return _sample(lib().sphgpu_sample_sr_shock_tube, C.c_double(dx), C.c_double(ly), C.c_double(gamma),
                   C.c_double(c_speed))


class Simulation:
    """A GPU context: Simulation + BHTree + the per-step modules."""

    def __init__(self, params: Params):
        self.params = params.copy()
        self._h = C.c_void_p()
        rc = lib().sphgpu_create(C.byref(self.params), C.byref(self._h))
        if rc < 0:
            msg = self._err()
            lib().sphgpu_destroy(self._h)
            self._h = C.c_void_p()
            raise SPHException(f"sphgpu_create failed ({rc}): {msg}")
        self.n = 0

    # ---- lifetime
    def close(self):
        if self._h:
            lib().sphgpu_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _err(self) -> str:
        e = lib().sphgpu_last_error(self._h)
        return e.decode() if e else ""

    def _check(self, rc: int, what: str) -> int:
        if rc < 0:
            raise SPHException(f"{what} failed ({rc}): {self._err()}")
        return rc

    # ---- state
    def upload(self, fields: Dict[str, np.ndarray]):
        n = len(next(iter(fields.values())))
        ptrs, keep = _field_ptrs({k: v for k, v in fields.items() if k in FIELD_INDEX}, n, False)
        self._check(lib().sphgpu_upload(self._h, n, ptrs), "upload")
        self.n = n
        del keep

    def download(self, names=None) -> Dict[str, np.ndarray]:
        names = list(FIELDS) if names is None else list(names)
        out = {f: np.zeros(self.n) for f in names}
        ptrs, _ = _field_ptrs(out, self.n, True)
        self._check(lib().sphgpu_download(self._h, ptrs), "download")
        return out

    def time_dt(self):
        t, dt = C.c_double(), C.c_double()
        self._check(lib().sphgpu_get_time(self._h, C.byref(t), C.byref(dt)), "get_time")
        return t.value, dt.value

    def set_dt(self, dt: float):
        self._check(lib().sphgpu_set_dt(self._h, dt), "set_dt")

    def h_per_v_sig(self) -> float:
        v = C.c_double()
        self._check(lib().sphgpu_get_h_per_v_sig(self._h, C.byref(v)), "h_per_v_sig")
        return v.value

    # ---- modules
    def tree_make(self):
        return self._check(lib().sphgpu_tree_make(self._h), "BHTree::make")

    def set_kernel(self):
        return self._check(lib().sphgpu_tree_set_kernel(self._h), "BHTree::set_kernel")

    def neighbor_search(self, is_ij: bool = False, exhaustive: bool = False):
        """All particles' lists (radius sml) as a CSR (offsets[n+1], ids) in caller order."""
        off = np.zeros(self.n + 1, dtype=np.int64)
        fn = lib().sphgpu_exhaustive_search if exhaustive else lib().sphgpu_neighbor_search
        i64p, i32p = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
        self._check(fn(self._h, int(is_ij), off.ctypes.data_as(i64p), None, 0), "neighbor_search")
        ids = np.zeros(max(int(off[-1]), 1), dtype=np.int32)
        self._check(fn(self._h, int(is_ij), off.ctypes.data_as(i64p), ids.ctypes.data_as(i32p), ids.size),
                    "neighbor_search")
        return off, ids[: int(off[-1])]

    def force_pairs(self):
        """The pairs FluidForce sums over now (r < max(h_i, h_j)), CSR in caller order."""
        off = np.zeros(self.n + 1, dtype=np.int64)
        i64p, i32p = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
        self._check(lib().sphgpu_force_pairs(self._h, off.ctypes.data_as(i64p), None, 0), "force_pairs")
        ids = np.zeros(max(int(off[-1]), 1), dtype=np.int32)
        self._check(lib().sphgpu_force_pairs(self._h, off.ctypes.data_as(i64p), ids.ctypes.data_as(i32p), ids.size),
                    "force_pairs")
        return off, ids[: int(off[-1])]

    def pre_interaction(self):
        return self._check(lib().sphgpu_pre_interaction(self._h), "PreInteraction::calculation")

    def fluid_force(self):
        return self._check(lib().sphgpu_fluid_force(self._h), "FluidForce::calculation")

    def gravity_force(self, direct: bool = False):
        fn = lib().sphgpu_gravity_direct if direct else lib().sphgpu_gravity_force
        return self._check(fn(self._h), "GravityForce::calculation")

    def timestep(self) -> float:
        dt = C.c_double()
        self._check(lib().sphgpu_timestep(self._h, C.byref(dt)), "TimeStep::calculation")
        return dt.value

    def predict(self):
        return self._check(lib().sphgpu_predict(self._h), "predict")

    def correct(self):
        return self._check(lib().sphgpu_correct(self._h), "correct")

    def initialize(self):
        return self._check(lib().sphgpu_initialize(self._h), "initialize")

    def integrate(self):
        return self._check(lib().sphgpu_integrate(self._h), "integrate")

    def integrate_host(self, fields: Dict[str, np.ndarray], out_names=None) -> Dict[str, np.ndarray]:
        """One step on host buffers (sphgpu_integrate_host): `fields` replace
        the device state, the step runs, the named fields come back."""
        names = list(FIELDS) if out_names is None else list(out_names)
        ptrs_in, keep = _field_ptrs({k: v for k, v in fields.items() if k in FIELD_INDEX}, self.n, False)
        out = {f: np.zeros(self.n) for f in names}
        ptrs_out, _ = _field_ptrs(out, self.n, True)
        self._check(lib().sphgpu_integrate_host(self._h, ptrs_in, ptrs_out), "integrate_host")
        del keep
        return out

    def energies(self):
        k, u, w = C.c_double(), C.c_double(), C.c_double()
        mom = (C.c_double * 3)()
        self._check(lib().sphgpu_energies(self._h, C.byref(k), C.byref(u), C.byref(w),
                                          C.cast(mom, C.POINTER(C.c_double))), "energies")
        return k.value, u.value, w.value, np.array(mom[:])

    def relax_step(self, xi, theta, dtheta, xi_1: float, alpha: float, K: float, first: bool = False) -> float:
        """One Lane-Emden relaxation step; returns dt_relax."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (xi, theta, dtheta)]
        dp = C.POINTER(C.c_double)
        le = LaneEmden(alpha, K, xi_1, arrs[0].ctypes.data_as(dp), arrs[1].ctypes.data_as(dp),
                       arrs[2].ctypes.data_as(dp), len(arrs[0]))
        d = C.c_double()
        self._check(lib().sphgpu_relax_step(self._h, C.byref(le), int(first), C.byref(d)), "relax_step")
        return d.value

    def write_csv(self, path: str, step: int = 0, precision: int = 16):
        """Snapshot in the reference's CSV v1 format (caller order, code units)."""
        self._check(lib().sphgpu_write_csv(self._h, path.encode(), int(step), int(precision)), "write_csv")

    def read_csv(self, path: str) -> int:
        """Resume from a CSV v1 snapshot (particles and time); returns its step."""
        n = C.c_int64()
        if lib().sphgpu_csv_read_host(path.encode(), C.byref(n), 0, None, None, None) < 0:
            raise SPHException(f"read_csv: cannot read {path}")
        step = C.c_int()
        self._check(lib().sphgpu_read_csv(self._h, path.encode(), C.byref(step)), "read_csv")
        self.n = n.value
        return step.value

    def set_walk_mode(self, mode: int):
        """0 = group walk (default), 1 = per-lane walk (cross-check)."""
        self._check(lib().sphgpu_set_walk_mode(self._h, int(mode)), "set_walk_mode")

    def set_initial_smoothing(self, on: bool):
        self._check(lib().sphgpu_set_initial_smoothing(self._h, int(on)), "set_initial_smoothing")

    def tree_nodes(self):
        """Preorder node table: ints (level, is_leaf, num), dbl (center3, edge, mass, mcenter3, ksize)."""
        k = self._check(lib().sphgpu_tree_nodes(self._h, None, None, 0), "tree_nodes")
        ints = np.zeros((k, 3), dtype=np.int32)
        dbl = np.zeros((k, 9), dtype=np.float64)
        self._check(lib().sphgpu_tree_nodes(self._h, ints.ctypes.data_as(C.POINTER(C.c_int32)),
                                            dbl.ctypes.data_as(C.POINTER(C.c_double)), k), "tree_nodes")
        return ints, dbl

    # ---- diagnostics
    def counters(self) -> Dict[str, int]:
        c = Counters()
        self._check(lib().sphgpu_get_counters(self._h, C.byref(c)), "counters")
        return {n: getattr(c, n) for n, _ in Counters._fields_}

    def reset_counters(self):
        self._check(lib().sphgpu_reset_counters(self._h), "reset_counters")

    def enable_timing(self, on: bool = True):
        self._check(lib().sphgpu_enable_timing(self._h, int(on)), "enable_timing")

    def stage_times(self):
        ms = (C.c_double * len(STAGES))()
        la = (C.c_int64 * len(STAGES))()
        self._check(lib().sphgpu_get_stage_times(self._h, C.cast(ms, C.POINTER(C.c_double)),
                                                 C.cast(la, C.POINTER(C.c_int64))), "stage_times")
        return {s: (ms[k], la[k]) for k, s in enumerate(STAGES)}

    def synchronize(self):
        self._check(lib().sphgpu_synchronize(self._h), "synchronize")

    # ---- learned Riemann guess
    def mlp_set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != lib().sphgpu_mlp_param_count():
            raise ValueError("wrong MLP parameter count")
        self._check(lib().sphgpu_mlp_set_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float))), "mlp_set_params")

    def load_riemann_mlp(self, path: Optional[str] = None):
        """Load trained weights (default: riemann_mlp_weights.npy beside this file)."""
        path = path or os.path.join(HERE, "riemann_mlp_weights.npy")
        self.mlp_set_params(np.load(path))

    def mlp_init(self, seed: int = 12345):
        self._check(lib().sphgpu_mlp_init(self._h, seed), "mlp_init")

    def mlp_predict(self, states: np.ndarray) -> np.ndarray:
        st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 7)
        y = np.zeros(len(st), dtype=np.float32)
        self._check(lib().sphgpu_mlp_predict(self._h, st.ctypes.data_as(C.POINTER(C.c_double)), len(st),
                                             y.ctypes.data_as(C.POINTER(C.c_float))), "mlp_predict")
        return y

    def mlp_train(self, states: np.ndarray, pstar: np.ndarray, epochs: int, batch: int = 16384,
                  lr: float = 2e-3, seed: int = 12345):
        """Train; epochs = 0 returns (loss, gradient) of the current parameters."""
        st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 7)
        ps = np.ascontiguousarray(pstar, dtype=np.float64)
        hist = np.zeros(max(epochs, 1), dtype=np.float32)
        grad = np.zeros(lib().sphgpu_mlp_param_count(), dtype=np.float32)
        fp = C.POINTER(C.c_float)
        self._check(lib().sphgpu_mlp_train(self._h, st.ctypes.data_as(C.POINTER(C.c_double)),
                                           ps.ctypes.data_as(C.POINTER(C.c_double)), len(st), epochs, batch, lr,
                                           seed, hist.ctypes.data_as(fp), grad.ctypes.data_as(fp)), "mlp_train")
        return (hist[0], grad) if epochs == 0 else hist

    def riemann_batch(self, states: np.ndarray, mode: int):
        """(p*, v*, iterations, fallbacks) for n x 7 states; mode as in sphgpu.h."""
        st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 7)
        n = len(st)
        p, v = np.zeros(n), np.zeros(n)
        it, fb = np.zeros(n, dtype=np.int32), np.zeros(n, dtype=np.int32)
        dp_ = C.POINTER(C.c_double)
        i32p = C.POINTER(C.c_int32)
        self._check(lib().sphgpu_riemann_batch(self._h, st.ctypes.data_as(dp_), n, mode, p.ctypes.data_as(dp_),
                                               v.ctypes.data_as(dp_), it.ctypes.data_as(i32p),
                                               fb.ctypes.data_as(i32p)), "riemann_batch")
        return p, v, it, fb

    def harvest_begin(self, capacity: int, sample_mod: int):
        self._check(lib().sphgpu_harvest_begin(self._h, capacity, sample_mod), "harvest_begin")

    def harvest_end(self, capacity: int) -> np.ndarray:
        out = np.zeros((capacity, 8))
        cnt = C.c_int64()
        self._check(lib().sphgpu_harvest_end(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), capacity,
                                             C.byref(cnt)), "harvest_end")
        return out[: cnt.value]

    def mlp_get_params(self) -> np.ndarray:
        p = np.zeros(lib().sphgpu_mlp_param_count(), dtype=np.float32)
        self._check(lib().sphgpu_mlp_get_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float))), "mlp_get_params")
        return p
