"""ctypes loaders for the parity checkers (TEST INFRASTRUCTURE ONLY).

    Oracle(params, fields, exhaustive=False)  the CPU restatement (liboracle.so)
    Reference(params, fields, exhaustive=False)  the reference's own modules
                                              compiled into _ref/ (when built)

Both expose the same methods as the GPU binding where they overlap
(initialize, integrate, tree_make, pre_interaction, fluid_force,
gravity_force, timestep, predict, correct, energies, download,
neighbor_lists).  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libsphref.so")
REF_EXH_LIB = os.path.join(HERE, "_ref", "libsphref_exh.so")
REF_GPU_LIB = os.path.join(HERE, "_ref", "libsphref_gpu.so")

# the field order of include/sphgpu.h
FIELDS = [
    "pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "velp_x", "velp_y", "velp_z",
    "acc_x", "acc_y", "acc_z", "mass", "dens", "pres", "ene", "ene_p", "dene", "sml", "sound",
    "balsara", "alpha", "gradh", "phi", "neighbor",
    "grad_d_x", "grad_d_y", "grad_d_z", "grad_p_x", "grad_p_y", "grad_p_z",
    "grad_v0_x", "grad_v0_y", "grad_v0_z", "grad_v1_x", "grad_v1_y", "grad_v1_z",
    "grad_v2_x", "grad_v2_y", "grad_v2_z",
    "sr_S_x", "sr_S_y", "sr_S_z", "sr_e", "sr_N", "sr_nu", "sr_gamma_lor", "sr_enthalpy",
    "sr_dS_x", "sr_dS_y", "sr_dS_z", "sr_de",
]
NF = len(FIELDS)
FI = {f: k for k, f in enumerate(FIELDS)}


def refdir() -> str:
    """The reference checkout: $REFDIR, else a "reference" directory beside
    the repository (the Makefile's default)."""
    return os.environ.get("REFDIR") or os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference"))


def build(reference: bool = True) -> None:
    """make -C oracle (the reference part only when its sources are present)."""
    targets = ["oracle"]
    if reference and os.path.isdir(refdir()):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def have_reference() -> bool:
    return os.path.exists(REF_LIB) and os.path.exists(REF_EXH_LIB)


def _ptrs(arrays: Dict[str, np.ndarray], n: int):
    ptrs = (C.POINTER(C.c_double) * NF)()
    keep = []
    for name, arr in arrays.items():
        if name not in FI:
            continue
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.shape == (n,)
        keep.append(a)
        ptrs[FI[name]] = a.ctypes.data_as(C.POINTER(C.c_double))
    return ptrs, keep


_libs: Dict[str, C.CDLL] = {}


def _load(path: str, prefix: str) -> C.CDLL:
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise ImportError(f"{path} not built (make -C oracle)")
    L = C.CDLL(path)
    vp, dp = C.c_void_p, C.POINTER(C.c_double)
    dpp = C.POINTER(C.POINTER(C.c_double))
    i64p, i32p = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
    if prefix == "oracle":
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [C.c_void_p, C.c_int64, dpp, C.c_int]
        L.oracle_gravity.argtypes = [vp, C.c_int]
        L.oracle_tree_nodes.restype = C.c_int64
        L.oracle_tree_nodes.argtypes = [vp, i32p, dp, C.c_int64]
        L.oracle_energies.argtypes = [vp, dp, dp, dp, dp]
        L.oracle_counters.argtypes = [vp, i64p]
        L.oracle_set_first.argtypes = [vp, C.c_int]
        for f in ("oracle_kernel_w", "oracle_kernel_dwc", "oracle_kernel_dhw"):
            getattr(L, f).restype = C.c_double
            getattr(L, f).argtypes = [C.c_int, C.c_double, C.c_double]
        L.oracle_riemann.restype = C.c_int
        L.oracle_riemann.argtypes = [C.c_int, dp, dp, C.c_double, dp, dp]
        L.oracle_relax_step.argtypes = [vp, dp, dp, dp, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_int, dp]
    else:
        L.ref_create.restype = vp
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_max_threads.restype = C.c_int
        L.ref_create.argtypes = [C.c_void_p, C.c_int64, dpp]
        L.ref_energies.argtypes = [vp, dp, dp, dp]
        L.ref_module_times.argtypes = [vp, dp]
        L.ref_relax_step.argtypes = [vp, C.c_char_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, dp]
        L.ref_set_swap_mode.restype = C.c_int
        L.ref_set_swap_mode.argtypes = [C.c_int]
    for name in ("destroy", "get", "set", "tree_make", "set_kernel", "pre", "force", "timestep", "predict",
                 "correct", "initialize", "integrate", "neighbor_lists", "get_dt", "set_dt", "get_time",
                 "get_h_per_v_sig", "last_error"):
        fn = getattr(L, f"{prefix}_{name}")
        if name in ("get_dt", "get_time", "get_h_per_v_sig"):
            fn.restype = C.c_double
            fn.argtypes = [vp]
        elif name == "set_dt":
            fn.argtypes = [vp, C.c_double]
        elif name == "last_error":
            fn.restype = C.c_char_p
            fn.argtypes = [vp]
        elif name in ("get", "set"):
            fn.argtypes = [vp, dpp]
        elif name == "neighbor_lists":
            fn.argtypes = [vp, C.c_int, i64p, i32p, C.c_int64]
        elif name == "destroy":
            fn.restype = None
            fn.argtypes = [vp]   # a 64-bit handle: undeclared, ctypes would pass a C int
        else:
            fn.argtypes = [vp]
    if prefix == "ref":
        L.ref_gravity.argtypes = [vp]
    _libs[path] = L
    return L


class _Base:
    prefix = ""

    def _call(self, name, *args):
        rc = getattr(self.L, f"{self.prefix}_{name}")(self.h, *args)
        if rc is not None and rc < 0:
            msg = getattr(self.L, f"{self.prefix}_last_error")(self.h)
            raise RuntimeError(f"{self.prefix}_{name} failed: {msg.decode() if msg else ''}")
        return rc

    def close(self):
        if self.h:
            getattr(self.L, f"{self.prefix}_destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def download(self, names=None) -> Dict[str, np.ndarray]:
        names = FIELDS if names is None else names
        out = {f: np.zeros(self.n) for f in names}
        ptrs, _ = _ptrs(out, self.n)
        self._call("get", ptrs)
        return out

    def upload_fields(self, fields: Dict[str, np.ndarray]):
        ptrs, keep = _ptrs(fields, self.n)
        self._call("set", ptrs)

    def tree_make(self):
        self._call("tree_make")

    def set_kernel(self):
        self._call("set_kernel")

    def pre_interaction(self):
        self._call("pre")

    def fluid_force(self):
        self._call("force")

    def timestep(self) -> float:
        self._call("timestep")
        return self.dt

    def predict(self):
        self._call("predict")

    def correct(self):
        self._call("correct")

    def initialize(self):
        self._call("initialize")

    def integrate(self):
        self._call("integrate")

    @property
    def dt(self) -> float:
        return getattr(self.L, f"{self.prefix}_get_dt")(self.h)

    def set_dt(self, dt: float):
        getattr(self.L, f"{self.prefix}_set_dt")(self.h, dt)

    @property
    def time(self) -> float:
        return getattr(self.L, f"{self.prefix}_get_time")(self.h)

    def h_per_v_sig(self) -> float:
        return getattr(self.L, f"{self.prefix}_get_h_per_v_sig")(self.h)

    def neighbor_lists(self, is_ij: bool = False):
        """Distance-sorted lists (radius sml) as CSR (offsets, ids)."""
        off = np.zeros(self.n + 1, dtype=np.int64)
        i64p, i32p = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
        self._call("neighbor_lists", int(is_ij), off.ctypes.data_as(i64p), None, 0)
        ids = np.zeros(max(int(off[-1]), 1), dtype=np.int32)
        self._call("neighbor_lists", int(is_ij), off.ctypes.data_as(i64p), ids.ctypes.data_as(i32p), ids.size)
        return off, ids[: int(off[-1])]


class Oracle(_Base):
    """The CPU restatement (oracle/sph_oracle.cpp)."""

    prefix = "oracle"

    def __init__(self, params, fields: Dict[str, np.ndarray], exhaustive: bool = False):
        self.L = _load(ORACLE_LIB, "oracle")
        self.n = len(fields["pos_x"])
        ptrs, keep = _ptrs(fields, self.n)
        self.h = self.L.oracle_create(C.byref(params), self.n, ptrs, int(exhaustive))

    def gravity_force(self, direct: bool = False):
        self._call("gravity", int(direct))

    def relax_step(self, table, xi_1: float, alpha: float, K: float, first: bool) -> float:
        """One Lane-Emden relaxation step; table = (xi, theta, dtheta) arrays.  Returns dt_relax."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in table]
        dp = C.POINTER(C.c_double)
        d = C.c_double()
        self._call("relax_step", *[a.ctypes.data_as(dp) for a in arrs], len(arrs[0]), xi_1, alpha, K, int(first),
                   C.byref(d))
        return d.value

    def energies(self):
        k, u, w = C.c_double(), C.c_double(), C.c_double()
        mom = (C.c_double * 3)()
        self.L.oracle_energies(self.h, C.byref(k), C.byref(u), C.byref(w), C.cast(mom, C.POINTER(C.c_double)))
        return k.value, u.value, w.value, np.array(mom[:])

    def counters(self):
        out = (C.c_int64 * 3)()
        self.L.oracle_counters(self.h, C.cast(out, C.POINTER(C.c_int64)))
        return {"newton_nonconverged": out[0], "riemann_solves": out[1], "riemann_iterations": out[2]}

    def set_first(self, first: bool):
        self.L.oracle_set_first(self.h, int(first))

    def tree_nodes(self):
        """Preorder node table: ints (level, is_leaf, num), dbl (center3, edge, mass, mcenter3, ksize)."""
        k = self.L.oracle_tree_nodes(self.h, None, None, 0)
        ints = np.zeros((k, 3), dtype=np.int32)
        dbl = np.zeros((k, 9), dtype=np.float64)
        self.L.oracle_tree_nodes(self.h, ints.ctypes.data_as(C.POINTER(C.c_int32)),
                                 dbl.ctypes.data_as(C.POINTER(C.c_double)), k)
        return ints, dbl


class Reference(_Base):
    """The reference's own modules (oracle/_ref), for pinning the oracle."""

    prefix = "ref"

    def __init__(self, params, fields: Dict[str, np.ndarray], exhaustive: bool = False, threads: int = 0):
        """threads: OpenMP team size (0: OMP_NUM_THREADS, else every host
        core, at least 2).  With one thread BHTree::make's root box is the
        particles' own bounding box (tree_root_origin = 0); with more it also
        covers the origin (tree_root_origin = 1)."""
        self.L = _load(REF_EXH_LIB if exhaustive else REF_LIB, "ref")
        if threads <= 0:
            threads = int(os.environ.get("OMP_NUM_THREADS", "0") or 0) or max(2, os.cpu_count() or 2)
        self.L.ref_set_threads(threads)
        self.n = len(fields["pos_x"])
        ptrs, keep = _ptrs(fields, self.n)
        self.h = self.L.ref_create(C.byref(params), self.n, ptrs)

    def gravity_force(self, direct: bool = False):
        self._call("gravity")

    def relax_step(self, refdir: str, alpha: float, rho_c: float, K: float, R: float, M: float) -> float:
        """One step of the reference's relaxation loop.  Returns dt_relax."""
        d = C.c_double()
        self._call("relax_step", refdir.encode(), alpha, rho_c, K, R, M, C.byref(d))
        return d.value

    def energies(self):
        k, u, w = C.c_double(), C.c_double(), C.c_double()
        self.L.ref_energies(self.h, C.byref(k), C.byref(u), C.byref(w))
        return k.value, u.value, w.value, None

    def module_times(self):
        out = (C.c_double * 7)()
        self.L.ref_module_times(self.h, C.cast(out, C.POINTER(C.c_double)))
        return list(out)


class ReferenceWithGpuModules(Reference):
    """The reference's Solver sequence (oracle/ref_harness.cpp) with the GPU
    modules of sph-code-simulation_b200/host/gpu_modules.hpp swapped in for
    TimeStep, PreInteraction, FluidForce, GravityForce and make_tree
    (oracle/_ref/libsphref_gpu.so).  resident=False keeps Solver::predict /
    correct on the host (MIRROR), True runs them on the device (RESIDENT)."""

    def __init__(self, params, fields: Dict[str, np.ndarray], resident: bool = False, threads: int = 0):
        self.L = _load(REF_GPU_LIB, "ref")
        if threads <= 0:
            threads = int(os.environ.get("OMP_NUM_THREADS", "0") or 0) or max(2, os.cpu_count() or 2)
        self.L.ref_set_threads(threads)
        self.L.ref_set_swap_mode(int(resident))
        self.n = len(fields["pos_x"])
        ptrs, keep = _ptrs(fields, self.n)
        self.h = self.L.ref_create(C.byref(params), self.n, ptrs)
        if not self.h:
            raise RuntimeError("ref_create failed")


def kernel_w(kind: int, r: float, h: float) -> float:
    return _load(ORACLE_LIB, "oracle").oracle_kernel_w(kind, r, h)


def kernel_dwc(kind: int, r: float, h: float) -> float:
    return _load(ORACLE_LIB, "oracle").oracle_kernel_dwc(kind, r, h)


def kernel_dhw(kind: int, r: float, h: float) -> float:
    return _load(ORACLE_LIB, "oracle").oracle_kernel_dhw(kind, r, h)


def riemann(solver: int, left, right, gamma: float):
    """(p*, v*, iterations) of the HLL (0) or iterative (1) solver; state = (u, rho, p, c)."""
    L = _load(ORACLE_LIB, "oracle")
    l = (C.c_double * 4)(*left)
    r = (C.c_double * 4)(*right)
    p, v = C.c_double(), C.c_double()
    it = L.oracle_riemann(solver, C.cast(l, C.POINTER(C.c_double)), C.cast(r, C.POINTER(C.c_double)), gamma,
                          C.byref(p), C.byref(v))
    return p.value, v.value, it
