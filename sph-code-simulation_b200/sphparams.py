"""Parameters of the SPH step (sphgpu_params, include/sphgpu.h) without the
device library: the struct, its defaults and the benchmark workloads'
parameter sets.  Importing this module loads no shared library, so callers
that only describe a workload (the CPU reference arm of bench.py, the IC
generators) stay off libsphgpu.so.

Defaults are the reference's JSON defaults (src/solver.cpp:311-438), the
same values sphgpu_default_params writes (tests/test_capi.py checks that the
two agree field by field).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict

# enums (include/sphgpu.h)
SSPH, DISPH, GSPH, GDISPH, SRGSPH = 0, 1, 2, 3, 4
CUBIC_SPLINE, WENDLAND, GAUSSIAN = 0, 1, 2
RIEMANN_HLL, RIEMANN_ITERATIVE = 0, 1
FP64, MIXED = 0, 1
GUESS_NONE, GUESS_MLP = 0, 1

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
NFIELDS = len(FIELDS)
FIELD_INDEX = {f: k for k, f in enumerate(FIELDS)}


class Params(C.Structure):
    """sphgpu_params (include/sphgpu.h); field names follow the JSON keys."""

    _fields_ = [
        ("sph_type", C.c_int32), ("kernel", C.c_int32), ("neighbor_number", C.c_int32),
        ("iterative_sml", C.c_int32), ("gamma", C.c_double), ("cfl_sound", C.c_double),
        ("cfl_force", C.c_double), ("av_alpha", C.c_double), ("use_balsara_switch", C.c_int32),
        ("use_time_dependent_av", C.c_int32), ("alpha_max", C.c_double), ("alpha_min", C.c_double),
        ("epsilon_av", C.c_double), ("use_ac", C.c_int32), ("max_tree_level", C.c_int32),
        ("alpha_ac", C.c_double), ("leaf_particle_num", C.c_int32), ("periodic", C.c_int32),
        ("range_min", C.c_double * 3), ("range_max", C.c_double * 3), ("use_gravity", C.c_int32),
        ("gsph_2nd_order", C.c_int32), ("g_constant", C.c_double), ("theta", C.c_double),
        ("riemann_solver", C.c_int32), ("precision", C.c_int32), ("riemann_guess", C.c_int32),
        ("mlp_max_newton", C.c_int32), ("sr_2nd_order", C.c_int32), ("tree_root_origin", C.c_int32),
        ("sr_c_speed", C.c_double), ("sr_c_shock", C.c_double), ("sr_c_cd", C.c_double), ("sr_eta", C.c_double),
        ("sr_c_smooth", C.c_double), ("mixed_acc_tol", C.c_double), ("riemann_tol", C.c_double),
        ("gather_skin", C.c_double),
    ]

    def copy(self) -> "Params":
        p = Params()
        C.memmove(C.byref(p), C.byref(self), C.sizeof(Params))
        return p

    def as_dict(self) -> Dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if name.startswith("range_") else v
        return out


DEFAULTS = dict(
    sph_type=SSPH, kernel=CUBIC_SPLINE, neighbor_number=50, iterative_sml=1, gamma=1.6666666666666667,
    cfl_sound=0.3, cfl_force=0.125, av_alpha=1.0, use_balsara_switch=1, use_time_dependent_av=0,
    alpha_max=2.0, alpha_min=0.1, epsilon_av=0.2, use_ac=0, max_tree_level=20, alpha_ac=1.0,
    leaf_particle_num=1, periodic=0, use_gravity=0, gsph_2nd_order=1, g_constant=1.0, theta=0.5,
    riemann_solver=RIEMANN_HLL, precision=FP64, riemann_guess=GUESS_NONE, mlp_max_newton=4,
    sr_2nd_order=1, tree_root_origin=1, sr_c_speed=1.0, sr_c_shock=3.0, sr_c_cd=1.0, sr_eta=1.0,
    sr_c_smooth=2.0, mixed_acc_tol=0.0, riemann_tol=1e-6, gather_skin=0.02,
)


def _set(p: Params, k: str, v) -> None:
    if not hasattr(p, k):
        raise KeyError(k)
    if k.startswith("range_"):
        setattr(p, k, (C.c_double * 3)(*v))
    else:
        setattr(p, k, v)


def defaults(**kw) -> Params:
    """The defaults above (range_min = range_max = 0), then the overrides."""
    p = Params()
    for k, v in DEFAULTS.items():
        setattr(p, k, v)
    for k, v in kw.items():
        _set(p, k, v)
    return p


def config_params(name: str, **overrides) -> Params:
    """Parameters of the benchmark workloads (names describe the workload)."""
    if name == "evrard_ssph":          # ssph Evrard sphere, cubic spline, K=50, leaf=1
        p = defaults(sph_type=SSPH, kernel=CUBIC_SPLINE, neighbor_number=50, use_balsara_switch=1,
                     av_alpha=1.0, use_gravity=1, g_constant=1.0, theta=0.5, leaf_particle_num=1,
                     gamma=5.0 / 3.0, cfl_sound=0.3)
    elif name == "shear_disph":        # disph periodic shear layer, Wendland, K=128, AC
        p = defaults(sph_type=DISPH, kernel=WENDLAND, neighbor_number=128, use_ac=1, alpha_ac=1.0,
                     periodic=1, range_min=(0.0, 0.0, 0.0), range_max=(1.0, 1.0, 0.125), gamma=5.0 / 3.0)
    elif name == "tube_gsph":          # gsph shock tube, MUSCL, iterative Riemann, cubic, K=50
        p = defaults(sph_type=GSPH, kernel=CUBIC_SPLINE, neighbor_number=50, gsph_2nd_order=1,
                     riemann_solver=RIEMANN_ITERATIVE, gamma=1.4, periodic=1,
                     range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.05, 0.05))
    elif name == "tube_gdisph":        # gdisph shock tube, MUSCL + HLL, cubic, K=50, Balsara, TD-AV, AC
        p = defaults(sph_type=GDISPH, kernel=CUBIC_SPLINE, neighbor_number=50, gsph_2nd_order=1,
                     riemann_solver=RIEMANN_HLL, gamma=1.4, periodic=1, use_balsara_switch=1,
                     use_time_dependent_av=1, alpha_min=0.1, alpha_max=2.0, epsilon_av=0.2, av_alpha=1.0,
                     use_ac=1, alpha_ac=1.0, range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.05, 0.05))
    elif name == "tube_srgsph":        # special-relativistic gsph Sod tube, MUSCL, exact SR solver, cubic, K=50
        p = defaults(sph_type=SRGSPH, kernel=CUBIC_SPLINE, neighbor_number=50, sr_2nd_order=1,
                     gamma=5.0 / 3.0, periodic=1, range_min=(-0.5, 0.0, 0.0), range_max=(0.5, 0.05, 0.05),
                     sr_c_speed=1.0, sr_c_shock=3.0, sr_c_cd=1.0, sr_eta=1.0, sr_c_smooth=2.0)
    elif name == "blast_gsph":         # gsph many-blast cube, MUSCL, iterative Riemann, cubic, K=50
        p = defaults(sph_type=GSPH, kernel=CUBIC_SPLINE, neighbor_number=50, gsph_2nd_order=1,
                     riemann_solver=RIEMANN_ITERATIVE, gamma=1.4, periodic=1,
                     range_min=(-0.5, -0.5, -0.5), range_max=(0.5, 0.5, 0.5))
    elif name == "evrard_disph":       # disph + gravity sphere, Wendland, K=128, TD-AV, AC
        p = defaults(sph_type=DISPH, kernel=WENDLAND, neighbor_number=128, use_time_dependent_av=1,
                     alpha_min=0.1, alpha_max=2.0, epsilon_av=0.2, use_balsara_switch=1, use_ac=1,
                     alpha_ac=1.0, use_gravity=1, g_constant=1.0, theta=0.5, gamma=5.0 / 3.0)
    else:
        raise KeyError(name)
    for k, v in overrides.items():
        _set(p, k, v)
    return p
