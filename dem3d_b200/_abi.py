"""ctypes mirror of ``include/dem3d_b200.h`` and the loader of the CUDA library.

The library is the product: there is no CPU fallback.  ``load_library`` raises
if ``libdem3d_b200.so`` is missing or cannot be loaded.
"""
from __future__ import annotations

import ctypes as C
import os

MAX_COMPONENTS = 16
MAX_WALLS = 8

DEM_OK = 0
DEM_ERR_INVALID = -1
DEM_ERR_CUDA = -2
DEM_ERR_CAPACITY = -3
DEM_ERR_UNSUPPORTED = -5
DEM_ERR_STATE = -6
DEM_ERR_NO_DEVICE = -7

WALL_RECTANGLE = 1
WALL_CONE = 2

PREC_FP64 = 0
PREC_MIXED = 1

_d3 = C.c_double * 3


class DemWall(C.Structure):
    """TWall (src/MDimension3D.f90:45-59)."""

    _fields_ = [
        ("shape", C.c_int32), ("order", C.c_int32),
        ("l1", C.c_double), ("l2", C.c_double), ("l3", C.c_double),
        ("u", _d3), ("w", _d3), ("n", _d3),
        ("position", _d3), ("velocity", _d3), ("omega", _d3),
    ]


_NCC = MAX_COMPONENTS * MAX_COMPONENTS
_NCW = MAX_COMPONENTS * MAX_WALLS


class DemParams(C.Structure):
    _fields_ = [
        ("n_components", C.c_int32), ("n_walls", C.c_int32), ("pbc", C.c_int32 * 3),
        ("method_order", C.c_int32), ("euler_intervals", C.c_int32), ("max_ncell", C.c_int32),
        ("precision", C.c_int32), ("hist_capacity", C.c_int32),
        ("lbox", _d3), ("gravity", _d3), ("time_step", C.c_double),
        ("comp_radius", C.c_double * MAX_COMPONENTS),
        ("comp_inv_mass", C.c_double * MAX_COMPONENTS),
        ("comp_inv_inertia", C.c_double * MAX_COMPONENTS),
        ("comp_eff_mass", C.c_double * MAX_COMPONENTS),
        ("min_dij", C.c_double * _NCC), ("min_dij_sq", C.c_double * _NCC),
        ("kn", C.c_double * _NCC), ("yn", C.c_double * _NCC), ("kt", C.c_double * _NCC),
        ("yt", C.c_double * _NCC), ("mu_sq", C.c_double * _NCC),
        ("knw", C.c_double * _NCW), ("ynw", C.c_double * _NCW), ("ktw", C.c_double * _NCW),
        ("ytw", C.c_double * _NCW), ("muw_sq", C.c_double * _NCW),
        ("pp_mass_coef", C.c_double), ("pp_density", C.c_double),
        ("pp_fluid_density", C.c_double), ("pp_rmax", C.c_double),
        ("pp_kn", C.c_double), ("pp_kt", C.c_double), ("pp_gamma_n", C.c_double),
        ("pp_gamma_t", C.c_double), ("pp_mu_sq", C.c_double),
        ("pp_knw", C.c_double * MAX_WALLS), ("pp_ktw", C.c_double * MAX_WALLS),
        ("pp_gamma_nw", C.c_double * MAX_WALLS), ("pp_gamma_tw", C.c_double * MAX_WALLS),
        ("pp_muw_sq", C.c_double * MAX_WALLS),
        ("walls", DemWall * MAX_WALLS),
    ]


class DemWallMotion(C.Structure):
    """TWallMovement (src/MDEM.f90:39-45): harmonic motion of one wall."""

    _fields_ = [
        ("constant_factor", _d3), ("amplitude", _d3), ("velocity_amplitude", _d3),
        ("two_pi_frequency", _d3), ("phase_angle", _d3),
    ]


# spatial decomposition: phases of a force pass and exchanges (dem3d_b200.h)
SLAB_RELINK, SLAB_TEST_PAIR, SLAB_FOLD, SLAB_FINISH = 0, 1, 2, 3
SLAB_GHOSTS, SLAB_LOWER, SLAB_JHALVES, SLAB_MIGRATE_UP, SLAB_MIGRATE_DOWN = 0, 1, 2, 3, 4

POUR_RECTANGLE = 1
POUR_CIRCLE = 2


class DemPouring(C.Structure):
    """Pouring settings (src/DEM.f90:745-800, src/MDEM.f90:412-532)."""

    _fields_ = [
        ("interval", C.c_int32), ("shape", C.c_int32), ("max_attempts", C.c_int32),
        ("target_number", C.c_int32 * MAX_COMPONENTS), ("size", C.c_double * 2),
        ("velocity_z", C.c_double),
    ]


class DemRng(C.Structure):
    """ranf's state (src/MUtil.f90:10-11)."""

    _fields_ = [("aam", C.c_double), ("dummy", C.c_int32), ("iix", C.c_int32),
                ("iiy", C.c_int32), ("iik", C.c_int32)]


class DemFluid(C.Structure):
    """Fluid settings (ReadFluidSpecifications, src/mFluid.f90:27-52)."""

    _fields_ = [("viscosity", C.c_double), ("flow_rate", C.c_double), ("density", C.c_double),
                ("comp_density", C.c_double * MAX_COMPONENTS), ("levels", C.c_int32),
                ("pad_", C.c_int32)]


class DemObservables(C.Structure):
    _fields_ = [
        ("kinetic_energy", C.c_double), ("potential_energy", C.c_double),
        ("mean_coordination", C.c_double), ("packing_fraction", C.c_double),
        ("wall_normal_force", C.c_double * MAX_WALLS), ("momentum", _d3),
        ("n_pair_contacts", C.c_int64), ("n_wall_contacts", C.c_int64),
        ("wall_pressure", C.c_double * MAX_WALLS), ("bed_height", C.c_double),
        ("n_pair_records", C.c_int64),
    ]


_P = C.c_void_p
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)
_DP = C.POINTER(C.c_double)

# name -> (restype, argtypes); the same table describes the oracle (prefix orc_)
SIGNATURES = {
    "create": (C.c_int, [C.POINTER(DemParams), C.POINTER(_P)]),
    "destroy": (None, [_P]),
    "last_error": (C.c_char_p, [_P]),
    "set_state": (C.c_int, [_P, C.c_int32, _I32P, _DP, _DP, _DP, _DP, _DP, _DP]),
    "get_state": (C.c_int, [_P, _DP, _DP, _DP, _DP, _DP]),
    "get_predicted": (C.c_int, [_P, _DP, _DP, _DP, _DP, _DP]),
    "update_state": (C.c_int, [_P, _DP, _DP, _DP, _DP, _DP]),
    "get_n": (C.c_int, [_P, _I32P]),
    "set_integration": (C.c_int, [_P, _DP, _I32P]),
    "get_integration": (C.c_int, [_P, _DP, _I32P]),
    "set_contacts": (C.c_int, [_P, C.c_int64, _I32P, _I32P, _DP, _DP, C.c_int64, _I32P, _I32P,
                               _DP, _DP]),
    "count_contacts": (C.c_int, [_P, _I64P, _I64P]),
    "get_contacts": (C.c_int, [_P, C.c_int64, _I32P, _I32P, _DP, _DP, C.c_int64, _I32P, _I32P,
                               _DP, _DP]),
    "initialize_cell_distribution": (C.c_int, [_P]),
    "get_grid": (C.c_int, [_P, _I32P]),
    "get_cell_count": (C.c_int, [_P, _I32P]),
    "get_cells": (C.c_int, [_P, _I32P, _I32P, _I32P]),
    "set_cells": (C.c_int, [_P, _I32P, _I32P]),
    "compute_accelerations": (C.c_int, [_P, C.c_int32, C.c_double, C.c_int32]),
    "compute_forces": (C.c_int, [_P, C.c_int32, C.c_double, C.c_int32, _DP, _DP]),
    "move_particles": (C.c_int, [_P, C.c_int32]),
    "move_particles_euler": (C.c_int, [_P]),
    "run": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "get_ncol": (C.c_int, [_P, _I64P]),
    "set_ncol": (C.c_int, [_P, C.c_int64]),
    "update_particle_list": (C.c_int, [_P, _I64P]),
    "set_particle_removal": (C.c_int, [_P, C.c_int32]),
    "get_components": (C.c_int, [_P, _I32P]),
    "get_removal_stats": (C.c_int, [_P, _I64P]),
    "set_pouring": (C.c_int, [_P, C.POINTER(DemPouring)]),
    "set_fluid": (C.c_int, [_P, C.POINTER(DemFluid)]),
    "pour_particle": (C.c_int, [_P, _I32P]),
    "set_rng": (C.c_int, [_P, C.POINTER(DemRng)]),
    "get_rng": (C.c_int, [_P, C.POINTER(DemRng)]),
    "get_escaped": (C.c_int, [_P, _I64P]),
    "get_observables": (C.c_int, [_P, C.POINTER(DemObservables)]),
    "set_wall_motion": (C.c_int, [_P, C.POINTER(DemWallMotion)]),
    "get_walls": (C.c_int, [_P, C.POINTER(DemWall)]),
}

# entry points only the CUDA library has
GPU_ONLY = {
    "version": (C.c_char_p, []),
    "select_device": (C.c_int, [C.c_int32]),
    "run_timed": (C.c_int, [_P, C.c_int32, C.c_int32, _DP]),
    "set_profiling": (C.c_int, [_P, C.c_int32]),
    "get_kernel_stats": (C.c_int, [_P, C.c_int32, C.c_char_p, C.c_int32, _I64P, _DP]),
    "reset_kernel_stats": (C.c_int, [_P]),
    "get_launch_count": (C.c_int, [_P, _I64P]),
    "timer_start": (C.c_int, [_P]),
    "timer_stop": (C.c_int, [_P, _DP]),
    "get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "get_pass_stats": (C.c_int, [_P, _I64P, _I64P, _I64P, _I32P]),
    "get_row_stats": (C.c_int, [_P, _I64P, _I32P]),
    "create_ensemble": (C.c_int, [C.POINTER(DemParams), C.c_int32, C.POINTER(_P)]),
    "set_system_counts": (C.c_int, [_P, _I32P]),
    "set_tuning": (C.c_int, [_P, C.c_double, C.c_int32]),
    "get_tuning": (C.c_int, [_P, _DP, _I32P]),
    "autotune": (C.c_int, [_P, C.c_int32, C.c_int32, _I32P, _DP]),
    "set_launch_shape": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "get_launch_shape": (C.c_int, [_P, _I32P, _I32P, _I32P, _I32P]),
    "set_early_launch": (C.c_int, [_P, C.c_int32]),
    "get_early_launch": (C.c_int, [_P, _I32P]),
    "set_persistent_barrier": (C.c_int, [_P, C.c_double, C.c_int32]),
    "get_persistent_blocks": (C.c_int, [_P, _I32P]),
    "set_reorder": (C.c_int, [_P, C.c_int32]),
    "get_reorder": (C.c_int, [_P, _I32P, _I64P]),
    "slab_set_range": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "slab_phase": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32]),
    "slab_pack": (C.c_int, [_P, C.c_int32, _P, C.c_int64, _I64P]),
    "slab_unpack": (C.c_int, [_P, C.c_int32, _P, C.c_int64]),
    "slab_displacement": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "slab_owned": (C.c_int, [_P, _I32P]),
    # device pointers for positions and outputs; see the header
    "distribute_particles_noalloc": (C.c_int, [C.POINTER(DemParams), C.c_int32, _P, _P, _P, _P,
                                               _I32P, _P, C.c_char_p, C.c_int32]),
}

NOALLOC_MAX_PARTICLES = 262144
NOALLOC_MAX_CELLS = 262144

HERE = os.path.dirname(os.path.abspath(__file__))
# DEM3D_B200_LIB selects another build of the same library (e.g. one compiled
# with different launch bounds); the default is the in-tree build.
LIB_PATH = os.environ.get("DEM3D_B200_LIB") or os.path.join(HERE, "libdem3d_b200.so")


def bind(lib: C.CDLL, prefix: str, table: dict) -> None:
    for name, (res, args) in table.items():
        f = getattr(lib, prefix + name)
        f.restype = res
        f.argtypes = args


def all_symbols() -> list[str]:
    return ["dem_" + k for k in list(SIGNATURES) + list(GPU_ONLY)]


_LIB = None


def load_library(path: str | None = None) -> C.CDLL:
    """Load the CUDA library; raises (never falls back to CPU code)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build it with `python -m dem3d_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(p)
    bind(lib, "dem_", SIGNATURES)
    bind(lib, "dem_", GPU_ONLY)
    if path is None:
        _LIB = lib
    return lib
