"""Python mirror of the reference's per-step interface, over the C-ABI.

``DEMSystem`` exposes the same operations, with the same argument meaning, as
the Fortran module routines the library replaces:

=================================  ==========================================
DEMSystem method                   reference routine
=================================  ==========================================
``__init__``                        InitializeAuxiliaries (src/MDEM.f90:110)
``set_state``                       Particle(1:NP) + InitializeIntegration-
                                    Variables / InitializeContacts
``initialize_cell_distribution``    InitializeCellDistribution
                                    (src/MForces.f90:110)
``compute_accelerations``           ComputeAccelerations (src/MForces.f90:145)
``compute_forces``                  the same, with its Force/Torque arrays
``move_particles``                  MoveParticles (src/MDEM.f90:285)
``move_particles_euler``            MoveParticlesEuler (src/MDEM.f90:258)
``run``                             main loop, src/DEM.f90:85-99
``set_wall_motion``                 WallsInMovement + WM(:) (MoveWalls,
                                    src/MDEM.f90:392, is called by the steps)
``walls``                           Wall(1:NW)%Position, %Velocity
``kinetic_energy`` etc.             KineticEnergy/PotentialEnergy
                                    (src/MDEM.f90:183-213)
=================================  ==========================================

Errors are raised as :class:`DEMError` (the reference ``stop``s).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import (MAX_WALLS, DemFluid, DemObservables, DemParams, DemPouring, DemRng,
                   DemWall, DemWallMotion)


class DEMError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"DEM error {code}: {message}")
        self.code = code


def _dptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int32))


def _vec(a, n):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(n, 3)
    return a


class DEMSystem:
    """One simulation context.

    ``lib``/``prefix`` select the implementation behind the same ABI: the
    CUDA library (default) or, in tests, the CPU oracle with prefix ``orc_``.
    """

    def __init__(self, params: DemParams, lib=None, prefix: str = "dem_"):
        self.lib = lib if lib is not None else _abi.load_library()
        self.prefix = prefix
        self.params = params
        self.nprev = int(params.method_order) - 1
        self._ctx = C.c_void_p()
        st = self._fn("create")(C.byref(params), C.byref(self._ctx))
        if st != 0:
            raise DEMError(st, "create failed" + (": no CUDA device" if st == -7 else ""))
        self.n = 0

    @classmethod
    def ensemble(cls, params_list, counts, lib=None):
        """Independent systems in one context (dem_create_ensemble): every
        stage of a step is one launch over all systems.  ``counts`` are the
        particles per system; particle arrays are concatenated by system."""
        self = cls.__new__(cls)
        self.lib = lib if lib is not None else _abi.load_library()
        self.prefix = "dem_"
        self.params = params_list[0]
        self.nprev = int(self.params.method_order) - 1
        self._ctx = C.c_void_p()
        arr = (DemParams * len(params_list))(*params_list)
        st = self.lib.dem_create_ensemble(arr, len(params_list), C.byref(self._ctx))
        if st != 0:
            raise DEMError(st, "create_ensemble failed")
        self.n = 0
        cnt = np.ascontiguousarray(counts, dtype=np.int32)
        self._call("set_system_counts", _iptr(cnt))
        return self

    # -- plumbing ---------------------------------------------------------
    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def _call(self, name, *args):
        st = self._fn(name)(self._ctx, *args)
        if st != 0:
            msg = self._fn("last_error")(self._ctx)
            raise DEMError(st, f"{self.prefix}{name}: " + (msg.decode() if msg else ""))
        return st

    def close(self):
        if self._ctx:
            self._fn("destroy")(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state ------------------------------------------------------------
    def set_state(self, pos, vel, omega, comp=None, radius=None, acc=None, alpha=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        n = pos.shape[0]
        self._keep = (
            pos.reshape(n, 3), _vec(vel, n), _vec(omega, n),
            None if comp is None else np.ascontiguousarray(comp, dtype=np.int32),
            None if radius is None else np.ascontiguousarray(radius, dtype=np.float64),
            _vec(acc, n), _vec(alpha, n))
        p, v, w, c, r, a, al = self._keep
        self._call("set_state", n, _iptr(c), _dptr(r), _dptr(p), _dptr(v), _dptr(w), _dptr(a),
                   _dptr(al))
        self.n = n
        # Particle%Index - 1, kept for state files (it does not change in a run)
        self.comp = np.zeros(n, np.int32) if c is None else c.copy()
        self._keep = None

    def update_state(self, pos=None, vel=None, omega=None, acc=None, alpha=None):
        """Overwrite Particle(1:n) keeping ring, contacts and cell lists."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(self.n, 3)
                for a in (pos, vel, omega, acc, alpha)]
        self._call("update_state", *(_dptr(a) for a in arrs))

    def _get(self, name):
        n = self.n
        out = {k: np.empty((n, 3)) for k in ("pos", "vel", "omega", "acc", "alpha")}
        self._call(name, *(_dptr(out[k]) for k in ("pos", "vel", "omega", "acc", "alpha")))
        return out

    def get_state(self):
        return self._get("get_state")

    def get_predicted(self):
        return self._get("get_predicted")

    def get_integration(self):
        prev = np.empty((max(self.nprev, 0), self.n, 9))
        ipc = np.zeros(max(self.nprev, 1), dtype=np.int32)
        self._call("get_integration", _dptr(prev), _iptr(ipc))
        return prev, ipc[: self.nprev]

    def logical_ring(self):
        """Previous(ipc(k)) for k = 1..NPrev, shape (NPrev, n, 9)."""
        prev, ipc = self.get_integration()
        return np.stack([prev[i - 1] for i in ipc]) if self.nprev > 0 else prev

    def set_integration(self, prev, ipc):
        prev = np.ascontiguousarray(prev, dtype=np.float64)
        ipc = np.ascontiguousarray(ipc, dtype=np.int32)
        self._call("set_integration", _dptr(prev), _iptr(ipc))

    def set_contacts(self, imin=(), imax=(), ft=None, vt=None, ip=(), iw=(), ftw=None,
                     vtw=None):
        imin = np.ascontiguousarray(imin, dtype=np.int32)
        imax = np.ascontiguousarray(imax, dtype=np.int32)
        m = imin.size
        ft = np.ascontiguousarray(np.zeros((m, 3)) if ft is None else ft, dtype=np.float64)
        vt = np.ascontiguousarray(np.zeros((m, 3)) if vt is None else vt, dtype=np.float64)
        ip = np.ascontiguousarray(ip, dtype=np.int32)
        iw = np.ascontiguousarray(iw, dtype=np.int32)
        mw = ip.size
        ftw = np.ascontiguousarray(np.zeros((mw, 3)) if ftw is None else ftw, dtype=np.float64)
        vtw = np.ascontiguousarray(np.zeros((mw, 3)) if vtw is None else vtw, dtype=np.float64)
        self._call("set_contacts", m, _iptr(imin), _iptr(imax), _dptr(ft), _dptr(vt), mw,
                   _iptr(ip), _iptr(iw), _dptr(ftw), _dptr(vtw))

    def count_contacts(self):
        a = C.c_int64()
        b = C.c_int64()
        self._call("count_contacts", C.byref(a), C.byref(b))
        return a.value, b.value

    def get_contacts(self):
        m, mw = self.count_contacts()
        out = dict(imin=np.empty(m, np.int32), imax=np.empty(m, np.int32), ft=np.empty((m, 3)),
                   vt=np.empty((m, 3)), ip=np.empty(mw, np.int32), iw=np.empty(mw, np.int32),
                   ftw=np.empty((mw, 3)), vtw=np.empty((mw, 3)))
        self._call("get_contacts", m, _iptr(out["imin"]), _iptr(out["imax"]), _dptr(out["ft"]),
                   _dptr(out["vt"]), mw, _iptr(out["ip"]), _iptr(out["iw"]), _dptr(out["ftw"]),
                   _dptr(out["vtw"]))
        return out

    # -- cells ------------------------------------------------------------
    def initialize_cell_distribution(self):
        self._call("initialize_cell_distribution")

    def grid(self):
        g = np.zeros(3, dtype=np.int32)
        self._call("get_grid", _iptr(g))
        return tuple(int(x) for x in g)

    def get_cells(self):
        nc = C.c_int32()
        self._call("get_cell_count", C.byref(nc))  # every system's cells
        ci = np.empty(self.n, np.int32)
        tr = np.empty(self.n, np.int32)
        cs = np.empty(nc.value + 1, np.int32)
        self._call("get_cells", _iptr(ci), _iptr(tr), _iptr(cs))
        return ci, tr, cs

    def set_cells(self, traversal, cell_start):
        """ReadCellDistribution: the cell lists as saved (list order per cell)."""
        tr = np.ascontiguousarray(traversal, dtype=np.int32)
        cs = np.ascontiguousarray(cell_start, dtype=np.int32)
        self._call("set_cells", _iptr(tr), _iptr(cs))

    # -- dynamics ---------------------------------------------------------
    def compute_accelerations(self, use_predicted=False, time_step=None, update=True):
        ts = float(self.params.time_step if time_step is None else time_step)
        self._call("compute_accelerations", 1 if use_predicted else 0, ts, 1 if update else 0)

    def compute_forces(self, use_predicted=False, time_step=None, update=True):
        """ComputeAccelerations, returning also its Force and Torque sums
        (src/MForces.f90:319-320, before the division by mass and inertia)
        as two (n, 3) arrays."""
        ts = float(self.params.time_step if time_step is None else time_step)
        f = np.zeros((self.n, 3))
        t = np.zeros((self.n, 3))
        self._call("compute_forces", 1 if use_predicted else 0, ts, 1 if update else 0,
                   _dptr(f), _dptr(t))
        return f, t

    def move_particles(self, step):
        self._call("move_particles", int(step))

    def move_particles_euler(self):
        self._call("move_particles_euler")

    def run(self, first_step, last_step):
        self._call("run", int(first_step), int(last_step))
        self._refresh_n()  # UpdateParticleList may have removed particles

    def run_timed(self, first_step, last_step):
        """dem_run with device-side CUDA-event timing; returns milliseconds."""
        ms = C.c_double()
        self._call("run_timed", int(first_step), int(last_step), C.byref(ms))
        self._refresh_n()
        return ms.value

    # -- diagnostics ------------------------------------------------------
    def ncol(self):
        v = C.c_int64()
        self._call("get_ncol", C.byref(v))
        return v.value

    # -- particle removal ---------------------------------------------------
    def _refresh_n(self):
        v = C.c_int32()
        self._call("get_n", C.byref(v))
        if v.value != self.n:
            self.n = v.value
            comp = np.zeros(self.n, np.int32)
            if self.n:
                self._call("get_components", _iptr(comp))
            self.comp = comp

    def update_particle_list(self) -> int:
        """UpdateParticleList: remove the particles outside the box."""
        v = C.c_int64()
        self._call("update_particle_list", C.byref(v))
        self._refresh_n()
        return v.value

    def set_particle_removal(self, on: bool) -> None:
        """Whether ``run`` removes escaped particles after every step."""
        self._call("set_particle_removal", 1 if on else 0)

    def removal_stats(self):
        s = (C.c_int64 * 3)()
        self._call("get_removal_stats", s)
        return {"removed": s[0], "swaps": s[1], "records_moved": s[2]}

    # -- fluid drag ----------------------------------------------------------
    def set_fluid(self, fluid: DemFluid | None) -> None:
        """FluidFlow with its settings (mFluid), or None for no fluid."""
        self._call("set_fluid", None if fluid is None else C.byref(fluid))

    # -- pouring -------------------------------------------------------------
    def set_pouring(self, pouring: DemPouring | None) -> None:
        """Pouring for ``run`` (PouringAttempt before every step), or None."""
        self._call("set_pouring", None if pouring is None else C.byref(pouring))

    def pour_particle(self) -> bool:
        """PourParticle once; True if a sphere went in."""
        v = C.c_int32()
        self._call("pour_particle", C.byref(v))
        self._refresh_n()
        return bool(v.value)

    def rng(self) -> dict:
        r = DemRng()
        self._call("get_rng", C.byref(r))
        return {"aam": r.aam, "dummy": r.dummy, "iix": r.iix, "iiy": r.iiy, "iik": r.iik}

    def set_rng(self, aam=0.0, dummy=0, iix=-1, iiy=-1, iik=0) -> None:
        r = DemRng(aam, dummy, iix, iiy, iik)
        self._call("set_rng", C.byref(r))

    def set_ncol(self, ncol: int) -> None:
        self._call("set_ncol", int(ncol))

    def escaped(self):
        v = C.c_int64()
        self._call("get_escaped", C.byref(v))
        return v.value

    # -- moving walls -----------------------------------------------------
    def set_wall_motion(self, motions):
        """WallsInMovement with WM(1:NW) = ``motions`` (dicts with the fields
        of :class:`DemWallMotion`), or ``None`` to stop the walls."""
        if motions is None:
            self._call("set_wall_motion", None)
            return
        arr = (DemWallMotion * max(len(motions), 1))()
        for j, m in enumerate(motions):
            for key, val in m.items():
                getattr(arr[j], key)[:] = [float(x) for x in val]
        self._call("set_wall_motion", arr)

    def walls(self):
        """Position and velocity of every wall, as the last step left them."""
        out = (DemWall * MAX_WALLS)()
        self._call("get_walls", out)
        nw = self.params.n_walls
        return {"position": np.array([list(out[j].position) for j in range(nw)]),
                "velocity": np.array([list(out[j].velocity) for j in range(nw)])}

    def observables(self):
        o = DemObservables()
        self._call("get_observables", C.byref(o))
        return {
            "kinetic_energy": o.kinetic_energy,
            "potential_energy": o.potential_energy,
            "mean_coordination": o.mean_coordination,
            "packing_fraction": o.packing_fraction,
            "wall_normal_force": list(o.wall_normal_force),
            "momentum": list(o.momentum),
            "n_pair_contacts": o.n_pair_contacts,
            "n_wall_contacts": o.n_wall_contacts,
            "wall_pressure": list(o.wall_pressure),
            "bed_height": o.bed_height,
            "n_pair_records": o.n_pair_records,
        }

    # -- GPU-only instrumentation -------------------------------------------
    def set_profiling(self, on: bool):
        self._call("set_profiling", 1 if on else 0)

    def kernel_stats(self):
        out = {}
        i = 0
        name = C.create_string_buffer(64)
        while True:
            la = C.c_int64()
            ms = C.c_double()
            st = self._fn("get_kernel_stats")(self._ctx, i, name, 64, C.byref(la), C.byref(ms))
            if st != 0:
                break
            out[name.value.decode()] = (la.value, ms.value)
            i += 1
        return out

    def reset_kernel_stats(self):
        self._call("reset_kernel_stats")

    def timer_start(self):
        self._call("timer_start")

    def timer_stop(self):
        ms = C.c_double()
        self._call("timer_stop", C.byref(ms))
        return ms.value

    def launch_count(self):
        v = C.c_int64()
        self._call("get_launch_count", C.byref(v))
        return v.value

    def stream_ptr(self):
        p = C.c_void_p()
        self._call("get_stream", C.byref(p))
        return p.value

    def pass_stats(self):
        a, b, m = C.c_int64(), C.c_int64(), C.c_int64()
        cap = C.c_int32()
        self._call("get_pass_stats", C.byref(a), C.byref(b), C.byref(m), C.byref(cap))
        return {"pair_contacts": a.value, "wall_contacts": b.value, "movers": m.value,
                "hist_capacity": cap.value}

    def set_tuning(self, skin_factor: float, pass_variant: int) -> None:
        self._call("set_tuning", C.c_double(skin_factor), C.c_int32(pass_variant))

    def tuning(self):
        f, v = C.c_double(), C.c_int32()
        self._call("get_tuning", C.byref(f), C.byref(v))
        return {"skin_factor": f.value, "pass_variant": v.value}

    def set_launch_shape(self, launch_mode: int = 0, test_block: int = 128,
                         particles_per_thread: int = 1, pair_waves: int = 2) -> None:
        """dem_set_launch_shape: launch_mode 1 runs each 4-step chunk as one
        persistent cooperative launch; the other knobs shape the test, fold
        and pair kernels' grids.  No result depends on them."""
        self._call("set_launch_shape", C.c_int32(launch_mode), C.c_int32(test_block),
                   C.c_int32(particles_per_thread), C.c_int32(pair_waves))

    def launch_shape(self):
        v = [C.c_int32() for _ in range(4)]
        self._call("get_launch_shape", *[C.byref(x) for x in v])
        return dict(zip(("launch_mode", "test_block", "particles_per_thread", "pair_waves"),
                        (x.value for x in v)))

    def set_early_launch(self, on: bool = True) -> None:
        """dem_set_early_launch: the test, pair and fold kernels of a pass
        launched with programmatic stream serialization (default on).  No
        result depends on it."""
        self._call("set_early_launch", C.c_int32(1 if on else 0))

    def early_launch(self) -> bool:
        v = C.c_int32()
        self._call("get_early_launch", C.byref(v))
        return bool(v.value)

    def set_persistent_barrier(self, timeout_ms: float = 2000.0, extra_blocks: int = 0) -> None:
        self._call("set_persistent_barrier", C.c_double(timeout_ms), C.c_int32(extra_blocks))

    def persistent_blocks(self) -> int:
        v = C.c_int32()
        self._call("get_persistent_blocks", C.byref(v))
        return v.value

    def set_reorder(self, every_steps: int) -> None:
        """dem_set_reorder: dem_run keeps the particle storage in cell order,
        permuting it every `every_steps` steps (0: never).  No result
        changes; every call that reads particle data sees the reference's
        order."""
        self._call("set_reorder", C.c_int32(every_steps))

    def reorder(self):
        e, k = C.c_int32(), C.c_int64()
        self._call("get_reorder", C.byref(e), C.byref(k))
        return {"every_steps": e.value, "reorders": k.value}

    # ---- one slab of a spatial decomposition (dem_slab_*; dem3d_b200.slab)
    def slab_set_range(self, z0: int, z1: int) -> None:
        self._call("slab_set_range", C.c_int32(z0), C.c_int32(z1))

    def slab_phase(self, step: int, pass_: int, phase: int) -> None:
        self._call("slab_phase", C.c_int32(step), C.c_int32(pass_), C.c_int32(phase))

    def slab_pack(self, what: int, buf_ptr: int, cap: int) -> int:
        """Packs exchange `what` into the device buffer at buf_ptr (cap
        bytes); returns its size."""
        n = C.c_int64()
        self._call("slab_pack", C.c_int32(what), C.c_void_p(buf_ptr), C.c_int64(cap),
                   C.byref(n))
        return n.value

    def slab_unpack(self, what: int, buf_ptr: int, nbytes: int) -> None:
        self._call("slab_unpack", C.c_int32(what), C.c_void_p(buf_ptr), C.c_int64(nbytes))

    def slab_displacement(self, set_bits=None) -> int:
        """The last pass's largest displacement (FP32 bits) as read; with
        set_bits, the context's value is then replaced by set_bits (the
        maximum over all slabs)."""
        out = C.c_uint32()
        if set_bits is None:
            self._call("slab_displacement", C.byref(out), None)
        else:
            v = C.c_uint32(set_bits)
            self._call("slab_displacement", C.byref(out), C.byref(v))
        return out.value

    def slab_owned(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.int32)
        self._call("slab_owned", _iptr(out))
        return out.astype(bool)

    AUTOTUNE_TRIALS = 16

    def autotune(self, first_step: int, steps_per_trial: int = 20):
        """Runs the timed trials of dem_autotune on the live system; returns
        the last step advanced, the chosen settings and the trial times
        (skin x pair variant, then particles per thread, test block, pair
        waves and the persistent launch)."""
        last = C.c_int32()
        ms = (C.c_double * self.AUTOTUNE_TRIALS)()
        self._call("autotune", C.c_int32(first_step), C.c_int32(steps_per_trial),
                   C.byref(last), ms)
        return {"last_step": last.value, **self.tuning(), **self.launch_shape(),
                "trial_ms": list(ms)}

    def row_stats(self):
        """Candidate-row entries of the last pass and the row capacity."""
        t, kc = C.c_int64(), C.c_int32()
        self._call("get_row_stats", C.byref(t), C.byref(kc))
        return {"candidates": t.value, "row_capacity": kc.value}
