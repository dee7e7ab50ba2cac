"""ctypes binding of the B200 carrier engine's C ABI (include/mcb200.h).

This module is a thin host-side mirror for Python callers (the test suite,
bench.py).  All computation happens in libmcb200.so on the GPU; importing
this module fails loudly if the library has not been built, and every call
raises EngineError when the library reports an error.  There is no CPU
fallback.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# MCB200_LIBRARY selects another build of the engine library (a tuning variant).
LIB_PATH = os.environ.get("MCB200_LIBRARY", os.path.join(PKG_DIR, "libmcb200.so"))
DEFAULT_TABLE_DIR = os.path.join(PKG_DIR, "tables")

OK = 0
COUNTER_NAMES = [
    "phonon", "impurity", "caught", "generated", "events", "unfinished", "too_many_events",
    "child_overflow", "no_tet", "zero_time",
]
NUM_COUNTERS = 16
FLAG_SURFACE_SCATTER = 1
FLAG_SURFACE_IMPURITY = 2
FLAG_HEAT = 4
FLAG_QUANTUM = 8
IDS_CONTACT, IDS_SECTIONS, IDS_INDUCED = 0, 1, 2  # serving's Ids estimators (MCB200_IDS_*)
WARM_OFF, WARM_CONVERGED, WARM_SETTLED = 0, 1, 2  # serving's warm-start donors (MCB200_WARM_*)
FLIGHT_FP64 = 0
FLIGHT_FP32 = 1
# Poisson preconditioners (mcb200_set_poisson_solver)
POISSON_AUTO = 0
POISSON_JACOBI = 1
POISSON_MULTIGRID = 2
UNIT_NAMES = ["T0", "eV0", "spr0", "time0", "conc0", "field0", "scrt0", "pot0", "a0pi", "sieg",
              "eps_silicon", "eps_oxide", "curr0", "dens0"]


class EngineError(RuntimeError):
    pass


class _Particles(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in
                ("x", "y", "z", "kx", "ky", "kz", "charge", "energy", "i", "j", "k", "itet", "isym", "type", "uid")]


class SurfaceParams(ctypes.Structure):
    """mcb200_surface_params; defaults are the reference's SurfSc_* values
    (src/mcmodel.cpp:4107-4121) with lengths in metres (converted by
    Engine.surface_rates)."""
    _fields_ = [(n, ctypes.c_double) for n in ("delta", "ail", "xiph", "theta", "gama", "nbmod", "npf", "pft",
                                               "pfn", "kpha")] + [("roughness", ctypes.c_int),
                                                                  ("phonon", ctypes.c_int)]


SURFACE_DEFAULTS = dict(delta_m=0.1126755e-9, ail_m=2.0e-9, xiph=12.0, theta=2.857703, gama=1.5, nbmod=2.0,
                        npf=-0.6, pft=0.7, pfn=0.3, kpha=3600e-4, roughness=1, phonon=1)

PARTICLE_FIELDS = {
    "x": np.float64, "y": np.float64, "z": np.float64, "kx": np.float64, "ky": np.float64, "kz": np.float64,
    "charge": np.float64, "energy": np.float64, "i": np.int32, "j": np.int32, "k": np.int32,
    "itet": np.int32, "isym": np.int32, "type": np.int32, "uid": np.uint32,
}


class DeckInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("nx", "ny", "nz", "total_step", "electron_number", "hole_number",
                                            "stat_step", "stat_heat_step", "heat_steps", "mr_step")] + \
               [("temperature", ctypes.c_double), ("dt_s", ctypes.c_double)] + \
               [(n, ctypes.c_int) for n in ("flag_multiple_refresh", "flag_compute_potential", "flag_compute_heat",
                                            "flag_surface_scatter", "flag_surface_roughness", "flag_surface_phonon",
                                            "flag_surface_impurity", "flag_restart", "n_contacts", "n_planes",
                                            "n_surfaces", "default_electrons", "default_holes")] + \
               [("output_dir", ctypes.c_char * 512), ("prepared", ctypes.c_int), ("dt", ctypes.c_double),
                ("flag_quantum_correction", ctypes.c_int), ("quantum_start_step", ctypes.c_int),
                ("restart_step", ctypes.c_int)]


class QuantumParams(ctypes.Structure):
    _fields_ = [("ratio", ctypes.c_double * 3), ("theta", ctypes.c_double * 3), ("eb", ctypes.c_double)]


class BatchMember(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("seed", ctypes.c_uint64), ("first_step", ctypes.c_uint32),
                ("self_consistent", ctypes.c_int), ("poisson_every", ctypes.c_int),
                ("poisson_rel_tol", ctypes.c_double), ("surface_rates", ctypes.c_int)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("flight_blocks_per_sm", ctypes.c_int), ("grid_per_sm", ctypes.c_int), ("overlap", ctypes.c_int),
                ("ms_per_step", ctypes.c_double), ("candidates", ctypes.c_int), ("pair_solves", ctypes.c_int),
                ("sort_bucket", ctypes.c_int), ("smem_table", ctypes.c_int),
                ("solo_min_particles", ctypes.c_uint64), ("solo_members", ctypes.c_int)]


class ServerOptions(ctypes.Structure):
    _fields_ = [("table_dir", ctypes.c_char_p), ("kelvin", ctypes.c_double), ("device", ctypes.c_int),
                ("flight_precision", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_size_t),
                ("max_slots", ctypes.c_int), ("quantum_steps", ctypes.c_int), ("use_graphs", ctypes.c_int)]


class Request(ctypes.Structure):
    _fields_ = [("input_path", ctypes.c_char_p), ("family", ctypes.c_char_p), ("bias", ctypes.c_double * 2),
                ("target_rel_err", ctypes.c_double), ("min_windows", ctypes.c_int), ("max_steps", ctypes.c_int),
                ("warm_windows_cold", ctypes.c_int), ("warm_windows_warm", ctypes.c_int),
                ("warm_start", ctypes.c_int), ("poisson_every", ctypes.c_int), ("drain_contact", ctypes.c_int),
                ("ids_estimator", ctypes.c_int), ("seed", ctypes.c_uint64), ("arrival_s", ctypes.c_double)]


class Result(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("status", ctypes.c_int), ("ids", ctypes.c_double),
                ("ids_stderr", ctypes.c_double), ("windows", ctypes.c_int), ("steps", ctypes.c_int),
                ("particle_steps", ctypes.c_uint64), ("arrival_s", ctypes.c_double), ("admit_s", ctypes.c_double),
                ("done_s", ctypes.c_double), ("warm_from", ctypes.c_uint64), ("particles", ctypes.c_size_t),
                ("bytes", ctypes.c_size_t)]


class ServerStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_uint64), ("particle_steps", ctypes.c_uint64), ("device_ms", ctypes.c_double),
                ("active", ctypes.c_int), ("pending", ctypes.c_int), ("cached", ctypes.c_int),
                ("bytes_in_use", ctypes.c_size_t)]


SERVE_CONVERGED = 1
SERVE_STEP_LIMIT = 2


class RunOptions(ctypes.Structure):
    _fields_ = [("table_dir", ctypes.c_char_p), ("data_dir", ctypes.c_char_p), ("flight_precision", ctypes.c_int),
                ("poisson_every", ctypes.c_int), ("poisson_rel_tol", ctypes.c_double), ("max_steps", ctypes.c_int),
                ("max_heat_steps", ctypes.c_int), ("write_outputs", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("verbose", ctypes.c_int), ("warmup_steps", ctypes.c_int), ("readback_every_step", ctypes.c_int),
                ("flush_l2_bytes", ctypes.c_size_t), ("profile_phases", ctypes.c_int)]


class RunReport(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("steps_done", "heat_steps_done", "windows", "refreshes")] + \
               [("initial_particles", ctypes.c_size_t), ("final_particles", ctypes.c_size_t),
                ("particle_steps", ctypes.c_uint64), ("wall_s", ctypes.c_double), ("flight_ms", ctypes.c_double),
                ("step_ms", ctypes.c_double), ("poisson_solves", ctypes.c_int),
                ("poisson_iterations", ctypes.c_longlong), ("poisson_max_residual", ctypes.c_double),
                ("last_current", ctypes.c_double * 1), ("heat_total", ctypes.c_double),
                ("phase_s", ctypes.c_double * 8), ("timed_device_ms", ctypes.c_double),
                ("timed_wall_s", ctypes.c_double), ("timed_particle_steps", ctypes.c_uint64),
                ("timed_steps", ctypes.c_int), ("timed_flight_ms", ctypes.c_double),
                ("timed_flight_launches", ctypes.c_uint64), ("timed_launches", ctypes.c_uint64)]


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise EngineError(f"{path} is missing: build it with `make -C c-mc_electron_b200` "
                          "(or __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    c = ctypes
    vp, i32p, dp = c.c_void_p, c.POINTER(c.c_int32), c.POINTER(c.c_double)
    lib.mcb200_create.argtypes = [c.c_char_p, c.c_double, c.c_int, c.c_size_t, c.POINTER(vp)]
    lib.mcb200_create_alike.argtypes = [vp, c.c_size_t, c.POINTER(vp)]
    lib.mcb200_batch_create.argtypes = [c.POINTER(vp), c.POINTER(BatchMember), c.c_int, c.POINTER(vp)]
    lib.mcb200_batch_destroy.argtypes = [vp]
    lib.mcb200_batch_destroy.restype = None
    lib.mcb200_batch_last_error.argtypes = [vp]
    lib.mcb200_batch_last_error.restype = c.c_char_p
    lib.mcb200_batch_step.argtypes = [vp]
    lib.mcb200_batch_sync.argtypes = [vp]
    lib.mcb200_batch_set_grid.argtypes = [vp, c.c_int]
    lib.mcb200_batch_set_overlap.argtypes = [vp, c.c_int]
    lib.mcb200_batch_set_pairing.argtypes = [vp, c.c_int]
    if hasattr(lib, "mcb200_batch_set_smem_table"):
        lib.mcb200_batch_set_smem_table.argtypes = [vp, c.c_int]
    if hasattr(lib, "mcb200_batch_set_solo"):
        lib.mcb200_batch_set_solo.argtypes = [vp, c.c_uint64, c.POINTER(c.c_int)]
    lib.mcb200_batch_mark.argtypes = [vp, c.c_int]
    lib.mcb200_batch_elapsed_ms.argtypes = [vp, c.c_int, c.c_int, dp]
    lib.mcb200_batch_info.argtypes = [vp, c.POINTER(c.c_int), c.POINTER(c.c_uint64), c.POINTER(c.c_uint64),
                                      c.POINTER(c.c_uint64), c.POINTER(c.c_uint64)]
    lib.mcb200_batch_run.argtypes = [vp, c.c_int]
    lib.mcb200_server_create.argtypes = [c.POINTER(ServerOptions), c.POINTER(vp)]
    lib.mcb200_server_destroy.argtypes = [vp]
    lib.mcb200_server_destroy.restype = None
    lib.mcb200_server_last_error.argtypes = [vp]
    lib.mcb200_server_last_error.restype = c.c_char_p
    lib.mcb200_server_now.argtypes = [vp]
    lib.mcb200_server_now.restype = c.c_double
    lib.mcb200_server_submit.argtypes = [vp, c.POINTER(Request), c.POINTER(c.c_uint64)]
    lib.mcb200_server_round.argtypes = [vp, c.POINTER(c.c_int), c.POINTER(c.c_int)]
    lib.mcb200_server_results.argtypes = [vp, c.POINTER(Result), c.c_int, c.POINTER(c.c_int)]
    lib.mcb200_server_stats.argtypes = [vp, c.POINTER(ServerStats)]
    lib.mcb200_copy_ensemble.argtypes = [vp, vp]
    lib.mcb200_batch_autotune.argtypes = [vp, c.c_int, c.POINTER(BatchTuning)]
    lib.mcb200_batch_use_graphs.argtypes = [vp, c.c_int]
    lib.mcb200_destroy.argtypes = [vp]
    lib.mcb200_destroy.restype = None
    lib.mcb200_last_error.argtypes = [vp]
    lib.mcb200_last_error.restype = c.c_char_p
    lib.mcb200_units.argtypes = [vp, dp, c.c_int]
    lib.mcb200_copy_table.argtypes = [vp, c.c_char_p, vp, c.c_size_t, c.POINTER(c.c_size_t)]
    lib.mcb200_set_mesh.argtypes = [vp, c.c_int, c.c_int, c.c_int, dp, dp, dp, dp, dp, dp]
    lib.mcb200_set_device.argtypes = [vp, i32p, dp, dp, c.c_int, dp, dp, c.c_int, i32p]
    lib.mcb200_deposit.argtypes = [vp]
    lib.mcb200_solve_poisson.argtypes = [vp, c.c_double, c.c_int, c.POINTER(c.c_int), dp]
    lib.mcb200_set_poisson_solver.argtypes = [vp, c.c_int, c.c_int]
    lib.mcb200_poisson_stats.argtypes = [vp, c.POINTER(c.c_int64), c.POINTER(c.c_int64), dp, c.c_int]
    lib.mcb200_particle_steps.argtypes = [vp, c.POINTER(c.c_uint64)]
    lib.mcb200_get_poisson_solver.argtypes = [vp, c.POINTER(c.c_int), c.POINTER(c.c_int), c.POINTER(c.c_int)]
    lib.mcb200_get_array.argtypes = [vp, c.c_char_p, dp, c.c_size_t]
    lib.mcb200_surface_rates.argtypes = [vp, c.POINTER(SurfaceParams), i32p]
    lib.mcb200_multiple_refresh.argtypes = [vp, i32p, i32p, c.c_uint32, c.c_uint64, c.POINTER(c.c_int64)]
    lib.mcb200_set_refresh_targets.argtypes = [vp, i32p, i32p]
    lib.mcb200_set_cells.argtypes = [vp, i32p, i32p, i32p, i32p, i32p, c.c_int, dp, c.c_int]
    lib.mcb200_set_fields.argtypes = [vp, dp, dp, dp]
    lib.mcb200_set_surface_rates.argtypes = [vp, dp, dp, dp, dp]
    lib.mcb200_upload_particles.argtypes = [vp, c.c_size_t, c.POINTER(_Particles)]
    lib.mcb200_download_particles.argtypes = [vp, c.POINTER(_Particles), c.c_size_t, c.POINTER(c.c_size_t)]
    lib.mcb200_num_particles.argtypes = [vp]
    lib.mcb200_num_particles.restype = c.c_size_t
    lib.mcb200_step.argtypes = [vp, c.c_uint32, c.c_uint64, c.c_double]
    lib.mcb200_sync.argtypes = [vp]
    lib.mcb200_get_tallies.argtypes = [vp, c.POINTER(c.c_uint64), dp, dp, dp, dp, dp]
    lib.mcb200_reset_tallies.argtypes = [vp]
    lib.mcb200_seed_particles.argtypes = [vp, c.c_size_t, i32p, dp, c.c_int, c.c_uint64]
    lib.mcb200_set_timing.argtypes = [vp, c.c_int]
    lib.mcb200_get_timing.argtypes = [vp, dp, c.c_int]
    lib.mcb200_deck_load.argtypes = [c.c_char_p, c.POINTER(vp)]
    lib.mcb200_deck_free.argtypes = [vp]
    lib.mcb200_deck_error.argtypes = [vp]
    lib.mcb200_deck_error.restype = c.c_char_p
    lib.mcb200_deck_get_info.argtypes = [vp, c.POINTER(DeckInfo)]
    lib.mcb200_deck_int_array.argtypes = [vp, c.c_char_p, i32p, c.c_size_t, c.POINTER(c.c_size_t)]
    lib.mcb200_deck_double_array.argtypes = [vp, c.c_char_p, dp, c.c_size_t, c.POINTER(c.c_size_t)]
    lib.mcb200_deck_prepare.argtypes = [vp, vp]
    lib.mcb200_apply_deck.argtypes = [vp, vp]
    lib.mcb200_seed_deck.argtypes = [vp, vp, c.c_uint64]
    lib.mcb200_run_deck.argtypes = [c.c_char_p, c.c_int, c.POINTER(RunOptions), c.POINTER(RunReport), c.c_char_p,
                                    c.c_size_t]
    lib.mcb200_stat_begin.argtypes = [vp, c.c_int]
    lib.mcb200_mark.argtypes = [vp, c.c_int]
    lib.mcb200_flush_l2.argtypes = [vp, c.c_size_t]
    lib.mcb200_elapsed_ms.argtypes = [vp, c.c_int, c.c_int, dp]
    lib.mcb200_stat_accumulate.argtypes = [vp]
    lib.mcb200_stat_get.argtypes = [vp, c.c_char_p, dp, c.c_size_t]
    if hasattr(lib, "mcb200_tallies_enqueue"):  # absent from libraries built before it (MCB200_LIBRARY)
        lib.mcb200_tallies_enqueue.argtypes = [vp, c.c_int]
        lib.mcb200_tallies_collect.argtypes = [vp, c.c_int, dp]
    if hasattr(lib, "mcb200_set_induced_current"):  # absent from libraries built before it (MCB200_LIBRARY)
        lib.mcb200_set_induced_current.argtypes = [vp, c.c_int]
        lib.mcb200_get_induced_current.argtypes = [vp, dp, dp]
    lib.mcb200_set_potential.argtypes = [vp, dp]
    lib.mcb200_set_potentials.argtypes = [vp, dp, dp]
    lib.mcb200_set_quantum_correction.argtypes = [vp, vp, i32p, i32p, c.c_int]
    lib.mcb200_quantum_potential.argtypes = [vp, dp, dp]
    lib.mcb200_set_heat_tally.argtypes = [vp, c.c_int]
    lib.mcb200_set_flight_precision.argtypes = [vp, c.c_int]
    lib.mcb200_get_flight_precision.argtypes = [vp]
    if hasattr(lib, "mcb200_set_sort_bucket"):
        lib.mcb200_set_sort_bucket.argtypes = [vp, c.c_int]
        lib.mcb200_get_sort_bucket.argtypes = [vp]
    return lib


_LIB = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load_library()
    return _LIB


def _ptr(a: np.ndarray | None, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


@dataclass
class Mesh:
    nx: int
    ny: int
    nz: int
    lx: np.ndarray
    ly: np.ndarray
    lz: np.ndarray

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def nnodes(self) -> int:
        return (self.nx + 1) * (self.ny + 1) * (self.nz + 1)


class Engine:
    """One engine context: full-band tables, mesh, particles, tallies on one GPU."""

    def __init__(self, table_dir: str = DEFAULT_TABLE_DIR, kelvin: float = 300.0, device: int = 0,
                 max_particles: int = 1 << 20, precision: int = FLIGHT_FP64, like: "Engine | None" = None):
        """like: an engine whose device and band tables this one shares
        (mcb200_create_alike; table_dir, kelvin and device are then unused)."""
        self._lib = lib()
        self._ctx = ctypes.c_void_p()
        self._like = like  # the shared tables live while a context uses them; keep the donor's wrapper alive
        if like is not None:
            rc = self._lib.mcb200_create_alike(like._ctx, max_particles, ctypes.byref(self._ctx))
        else:
            rc = self._lib.mcb200_create(table_dir.encode(), kelvin, device, max_particles, ctypes.byref(self._ctx))
        if rc != OK:
            msg = self._lib.mcb200_last_error(self._ctx).decode() if self._ctx else "no context"
            if self._ctx:
                self._lib.mcb200_destroy(self._ctx)
                self._ctx = ctypes.c_void_p()
            raise EngineError(f"mcb200_create failed ({rc}): {msg}")
        self.mesh: Mesh | None = None
        if precision != FLIGHT_FP64:
            self.set_flight_precision(precision)

    def close(self):
        if self._ctx:
            self._lib.mcb200_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != OK:
            raise EngineError(f"{what} failed ({rc}): {self._lib.mcb200_last_error(self._ctx).decode()}")

    def set_flight_precision(self, precision: int):
        """FLIGHT_FP64 (reference arithmetic) or FLIGHT_FP32 (float kinematics,
        56-byte store); only while the store is empty."""
        self._check(self._lib.mcb200_set_flight_precision(self._ctx, precision), "mcb200_set_flight_precision")

    @property
    def precision(self) -> int:
        return self._lib.mcb200_get_flight_precision(self._ctx)

    def set_sort_bucket(self, cells_per_bucket: int):
        """Cells per bucket of the step's counting sort (a power of two,
        1-64); results do not depend on it."""
        self._check(self._lib.mcb200_set_sort_bucket(self._ctx, cells_per_bucket), "mcb200_set_sort_bucket")

    @property
    def sort_bucket(self) -> int:
        return self._lib.mcb200_get_sort_bucket(self._ctx)

    def units(self) -> dict:
        out = np.zeros(len(UNIT_NAMES))
        self._check(self._lib.mcb200_units(self._ctx, _ptr(out, ctypes.c_double), len(out)), "units")
        return dict(zip(UNIT_NAMES, out.tolist()))

    def table(self, name: str, dtype) -> np.ndarray:
        need = ctypes.c_size_t()
        self._check(self._lib.mcb200_copy_table(self._ctx, name.encode(), None, 0, ctypes.byref(need)), name)
        out = np.empty(need.value // np.dtype(dtype).itemsize, dtype=dtype)
        self._check(self._lib.mcb200_copy_table(self._ctx, name.encode(), out.ctypes.data_as(ctypes.c_void_p),
                                                out.nbytes, ctypes.byref(need)), name)
        return out

    def set_mesh(self, lx, ly, lz, dx=None, dy=None, dz=None):
        lx, ly, lz = (np.ascontiguousarray(a, dtype=np.float64) for a in (lx, ly, lz))
        w = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (dx, dy, dz)]
        m = Mesh(len(lx) - 1, len(ly) - 1, len(lz) - 1, lx, ly, lz)
        self._check(self._lib.mcb200_set_mesh(self._ctx, m.nx, m.ny, m.nz, _ptr(lx, ctypes.c_double),
                                              _ptr(ly, ctypes.c_double), _ptr(lz, ctypes.c_double),
                                              *[_ptr(a, ctypes.c_double) for a in w]), "set_mesh")
        self.mesh = m

    def set_device(self, material, donor, acceptor, vapp=(), phims=(), planes=()):
        """Deposition / Poisson description (mcb200_set_device); planes: rows of
        (contact, i0, i1, j0, j1, k0, k1) node ranges."""
        mat = np.ascontiguousarray(material, dtype=np.int32)
        don, acc = (np.ascontiguousarray(a, dtype=np.float64) for a in (donor, acceptor))
        va, ph = (np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (vapp, phims))
        pl = np.ascontiguousarray(planes, dtype=np.int32).reshape(-1)
        self._check(self._lib.mcb200_set_device(self._ctx, _ptr(mat, ctypes.c_int32), _ptr(don, ctypes.c_double),
                                                _ptr(acc, ctypes.c_double), len(va), _ptr(va, ctypes.c_double),
                                                _ptr(ph, ctypes.c_double), len(pl) // 7, _ptr(pl, ctypes.c_int32)),
                    "set_device")

    def surface_rates(self, eeff_direction, **overrides):
        """Per-cell surface rates from the current fields (mcb200_surface_rates)."""
        p = dict(SURFACE_DEFAULTS, **overrides)
        spr0 = self.units()["spr0"]
        sp = SurfaceParams(p["delta_m"] / spr0, p["ail_m"] / spr0, p["xiph"], p["theta"], p["gama"], p["nbmod"],
                           p["npf"], p["pft"], p["pfn"], p["kpha"], int(p["roughness"]), int(p["phonon"]))
        d = np.ascontiguousarray(eeff_direction, dtype=np.int32)
        self._check(self._lib.mcb200_surface_rates(self._ctx, ctypes.byref(sp), _ptr(d, ctypes.c_int32)),
                    "surface_rates")

    def multiple_refresh(self, desired_e, desired_h, step: int, seed: int, wait: bool = True):
        """MultipleRefresh; returns the change in particle count, or None
        without waiting for the GPU (wait=False)."""
        de, dh = (np.ascontiguousarray(a, dtype=np.int32) for a in (desired_e, desired_h))
        gen = ctypes.c_int64()
        self._check(self._lib.mcb200_multiple_refresh(self._ctx, _ptr(de, ctypes.c_int32), _ptr(dh, ctypes.c_int32),
                                                      step, seed, ctypes.byref(gen) if wait else None),
                    "multiple_refresh")
        return gen.value if wait else None

    def set_refresh_targets(self, desired_e, desired_h):
        """Upload the MultipleRefresh targets now, not at the first refresh."""
        de, dh = (np.ascontiguousarray(a, dtype=np.int32) for a in (desired_e, desired_h))
        self._check(self._lib.mcb200_set_refresh_targets(self._ctx, _ptr(de, ctypes.c_int32), _ptr(dh, ctypes.c_int32)),
                    "set_refresh_targets")

    def deposit(self):
        self._check(self._lib.mcb200_deposit(self._ctx), "deposit")

    def solve_poisson(self, rel_tol=1e-10, max_iter=20000):
        it, res = ctypes.c_int(), ctypes.c_double()
        self._check(self._lib.mcb200_solve_poisson(self._ctx, rel_tol, max_iter, ctypes.byref(it),
                                                   ctypes.byref(res)), "solve_poisson")
        return it.value, res.value

    def solve_poisson_async(self, rel_tol=1e-10, max_iter=20000):
        """A solve the host does not wait for (results in poisson_stats())."""
        self._check(self._lib.mcb200_solve_poisson(self._ctx, rel_tol, max_iter, None, None), "solve_poisson")

    def poisson_stats(self, reset=False):
        """(solves, CG iterations, largest relative residual) since the last reset."""
        n, it, res = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double()
        self._check(self._lib.mcb200_poisson_stats(self._ctx, ctypes.byref(n), ctypes.byref(it), ctypes.byref(res),
                                                   1 if reset else 0), "poisson_stats")
        return n.value, it.value, res.value

    def particle_steps(self) -> int:
        """Particle-steps flown since the context was created (device count)."""
        v = ctypes.c_uint64()
        self._check(self._lib.mcb200_particle_steps(self._ctx, ctypes.byref(v)), "particle_steps")
        return v.value

    def set_potential(self, potential):
        """Node potential (normalised) and the cell fields derived from it."""
        pot = np.ascontiguousarray(potential, dtype=np.float64)
        assert pot.size == self.mesh.nnodes
        self._check(self._lib.mcb200_set_potential(self._ctx, _ptr(pot, ctypes.c_double)), "set_potential")

    def set_potentials(self, potential, electron_potential=None):
        """The holes' field from `potential`, the electrons' from
        `electron_potential` (default: the same) -- heat_field's pair of
        mean potentials."""
        pot = np.ascontiguousarray(potential, dtype=np.float64)
        assert pot.size == self.mesh.nnodes
        pe = None if electron_potential is None else np.ascontiguousarray(electron_potential, dtype=np.float64)
        self._check(self._lib.mcb200_set_potentials(self._ctx, _ptr(pot, ctypes.c_double),
                                                    None if pe is None else _ptr(pe, ctypes.c_double)),
                    "set_potentials")

    def set_quantum_correction(self, material=None, quantum_region=None, ratio=(0, 0, 0), theta=(0, 0, 0), eb=0.0,
                               enable=False, setup=True):
        """Effective-potential quantum correction (mcb200_set_quantum_correction):
        with setup, built from per-cell material and quantum-region flags and
        the normalised window (ratio, theta per axis, barrier eb); enable
        switches it on for later Poisson solves."""
        if setup:
            p = QuantumParams((ctypes.c_double * 3)(*ratio), (ctypes.c_double * 3)(*theta), eb)
            mat = np.ascontiguousarray(material, dtype=np.int32)
            reg = np.ascontiguousarray(quantum_region, dtype=np.int32)
            self._check(self._lib.mcb200_set_quantum_correction(self._ctx, ctypes.byref(p), _ptr(mat, ctypes.c_int32),
                                                                _ptr(reg, ctypes.c_int32), int(bool(enable))),
                        "set_quantum_correction")
        else:
            self._check(self._lib.mcb200_set_quantum_correction(self._ctx, None, None, None, int(bool(enable))),
                        "set_quantum_correction")

    def quantum_potential(self, potential) -> np.ndarray:
        """The effective potential of `potential` (mcb200_quantum_potential)."""
        pot = np.ascontiguousarray(potential, dtype=np.float64)
        out = np.empty_like(pot)
        self._check(self._lib.mcb200_quantum_potential(self._ctx, _ptr(pot, ctypes.c_double),
                                                       _ptr(out, ctypes.c_double)), "quantum_potential")
        return out

    def set_poisson_solver(self, method=POISSON_AUTO, blocks=0):
        """Preconditioner of the following solves (POISSON_AUTO / _JACOBI /
        _MULTIGRID) and their cooperative grid (0: the largest co-resident)."""
        self._check(self._lib.mcb200_set_poisson_solver(self._ctx, method, blocks), "set_poisson_solver")

    def poisson_solver(self):
        """(preconditioner of the last solve, its grid, multigrid levels)."""
        m, b, l = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.mcb200_get_poisson_solver(self._ctx, ctypes.byref(m), ctypes.byref(b), ctypes.byref(l)),
                    "poisson_solver")
        return m.value, b.value, l.value

    def array(self, name: str) -> np.ndarray:
        m = self.mesh
        per = {"rho": m.ncells, "efield": 3 * m.ncells, "hfield": 3 * m.ncells, "induced_field": 3 * m.ncells,
               "cell_charge_e": m.ncells,
               "cell_charge_h": m.ncells, "cell_volume": m.ncells, "stencil": 7 * m.nnodes,
               "e_rough": m.ncells, "e_phonon": m.ncells, "h_rough": m.ncells, "h_phonon": m.ncells}
        out = np.zeros(per.get(name, m.nnodes))
        self._check(self._lib.mcb200_get_array(self._ctx, name.encode(), _ptr(out, ctypes.c_double), out.size),
                    name)
        return out

    def set_cells(self, motion_rule, da, attached_contact=None, in_surf_region=None, nearest_surf=None,
                  surface_dir=None, flags: int = 0):
        i32 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.int32)
        mr, ac, isr, ns, sd = (i32(a) for a in (motion_rule, attached_contact, in_surf_region, nearest_surf,
                                                  surface_dir))
        da = np.ascontiguousarray(da, dtype=np.float64)
        assert mr.size == 6 * self.mesh.ncells and da.size == self.mesh.ncells
        nsd = 0 if sd is None else int(sd.size)
        self._check(self._lib.mcb200_set_cells(self._ctx, _ptr(mr, ctypes.c_int32), _ptr(ac, ctypes.c_int32),
                                               _ptr(isr, ctypes.c_int32), _ptr(ns, ctypes.c_int32),
                                               _ptr(sd, ctypes.c_int32), nsd, _ptr(da, ctypes.c_double), flags),
                    "set_cells")

    def set_fields(self, efield_xyz, hfield_xyz, rho):
        e, h, r = (np.ascontiguousarray(a, dtype=np.float64) for a in (efield_xyz, hfield_xyz, rho))
        assert e.size == 3 * self.mesh.ncells and h.size == 3 * self.mesh.ncells and r.size == self.mesh.ncells
        self._check(self._lib.mcb200_set_fields(self._ctx, _ptr(e, ctypes.c_double), _ptr(h, ctypes.c_double),
                                                _ptr(r, ctypes.c_double)), "set_fields")

    def set_surface_rates(self, e_rough, e_phonon, h_rough, h_phonon):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (e_rough, e_phonon, h_rough, h_phonon)]
        self._check(self._lib.mcb200_set_surface_rates(self._ctx, *[_ptr(a, ctypes.c_double) for a in arrs]),
                    "set_surface_rates")

    @staticmethod
    def _soa(arrays: dict) -> _Particles:
        p = _Particles()
        for name in PARTICLE_FIELDS:
            setattr(p, name, arrays[name].ctypes.data)
        return p

    def upload(self, particles: dict):
        arrs = {k: np.ascontiguousarray(particles[k], dtype=t) for k, t in PARTICLE_FIELDS.items()}
        n = len(arrs["x"])
        self._check(self._lib.mcb200_upload_particles(self._ctx, n, ctypes.byref(self._soa(arrs))), "upload")

    def seed(self, cell_of, charge, carrier_type: int, seed: int):
        """Append particles sampled on the GPU (mcb200_seed_particles)."""
        cell_of = np.ascontiguousarray(cell_of, dtype=np.int32)
        charge = np.ascontiguousarray(charge, dtype=np.float64)
        self._check(self._lib.mcb200_seed_particles(self._ctx, cell_of.size, _ptr(cell_of, ctypes.c_int32),
                                                    _ptr(charge, ctypes.c_double), carrier_type, seed), "seed")

    def set_timing(self, enable=True):
        """Time steps with CUDA events: False off, True every step, an int k
        one step in k (mcb200_set_timing)."""
        self._check(self._lib.mcb200_set_timing(self._ctx, int(enable)), "set_timing")

    def timing(self) -> dict:
        out = np.zeros(6)
        self._check(self._lib.mcb200_get_timing(self._ctx, _ptr(out, ctypes.c_double), 6), "timing")
        keys = ["flight_ms", "flight_launches", "step_ms", "steps", "particles_flown", "launches"]
        return dict(zip(keys, out.tolist()))

    def num_particles(self) -> int:
        return int(self._lib.mcb200_num_particles(self._ctx))

    def download(self) -> dict:
        n = self.num_particles()
        arrs = {k: np.empty(n, dtype=t) for k, t in PARTICLE_FIELDS.items()}
        got = ctypes.c_size_t()
        self._check(self._lib.mcb200_download_particles(self._ctx, ctypes.byref(self._soa(arrs)), n,
                                                        ctypes.byref(got)), "download")
        return arrs

    def step(self, step: int, seed: int, dt: float):
        self._check(self._lib.mcb200_step(self._ctx, step, seed, dt), "step")

    def sync(self):
        self._check(self._lib.mcb200_sync(self._ctx), "sync")

    def tallies(self) -> dict:
        m = self.mesh
        counters = np.zeros(NUM_COUNTERS, dtype=np.uint64)
        contact = np.zeros(16 * 6)
        lcur, rcur = np.zeros(m.ny + 1), np.zeros(m.ny + 1)
        he, hh = np.zeros(m.nnodes), np.zeros(m.nnodes)
        self._check(self._lib.mcb200_get_tallies(
            self._ctx, _ptr(counters, ctypes.c_uint64), _ptr(contact, ctypes.c_double), _ptr(lcur, ctypes.c_double),
            _ptr(rcur, ctypes.c_double), _ptr(he, ctypes.c_double), _ptr(hh, ctypes.c_double)), "tallies")
        out = {name: int(counters[i]) for i, name in enumerate(COUNTER_NAMES)}
        out.update(contact=contact.reshape(16, 6), lcurrent=lcur, rcurrent=rcur, heat_e=he, heat_h=hh)
        return out

    def tallies_enqueue(self, slot: int):
        """Copy the contact tallies into ring slot `slot` (0-3) without
        waiting (mcb200_tallies_enqueue)."""
        self._check(self._lib.mcb200_tallies_enqueue(self._ctx, int(slot)), "tallies_enqueue")

    def tallies_collect(self, slot: int) -> np.ndarray:
        """The contact tallies of slot `slot` ([16, 6], as tallies()['contact']),
        waiting for that copy only."""
        contact = np.zeros(16 * 6)
        self._check(self._lib.mcb200_tallies_collect(self._ctx, int(slot), _ptr(contact, ctypes.c_double)),
                    "tallies_collect")
        return contact.reshape(16, 6)

    def reset_tallies(self):
        self._check(self._lib.mcb200_reset_tallies(self._ctx), "reset_tallies")

    def set_induced_current(self, contact: int):
        """Weighting field of `contact` (Ramo-Shockley); every transport
        step then tallies the current it carries by induction."""
        self._check(self._lib.mcb200_set_induced_current(self._ctx, int(contact)), "set_induced_current")

    def induced_current(self) -> tuple:
        """(sum over steps of sum_i q v . E_w, steps) since the last reset."""
        s, n = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.mcb200_get_induced_current(self._ctx, ctypes.byref(s), ctypes.byref(n)),
                    "get_induced_current")
        return s.value, n.value

    def stat_begin(self, window_steps: int):
        self._check(self._lib.mcb200_stat_begin(self._ctx, int(window_steps)), "stat_begin")

    def stat_accumulate(self):
        self._check(self._lib.mcb200_stat_accumulate(self._ctx), "stat_accumulate")

    def stat(self, name: str, n: int = 0) -> np.ndarray:
        """A window sum (mcb200_stat_get); n: entries (default: per node,
        1 for "steps", per cell for "cell_count")."""
        if not n:
            n = 1 if name == "steps" else (self.mesh.ncells if name == "cell_count" else self.mesh.nnodes)
        out = np.zeros(n)
        self._check(self._lib.mcb200_stat_get(self._ctx, name.encode(), _ptr(out, ctypes.c_double), n), name)
        return out


class Batch:
    """Engines made alike stepped together (mcb200_batch_*): one persistent
    flight launch over all members per step.  members: [(engine, dt, seed,
    first_step)] or [(engine, dict of BatchMember fields)]."""

    def __init__(self, members):
        self._lib = lib()
        self._b = ctypes.c_void_p()
        self.engines = [m[0] for m in members]
        ctxs = (ctypes.c_void_p * len(members))(*[m[0]._ctx.value for m in members])

        def member(m):
            if isinstance(m[1], dict):
                return BatchMember(**m[1])
            return BatchMember(m[1], m[2], m[3])

        cfg = (BatchMember * len(members))(*[member(m) for m in members])
        rc = self._lib.mcb200_batch_create(ctxs, cfg, len(members), ctypes.byref(self._b))
        if rc != OK:
            msg = self._lib.mcb200_batch_last_error(self._b).decode() if self._b else "no batch"
            self.close()
            raise EngineError(f"mcb200_batch_create failed ({rc}): {msg}")

    def close(self):
        if self._b:
            self._lib.mcb200_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != OK:
            raise EngineError(f"{what} failed ({rc}): {self._lib.mcb200_batch_last_error(self._b).decode()}")

    def step(self):
        self._check(self._lib.mcb200_batch_step(self._b), "mcb200_batch_step")

    def run(self, steps: int):
        """Full timesteps of every member (mcb200_batch_run)."""
        self._check(self._lib.mcb200_batch_run(self._b, steps), "mcb200_batch_run")

    def autotune(self, trial_steps: int) -> dict:
        """Launch shapes picked by timing real steps (mcb200_batch_autotune)."""
        t = BatchTuning()
        self._check(self._lib.mcb200_batch_autotune(self._b, trial_steps, ctypes.byref(t)), "mcb200_batch_autotune")
        return {name: getattr(t, name) for name, _ in BatchTuning._fields_}

    def use_graphs(self, enable: bool = True):
        self._check(self._lib.mcb200_batch_use_graphs(self._b, int(enable)), "mcb200_batch_use_graphs")

    def sync(self):
        self._check(self._lib.mcb200_batch_sync(self._b), "mcb200_batch_sync")

    def set_grid(self, blocks_per_sm: int):
        self._check(self._lib.mcb200_batch_set_grid(self._b, blocks_per_sm), "mcb200_batch_set_grid")

    def set_solo(self, min_particles: int) -> int:
        """Members with at least min_particles particles (0: none) fly in
        launches of their own; returns how many."""
        k = ctypes.c_int()
        self._check(self._lib.mcb200_batch_set_solo(self._b, int(min_particles), ctypes.byref(k)),
                    "mcb200_batch_set_solo")
        return k.value

    def set_smem_table(self, enable: bool = True):
        """Copy the member table into each flight block's shared memory
        (default off: read in place)."""
        self._check(self._lib.mcb200_batch_set_smem_table(self._b, int(bool(enable))), "mcb200_batch_set_smem_table")

    def set_overlap(self, enable: bool = True):
        """Fly the members not solving Poisson beside the solves (default on)."""
        self._check(self._lib.mcb200_batch_set_overlap(self._b, int(bool(enable))), "mcb200_batch_set_overlap")

    def set_pairing(self, enable: bool = True):
        """Two due multigrid solves of the same shape per launch (default on)."""
        self._check(self._lib.mcb200_batch_set_pairing(self._b, int(bool(enable))), "mcb200_batch_set_pairing")

    def mark(self, slot: int):
        self._check(self._lib.mcb200_batch_mark(self._b, slot), "mcb200_batch_mark")

    def elapsed_ms(self, a: int, b: int) -> float:
        v = ctypes.c_double()
        self._check(self._lib.mcb200_batch_elapsed_ms(self._b, a, b, ctypes.byref(v)), "mcb200_batch_elapsed_ms")
        return v.value

    def info(self) -> dict:
        n, st, la, gc, gr = ctypes.c_int(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self._lib.mcb200_batch_info(self._b, ctypes.byref(n), ctypes.byref(st), ctypes.byref(la),
                                                ctypes.byref(gc), ctypes.byref(gr)), "mcb200_batch_info")
        return {"members": n.value, "steps": st.value, "launches": la.value, "graph_captures": gc.value,
                "graph_replays": gr.value}


class Server:
    """Bias-point requests served by continuous batching (mcb200_server_*)."""

    def __init__(self, table_dir: str = DEFAULT_TABLE_DIR, device: int = 0, precision: int = FLIGHT_FP32,
                 hbm_budget_bytes: int = 0, max_slots: int = 64, quantum_steps: int = 50, use_graphs: bool = False,
                 kelvin: float = 300.0):
        self._lib = lib()
        self._s = ctypes.c_void_p()
        self._table_dir = table_dir.encode()
        opt = ServerOptions(self._table_dir, kelvin, device, precision, hbm_budget_bytes, max_slots, quantum_steps,
                            int(use_graphs))
        rc = self._lib.mcb200_server_create(ctypes.byref(opt), ctypes.byref(self._s))
        if rc != OK:
            msg = self._lib.mcb200_server_last_error(self._s).decode() if self._s else "no server"
            self.close()
            raise EngineError(f"mcb200_server_create failed ({rc}): {msg}")

    def close(self):
        if self._s:
            self._lib.mcb200_server_destroy(self._s)
            self._s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != OK:
            raise EngineError(f"{what} failed ({rc}): {self._lib.mcb200_server_last_error(self._s).decode()}")

    def now(self) -> float:
        return self._lib.mcb200_server_now(self._s)

    def submit(self, input_path: str, family: str, bias, seed: int, target_rel_err: float = 0.01,
               min_windows: int = 5, max_steps: int = 0, warm_windows_cold: int = 10, warm_windows_warm: int = 1,
               warm_start: int = WARM_CONVERGED, poisson_every: int = 0, drain_contact: int = 1, ids_estimator: int = 0,
               arrival_s=None) -> int:
        req = Request(os.fspath(input_path).encode(), family.encode(), (ctypes.c_double * 2)(*bias), target_rel_err,
                      min_windows, max_steps, warm_windows_cold, warm_windows_warm, int(warm_start), poisson_every,
                      drain_contact, int(ids_estimator), seed, self.now() if arrival_s is None else arrival_s)
        rid = ctypes.c_uint64()
        self._check(self._lib.mcb200_server_submit(self._s, ctypes.byref(req), ctypes.byref(rid)),
                    "mcb200_server_submit")
        return rid.value

    def round(self):
        """One scheduling round; returns (active, pending)."""
        a, p = ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.mcb200_server_round(self._s, ctypes.byref(a), ctypes.byref(p)), "mcb200_server_round")
        return a.value, p.value

    def results(self) -> list:
        out = []
        buf = (Result * 64)()
        while True:
            n = ctypes.c_int()
            self._check(self._lib.mcb200_server_results(self._s, buf, 64, ctypes.byref(n)), "mcb200_server_results")
            for r in buf[:n.value]:
                out.append({f: getattr(r, f) for f, _ in Result._fields_})
            if n.value < 64:
                return out

    def stats(self) -> dict:
        st = ServerStats()
        self._check(self._lib.mcb200_server_stats(self._s, ctypes.byref(st)), "mcb200_server_stats")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}


class Deck:
    """A reference input deck (input.txt + lgrid.txt + ldg.txt) read by the
    engine library's own parser (mcb200_deck_load)."""

    def __init__(self, input_path: str):
        self._lib = lib()
        self._deck = ctypes.c_void_p()
        rc = self._lib.mcb200_deck_load(os.fspath(input_path).encode(), ctypes.byref(self._deck))
        if rc != OK:
            msg = self._lib.mcb200_deck_error(self._deck).decode() if self._deck else "no deck"
            self.close()
            raise EngineError(f"mcb200_deck_load failed ({rc}): {msg}")

    def close(self):
        if self._deck:
            self._lib.mcb200_deck_free(self._deck)
            self._deck = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != OK:
            raise EngineError(f"{what} failed ({rc}): {self._lib.mcb200_deck_error(self._deck).decode()}")

    def info(self) -> dict:
        inf = DeckInfo()
        self._check(self._lib.mcb200_deck_get_info(self._deck, ctypes.byref(inf)), "mcb200_deck_get_info")
        out = {name: getattr(inf, name) for name, _ in DeckInfo._fields_}
        out["output_dir"] = inf.output_dir.decode()
        return out

    def int_array(self, name: str) -> np.ndarray:
        need = ctypes.c_size_t()
        self._check(self._lib.mcb200_deck_int_array(self._deck, name.encode(), None, 0, ctypes.byref(need)), name)
        out = np.empty(need.value, dtype=np.int32)
        self._check(self._lib.mcb200_deck_int_array(self._deck, name.encode(), _ptr(out, ctypes.c_int32), out.size,
                                                    ctypes.byref(need)), name)
        return out

    def double_array(self, name: str) -> np.ndarray:
        need = ctypes.c_size_t()
        self._check(self._lib.mcb200_deck_double_array(self._deck, name.encode(), None, 0, ctypes.byref(need)), name)
        out = np.empty(need.value, dtype=np.float64)
        self._check(self._lib.mcb200_deck_double_array(self._deck, name.encode(), _ptr(out, ctypes.c_double),
                                                       out.size, ctypes.byref(need)), name)
        return out

    def prepare(self, engine: "Engine"):
        self._check(self._lib.mcb200_deck_prepare(self._deck, engine._ctx), "mcb200_deck_prepare")

    def apply(self, engine: "Engine"):
        """Mesh, cells and device of the deck into `engine`."""
        self._check(self._lib.mcb200_apply_deck(engine._ctx, self._deck), "mcb200_apply_deck")
        lx, ly, lz = (self.double_array(n) for n in ("lx", "ly", "lz"))
        engine.mesh = Mesh(len(lx) - 1, len(ly) - 1, len(lz) - 1, lx, ly, lz)

    def seed(self, engine: "Engine", seed: int):
        """The deck's initial ensemble (init_particle_data) into `engine`."""
        self._check(self._lib.mcb200_seed_deck(engine._ctx, self._deck, seed), "mcb200_seed_deck")


def run_deck(input_path: str, device: int = 0, data_dir: str | None = None, precision: int = FLIGHT_FP64,
             max_steps: int = 0, max_heat_steps: int = -1, poisson_every: int = 0, seed: int = 1,
             write_outputs: bool = True, table_dir: str = DEFAULT_TABLE_DIR, verbose: bool = False,
             warmup_steps: int = 0, readback_every_step: bool = False, flush_l2_bytes: int = 0,
             profile_phases: bool = False) -> dict:
    """The self-consistent simulation of a deck (mcb200_run_deck, the engine's
    `main input.txt`).  Returns the run report as a dict."""
    opt = RunOptions(table_dir=table_dir.encode(), data_dir=data_dir.encode() if data_dir else None,
                     flight_precision=precision, poisson_every=poisson_every, poisson_rel_tol=0.0,
                     max_steps=max_steps, max_heat_steps=max_heat_steps, write_outputs=int(write_outputs),
                     seed=seed, verbose=int(verbose), warmup_steps=warmup_steps,
                     readback_every_step=int(readback_every_step), flush_l2_bytes=flush_l2_bytes,
                     profile_phases=int(profile_phases))
    rep = RunReport()
    err = ctypes.create_string_buffer(1024)
    rc = lib().mcb200_run_deck(os.fspath(input_path).encode(), device, ctypes.byref(opt), ctypes.byref(rep), err,
                               len(err))
    if rc != OK:
        raise EngineError(f"mcb200_run_deck failed ({rc}): {err.value.decode()}")
    out = {name: getattr(rep, name) for name, _ in RunReport._fields_}
    out["last_current"] = rep.last_current[0]
    out["phase_s"] = dict(zip(("statistics", "deposition", "poisson", "surface_rates", "step", "refresh", "outputs"),
                              list(rep.phase_s)[:7]))
    return out
