"""ctypes bridge to the CPU oracle (oracle/_ref/libref_oracle.so).

TEST INFRASTRUCTURE: the oracle is the reference's own hot-path code compiled
by oracle/Makefile; the harness entry points (orc_*) are defined in
oracle/harness/harness.cpp.  Only tests, smoke() and bench.py's CPU baseline
use this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_oracle.so")
ORACLE_TABLES = os.path.join(ROOT, "oracle", "_ref", "input")

D_FIELDS = ["x", "y", "z", "kx", "ky", "kz", "charge", "energy", "left_time"]
I_FIELDS = ["i", "j", "k", "itet", "isym", "type", "flag", "seed", "uid"]

# Band member shapes (include/Band.h), for orc_band_ptr views.
BAND_SHAPES = {
    "tet": (np.int32, (4, 56000)), "NeibrTet": (np.int32, (4, 56000)), "ibt": (np.int32, (56000,)),
    "xkk": (np.float64, (13000,)), "ykk": (np.float64, (13000,)), "zkk": (np.float64, (13000,)),
    "eek": (np.float64, (13000,)), "vt": (np.float64, (4 * 56000,)), "vgt": (np.float64, (56000,)),
    "datantlin": (np.float64, (4, 4, 56000)), "faclow": (np.float64, (56000,)),
    "facmedium": (np.float64, (56000,)), "fachigh": (np.float64, (56000,)), "gamtet": (np.float64, (56000,)),
    "matsym": (np.int32, (6, 48)), "indmat": (np.int32, (729,)), "newisym": (np.int32, (5, 48)),
    "xbz": (np.float64, (5, 48)), "ybz": (np.float64, (5, 48)), "zbz": (np.float64, (5, 48)),
    "ntlist": (np.int32, (325, 8)), "ptlist": (np.int32, (325, 8)), "tlist": (np.int32, (470000,)),
    "nslist": (np.int32, (325, 8)), "pslist": (np.int32, (325, 8)), "slist": (np.int32, (16000,)),
    "ntlists": (np.int32, (60, 8)), "ptlists": (np.int32, (60, 8)), "tlists": (np.int32, (101000,)),
    "dos": (np.float64, (8, 7501)), "sumdos": (np.float64, (7501, 3)), "dostetmax": (np.float64, (8, 7501)),
    "sumscatt": (np.float64, (7501, 8)), "scatte": (np.float64, (14, 4, 4)),
    "scattiie": (np.float64, (4, 4, 7501)), "scatth": (np.float64, (4, 3, 3)),
    "scattiih": (np.float64, (3, 3, 7501)), "dose": (np.float64, (14, 4, 7501)),
    "dosh": (np.float64, (4, 3, 7501)), "energy": (np.float64, (7501,)),
}


class Oracle:
    def __init__(self, path: str = ORACLE_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the reference sources exist")
        lib = ctypes.CDLL(path)
        c = ctypes
        lib.orc_init.argtypes = [c.c_char_p, c.c_char_p, c.c_uint64, c.c_int]
        lib.orc_scalar.argtypes = [c.c_char_p]
        lib.orc_scalar.restype = c.c_double
        lib.orc_set_scalar.argtypes = [c.c_char_p, c.c_double]
        lib.orc_array_len.argtypes = [c.c_char_p]
        lib.orc_get_array.argtypes = [c.c_char_p, c.c_void_p]
        lib.orc_set_array.argtypes = [c.c_char_p, c.c_void_p]
        lib.orc_get_particles.argtypes = [c.c_void_p, c.c_void_p]
        lib.orc_set_particles.argtypes = [c.c_int, c.c_void_p, c.c_void_p]
        lib.orc_flight_step.argtypes = [c.c_uint32, c.POINTER(c.c_int)]
        lib.orc_contacts.argtypes = [c.c_void_p]
        lib.orc_band_ptr.argtypes = [c.c_char_p]
        lib.orc_band_ptr.restype = c.c_void_p
        lib.orc_band_scalar.argtypes = [c.c_char_p]
        lib.orc_band_scalar.restype = c.c_double
        lib.orc_build_band_only.argtypes = [c.c_char_p, c.c_double]
        lib.orc_time_update_particle.argtypes = [c.c_int, c.c_int]
        lib.orc_time_update_particle.restype = c.c_double
        lib.orc_mesh_dims.argtypes = [c.c_void_p]
        lib.orc_quiet.argtypes = [c.c_int]
        self.lib = lib

    # -- set-up -------------------------------------------------------------
    def init(self, input_file: str, seed: int, make_particles: bool = True, table_dir: str = ORACLE_TABLES):
        self.lib.orc_quiet(1)
        rc = self.lib.orc_init(os.path.abspath(input_file).encode(), table_dir.encode(), seed, int(make_particles))
        if rc != 0:
            raise RuntimeError("orc_init failed")

    def build_band_only(self, kelvin: float = 300.0, table_dir: str = ORACLE_TABLES):
        self.lib.orc_quiet(1)
        if self.lib.orc_build_band_only(table_dir.encode(), kelvin) != 0:
            raise RuntimeError("orc_build_band_only failed")

    # -- accessors ------------------------------------------------------------
    def scalar(self, name: str) -> float:
        return float(self.lib.orc_scalar(name.encode()))

    def set_scalar(self, name: str, v: float):
        if self.lib.orc_set_scalar(name.encode(), float(v)) != 0:
            raise KeyError(name)

    def dims(self):
        d = np.zeros(6, dtype=np.int32)
        self.lib.orc_mesh_dims(d.ctypes.data)
        return tuple(int(v) for v in d)

    def array(self, name: str) -> np.ndarray:
        n = self.lib.orc_array_len(name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        self.lib.orc_get_array(name.encode(), out.ctypes.data)
        return out

    def set_array(self, name: str, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        if v.size != self.lib.orc_array_len(name.encode()) or self.lib.orc_set_array(name.encode(), v.ctypes.data):
            raise KeyError(name)

    def band(self, name: str) -> np.ndarray:
        dt, shape = BAND_SHAPES[name]
        p = self.lib.orc_band_ptr(name.encode())
        buf = (ctypes.c_char * (int(np.prod(shape)) * np.dtype(dt).itemsize)).from_address(p)
        return np.frombuffer(buf, dtype=dt).reshape(shape).copy()

    def band_scalar(self, name: str) -> float:
        return float(self.lib.orc_band_scalar(name.encode()))

    # -- particles ------------------------------------------------------------
    def particles(self) -> dict:
        n = self.lib.orc_num_particles()
        d = np.zeros((n, 9))
        iv = np.zeros((n, 9), dtype=np.int32)
        self.lib.orc_get_particles(d.ctypes.data, iv.ctypes.data)
        out = {k: d[:, q].copy() for q, k in enumerate(D_FIELDS)}
        out.update({k: iv[:, q].copy() for q, k in enumerate(I_FIELDS)})
        out["uid"] = out["uid"].astype(np.uint32)
        return out

    def set_particles(self, p: dict, dt: float):
        n = len(p["x"])
        d = np.zeros((n, 9))
        iv = np.zeros((n, 9), dtype=np.int32)
        for q, k in enumerate(D_FIELDS):
            d[:, q] = p[k] if k != "left_time" else dt
        for q, k in enumerate(I_FIELDS):
            if k in p:
                iv[:, q] = p[k]
        iv[:, I_FIELDS.index("flag")] = 1
        self.lib.orc_set_particles(n, d.ctypes.data, iv.ctypes.data)

    def flight_step(self, step: int):
        unfinished = ctypes.c_int()
        n = self.lib.orc_flight_step(step, ctypes.byref(unfinished))
        return n, unfinished.value

    def compute_cell_charge(self):
        self.lib.orc_compute_cell_charge()

    def surface_rates(self):
        self.lib.orc_surface_rates()

    def reset_tallies(self):
        self.lib.orc_reset_tallies()

    def multiple_refresh(self, step: int) -> int:
        self.lib.orc_multiple_refresh.argtypes = [ctypes.c_uint32]
        return int(self.lib.orc_multiple_refresh(step))

    def init_quantum(self):
        """The reference's quantum-correction set-up (init_effective_potential,
        init_p_mat, init_ep_range), from the deck's ep_parm and quantumRegion."""
        self.lib.orc_init_quantum()

    def dispersion(self, which: int, rows: int, cols: int) -> np.ndarray:
        out = np.zeros(rows * cols)
        self.lib.orc_dispersion.argtypes = [ctypes.c_int, ctypes.c_void_p]
        assert self.lib.orc_dispersion(which, out.ctypes.data) == 0
        return out

    def quantum_potential(self):
        """quantumPotential: p_poisson_pot corrected at the quantum nodes."""
        self.lib.orc_quantum_potential()

    def density_and_field(self):
        """particle_to_density -> compute_field (Poisson + pot2field) -> compute_cell_charge."""
        self.lib.orc_density_and_field()

    def contact_info(self):
        per = np.zeros(16 * 3)
        planes = np.zeros(64 * 7, dtype=np.int32)
        n = self.lib.orc_contact_info(per.ctypes.data, planes.ctypes.data, 64)
        nc = int(self.scalar("num_contact"))
        per = per[:3 * nc].reshape(nc, 3)
        return per[:, 1].copy(), per[:, 2].copy(), planes[:7 * n].reshape(n, 7).copy()

    def poisson_stencil(self) -> np.ndarray:
        nx, ny, nz, px, py, pz = self.dims()
        out = np.zeros(px * py * pz * 7)
        self.lib.orc_poisson_stencil(out.ctypes.data)
        return out

    def contacts(self) -> np.ndarray:
        out = np.zeros((16, 6))
        n = self.lib.orc_contacts(out.ctypes.data)
        return out[:n]

    def statistic(self):
        """statistic(): one step's sums added to the stat_* vectors."""
        self.lib.orc_statistic()

    def set_stat_zero(self):
        """set_stat_zero(): statistics, contact tallies and section currents cleared."""
        self.lib.orc_set_stat_zero()

    def write_outputs(self, folder: str, step: int):
        """output_stat + output_for_restart for `step`, under folder/data/."""
        self.lib.orc_write_outputs.argtypes = [ctypes.c_char_p, ctypes.c_int]
        if self.lib.orc_write_outputs(os.path.abspath(folder).encode(), int(step)) != 0:
            raise RuntimeError("orc_write_outputs failed")

    def seed_particle(self, seed: int, uid: int, i: int, j: int, k: int, carrier: int, charge: float) -> dict:
        """One initial-ensemble particle (init_particle_data's placement +
        select_kstate) on the per-particle stream (seed, uid, 0xfffffffd, 0)."""
        c = ctypes
        self.lib.orc_seed_particle.argtypes = [c.c_uint64, c.c_uint32, c.c_int, c.c_int, c.c_int, c.c_int,
                                               c.c_double, c.c_void_p, c.c_void_p]
        d = np.zeros(9)
        iv = np.zeros(9, dtype=np.int32)
        self.lib.orc_seed_particle(seed, uid, i, j, k, carrier, charge, d.ctypes.data, iv.ctypes.data)
        out = {k_: float(d[q]) for q, k_ in enumerate(D_FIELDS)}
        out.update({k_: int(iv[q]) for q, k_ in enumerate(I_FIELDS)})
        return out

    def time_update_particle(self, nsteps: int, with_cell_charge: bool = True) -> float:
        return float(self.lib.orc_time_update_particle(nsteps, int(with_cell_charge)))
