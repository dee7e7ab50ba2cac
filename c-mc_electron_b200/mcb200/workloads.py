"""Synthetic workloads built directly through the engine API.

bulk_box_engine: the frozen-field bulk n-Si box -- nx*ny*nz cubic cells,
uniform donors, REFLECT on the six outer faces and PASS inside, a uniform
field along x, electrons seeded per cell from the engine's equilibrium
sampler (select_kstate, src/mcmodel.cpp:3006-3057).  This is the physics of
the reference's bulk deck (cell counts, doping and motion rules as
decks.bulk_box writes them) without going through deck files, so it scales
to millions of electrons.
"""
from __future__ import annotations

import numpy as np

from . import FLIGHT_FP64, Engine, DEFAULT_TABLE_DIR

BULK_BOX = dict(nx=40, ny=20, nz=20, cell_nm=5.0, donor_m3=1e23, field_v_per_m=1e6, dt_s=1e-15, kelvin=300.0)


def motion_rules(nx: int, ny: int, nz: int) -> np.ndarray:
    """PASS inside, REFLECT on the outer faces; [cells * 6] in cell order
    (j * nx + i) * nz + k, faces UP, DOWN, LEFT, RIGHT, FRONT, BACK."""
    mr = np.full((nx, ny, nz, 6), 1, dtype=np.int32)  # indexed [i, j, k, face]
    mr[0, :, :, 0] = 2
    mr[nx - 1, :, :, 1] = 2
    mr[:, 0, :, 2] = 2
    mr[:, ny - 1, :, 3] = 2
    mr[:, :, 0, 4] = 2
    mr[:, :, nz - 1, 5] = 2
    return np.ascontiguousarray(mr.transpose(1, 0, 2, 3)).reshape(-1)


def uniform_fields(eng: Engine, field_v_per_m: float, donor_m3: float):
    """Cell fields of a neutral box under a uniform field along +x: the
    electron-felt field (ChargeSign = -1), the hole-felt field, and the
    screening density |q|/vol = N_D."""
    u = eng.units()
    cells = eng.mesh.ncells
    e = np.zeros((cells, 3))
    e[:, 0] = -field_v_per_m / u["field0"]
    return e.ravel(), (-e).ravel(), np.full(cells, donor_m3 / u["conc0"])


def bulk_box_engine(particles: int, seed: int, device: int = 0, precision: int = FLIGHT_FP64, like=None,
                    table_dir: str = DEFAULT_TABLE_DIR, **overrides):
    """Engine holding the bulk box with `particles` electrons (rounded down to
    a multiple of the cell count); like: an engine to share band tables with.
    Returns (engine, dt normalised, fields)."""
    box = dict(BULK_BOX, **overrides)
    eng = Engine(table_dir=table_dir, kelvin=box["kelvin"], device=device,
                 max_particles=particles + particles // 8 + 4096, precision=precision, like=like)
    u = eng.units()
    nx, ny, nz = box["nx"], box["ny"], box["nz"]
    h = box["cell_nm"] * 1e-9 / u["spr0"]
    eng.set_mesh(np.arange(nx + 1) * h, np.arange(ny + 1) * h, np.arange(nz + 1) * h)
    cells = nx * ny * nz
    doping = box["donor_m3"] / u["conc0"]
    eng.set_cells(motion_rules(nx, ny, nz), np.full(cells, doping))
    fields = uniform_fields(eng, box["field_v_per_m"], box["donor_m3"])
    eng.set_fields(*fields)
    per_cell = max(particles // cells, 1)
    cell_of = np.repeat(np.arange(cells, dtype=np.int32), per_cell)
    charge = np.full(cell_of.size, -doping * h ** 3 / per_cell)
    eng.seed(cell_of, charge, 0, seed)
    return eng, box["dt_s"] / u["time0"], fields
