"""The allocation-free sort entry point (mcb200_sort_particles_static) against
the engine's own sort.

mcb200_sort_particles_static serves callers that cannot allocate device
memory (a framework that owns every device buffer, code that must not
allocate while other work holds the device): they pass input and output
arrays and the sort's scratch is a static device array inside the library.
Here the caller's buffers come from torch.  The reference result is the
existing entry point: mcb200_step with dt = 0 flies nobody and ends with the
same counting sort by cell.  The two must agree exactly (a sort is a
permutation) on two calls in a row, the second into a poisoned output.
Order inside a cell is unspecified, so both sides are compared in
(cell, uid) order.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import mcb200

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "kx", "ky", "kz", "energy", "charge", "cell", "itet", "meta", "uid")
DTYPES = dict(x=np.float64, y=np.float64, z=np.float64, kx=np.float64, ky=np.float64, kz=np.float64,
              energy=np.float64, charge=np.float64, cell=np.uint32, itet=np.int32, meta=np.uint32, uid=np.uint32)


class DeviceParticles(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in FIELDS]


def packed(host: dict) -> dict:
    """Host particles (mcb200.Engine.download layout) -> the engine's device layout."""
    out = {k: np.ascontiguousarray(host[k], dtype=DTYPES[k]) for k in FIELDS if k in host}
    out["cell"] = (host["i"].astype(np.uint32) | (host["j"].astype(np.uint32) << 10)
                   | (host["k"].astype(np.uint32) << 20))
    out["meta"] = host["isym"].astype(np.uint32) | (host["type"].astype(np.uint32) << 8)
    return out


def canonical(p: dict, nx: int, nz: int) -> dict:
    c = p["cell"].astype(np.int64)
    lin = (((c >> 10) & 1023) * nx + (c & 1023)) * nz + ((c >> 20) & 1023)
    order = np.lexsort((p["uid"], lin))
    return {k: v[order] for k, v in p.items()}, lin


def make_engine(nx=8, ny=6, nz=6, electrons=4000, holes=600):
    eng = mcb200.Engine(kelvin=300.0, device=0, max_particles=2 * (electrons + holes))
    u = eng.units()
    h = 5e-9 / u["spr0"]
    eng.set_mesh(np.arange(nx + 1) * h, np.arange(ny + 1) * h, np.arange(nz + 1) * h)
    cells = nx * ny * nz
    eng.set_cells(np.full(cells * 6, 2, dtype=np.int32), np.full(cells, 1e23 / u["conc0"]))
    eng.set_fields(np.zeros(cells * 3), np.zeros(cells * 3), np.full(cells, 1e23 / u["conc0"]))
    rng = np.random.default_rng(5)
    eng.seed(rng.integers(0, cells, electrons).astype(np.int32), np.full(electrons, -1e-5), 0, 17)
    eng.seed(rng.integers(0, cells, holes).astype(np.int32), np.full(holes, 1e-7), 1, 18)
    return eng, (nx, ny, nz)


def test_static_sort_matches_engine_sort():
    torch = pytest.importorskip("torch")
    eng, (nx, ny, nz) = make_engine()
    host = eng.download()
    n = len(host["x"])
    perm = np.random.default_rng(1).permutation(n)
    shuffled = {k: v[perm] for k, v in host.items()}
    eng.upload(shuffled)
    eng.step(0, 1, 0.0)  # existing entry point: dt = 0 moves nothing, then the cell sort
    ref, ref_lin = canonical(packed(eng.download()), nx, nz)
    eng.close()

    src = packed(shuffled)
    dev_in = {k: torch.from_numpy(src[k].view(np.int32) if src[k].dtype == np.uint32 else src[k]).cuda()
              for k in FIELDS}
    dev_out = {k: torch.empty_like(t) for k, t in dev_in.items()}
    desc_in = DeviceParticles(*[dev_in[k].data_ptr() for k in FIELDS])
    desc_out = DeviceParticles(*[dev_out[k].data_ptr() for k in FIELDS])
    lib = mcb200.lib()
    lib.mcb200_sort_particles_static.argtypes = [ctypes.POINTER(DeviceParticles), ctypes.c_size_t, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_int, ctypes.POINTER(DeviceParticles),
                                                 ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p]
    for call in range(2):
        for t in dev_out.values():  # poison the output so every entry must be written
            t.fill_(-1)
        torch.cuda.synchronize()
        kept = ctypes.c_size_t(0)
        rc = lib.mcb200_sort_particles_static(ctypes.byref(desc_in), n, nx, ny, nz, ctypes.byref(desc_out),
                                              ctypes.byref(kept), None)
        torch.cuda.synchronize()
        assert rc == 0, f"call {call}: status {rc}"
        assert kept.value == n
        got = {k: dev_out[k].cpu().numpy() for k in FIELDS}
        got = {k: (v.view(np.uint32) if DTYPES[k] == np.uint32 else v) for k, v in got.items()}
        c = got["cell"].astype(np.int64)
        in_order = (((c >> 10) & 1023) * nx + (c & 1023)) * nz + ((c >> 20) & 1023)
        assert np.all(np.diff(in_order) >= 0), f"call {call}: output not grouped by cell"
        got_c, lin = canonical(got, nx, nz)
        assert np.array_equal(lin, ref_lin)
        for k in FIELDS:
            assert np.array_equal(got_c[k], ref[k]), f"call {call}: field {k} differs"


def test_static_sort_rejects_oversized_mesh():
    lib = mcb200.lib()
    lib.mcb200_sort_particles_static.argtypes = [ctypes.POINTER(DeviceParticles), ctypes.c_size_t, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_int, ctypes.POINTER(DeviceParticles),
                                                 ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p]
    empty = DeviceParticles()
    rc = lib.mcb200_sort_particles_static(ctypes.byref(empty), 0, 1000, 1000, 1, ctypes.byref(empty), None, None)
    assert rc == 4  # MCB200_ERR_CAPACITY: 10^6 cells exceed the static scratch
