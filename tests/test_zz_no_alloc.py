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
(cell, uid) order.  Particles marked dropped must be left out, cells off
the mesh and overlapping stores must be refused.  This file is collected
last on purpose.
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


def sort_fn():
    lib = mcb200.lib()
    lib.mcb200_sort_particles_static.argtypes = [ctypes.POINTER(DeviceParticles), ctypes.c_size_t, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_int, ctypes.POINTER(DeviceParticles),
                                                 ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p]
    return lib.mcb200_sort_particles_static


def to_device(torch, src: dict) -> dict:
    return {k: torch.from_numpy(src[k].view(np.int32) if src[k].dtype == np.uint32 else src[k]).cuda()
            for k in FIELDS}


def describe(dev: dict) -> DeviceParticles:
    return DeviceParticles(*[dev[k].data_ptr() for k in FIELDS])


def test_static_sort_matches_engine_sort():
    """Two calls in a row against the engine's own sort, with a few particles
    marked dropped (meta bit 16); the second call on a caller's stream."""
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
    dropped = np.random.default_rng(2).choice(n, 37, replace=False)
    src["meta"][dropped] |= np.uint32(1 << 16)
    keep = ~np.isin(ref["uid"], src["uid"][dropped])
    ref = {k: v[keep] for k, v in ref.items()}
    ref_lin = ref_lin[keep]
    dev_in = to_device(torch, src)
    dev_out = {k: torch.empty_like(t) for k, t in dev_in.items()}
    desc_in, desc_out = describe(dev_in), describe(dev_out)
    sort = sort_fn()
    side = torch.cuda.Stream()
    for call in range(2):
        for t in dev_out.values():  # poison the output so every kept entry must be written
            t.fill_(-1)
        torch.cuda.synchronize()
        kept = ctypes.c_size_t(0)
        handle = None if call == 0 else ctypes.c_void_p(side.cuda_stream)
        rc = sort(ctypes.byref(desc_in), n, nx, ny, nz, ctypes.byref(desc_out), ctypes.byref(kept), handle)
        torch.cuda.synchronize()
        assert rc == 0, f"call {call}: status {rc}"
        assert kept.value == n - len(dropped)
        m = kept.value
        got = {k: dev_out[k][:m].cpu().numpy() for k in FIELDS}
        got = {k: (v.view(np.uint32) if DTYPES[k] == np.uint32 else v) for k, v in got.items()}
        c = got["cell"].astype(np.int64)
        in_order = (((c >> 10) & 1023) * nx + (c & 1023)) * nz + ((c >> 20) & 1023)
        assert np.all(np.diff(in_order) >= 0), f"call {call}: output not grouped by cell"
        assert not np.isin(got["uid"], src["uid"][dropped]).any(), f"call {call}: a dropped particle was kept"
        got_c, lin = canonical(got, nx, nz)
        assert np.array_equal(lin, ref_lin)
        for k in FIELDS:
            assert np.array_equal(got_c[k], ref[k]), f"call {call}: field {k} differs"


def test_static_sort_rejects_cells_off_the_mesh():
    """A live particle whose cell lies outside the mesh is an argument error;
    the kernels skip it (no access past the mesh), and a correct call right
    after gives the full result."""
    torch = pytest.importorskip("torch")
    eng, (nx, ny, nz) = make_engine(electrons=800, holes=100)
    src = packed(eng.download())
    eng.close()
    n = len(src["x"])
    good = {k: v.copy() for k, v in src.items()}
    src["cell"][5] = np.uint32(nx | (1 << 10))       # i = nx
    src["cell"][9] = np.uint32(2 | ((ny + 3) << 10))  # j beyond ny
    src["cell"][11] = np.uint32(1 | (1023 << 20))     # k = 1023
    dev_in, dev_good = to_device(torch, src), to_device(torch, good)
    dev_out = {k: torch.empty_like(t) for k, t in dev_in.items()}
    sort = sort_fn()
    kept = ctypes.c_size_t(0)
    rc = sort(ctypes.byref(describe(dev_in)), n, nx, ny, nz, ctypes.byref(describe(dev_out)), ctypes.byref(kept),
              None)
    assert rc == 1  # MCB200_ERR_ARG
    assert kept.value == n - 3
    rc = sort(ctypes.byref(describe(dev_good)), n, nx, ny, nz, ctypes.byref(describe(dev_out)), ctypes.byref(kept),
              None)
    assert rc == 0 and kept.value == n


def test_static_sort_rejects_overlapping_stores():
    torch = pytest.importorskip("torch")
    eng, (nx, ny, nz) = make_engine(electrons=200, holes=20)
    src = packed(eng.download())
    eng.close()
    n = len(src["x"])
    dev = to_device(torch, src)
    sort = sort_fn()
    same = describe(dev)
    assert sort(ctypes.byref(same), n, nx, ny, nz, ctypes.byref(same), None, None) == 1
    other = {k: torch.empty_like(t) for k, t in dev.items()}
    out = describe(other)
    out.energy = dev["charge"].data_ptr() + 8  # one output array inside an input array
    assert sort(ctypes.byref(same), n, nx, ny, nz, ctypes.byref(out), None, None) == 1


def test_static_sort_rejects_oversized_mesh():
    empty = DeviceParticles()
    rc = sort_fn()(ctypes.byref(empty), 0, 1000, 1000, 1, ctypes.byref(empty), None, None)
    assert rc == 4  # MCB200_ERR_CAPACITY: 10^6 cells exceed the static scratch
