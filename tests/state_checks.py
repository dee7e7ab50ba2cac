"""Physical consistency of a downloaded particle store, from the band tables.

For every particle: its k point, folded into the irreducible wedge of its
isym (in_wedge, src/ParticleUtils.cpp:295-305), must lie in its tetrahedron
(the face tests of Band::HESSTET's planes, src/Band.cpp:356-463, measured as
a k-space distance with unit normals); its carried energy must match the
band energy at k (GetEnergy, src/ParticleUtils.cpp:315-329); its position
must lie in its cell.  These hold for any correct flight, whatever the
precision or the random stream, so they check the FP32 path where
bit-exact comparison does not apply.
"""
from __future__ import annotations

import numpy as np

_CACHE: dict = {}


def _tables(eng):
    key = id(eng)
    if key not in _CACHE:
        nt = len(eng.table("ibt", np.int32))
        D = eng.table("datantlin", np.float64).reshape(4, 4, nt)  # [comp][face][tet]
        length = np.sqrt((D[:3] ** 2).sum(0))
        normals = D / np.where(length > 0, length, 1.0)
        _CACHE[key] = dict(
            normals=normals,
            vt=eng.table("vt", np.float64).reshape(nt, 4),
            tet=eng.table("tet", np.int32).reshape(4, nt),
            knode=np.stack([eng.table(n, np.float64) for n in ("xkk", "ykk", "zkk")], axis=1),
            matsym=eng.table("matsym", np.int32).reshape(6, 48),
            ibt=eng.table("ibt", np.int32))
    return _CACHE[key]


def in_wedge(matsym, isym, kx, ky, kz):
    p0 = matsym[0, isym] - 1
    p1 = matsym[1, isym] - 1
    a, b, c = kx * matsym[3, isym], ky * matsym[4, isym], kz * matsym[5, isym]
    xo = np.where(p0 == 0, a, np.where(p1 == 0, b, c))
    yo = np.where(p0 == 1, a, np.where(p1 == 1, b, c))
    zo = np.where(p0 == 2, a, np.where(p1 == 2, b, c))
    return xo, yo, zo


def consistency(eng, p: dict) -> dict:
    """Worst-case and typical violations over the store `p` (Engine.download())."""
    t = _tables(eng)
    it, isym = p["itet"], p["isym"]
    a, b, c = in_wedge(t["matsym"], isym, p["kx"], p["ky"], p["kz"])
    n = t["normals"][:, :, it]  # [comp][face][particle]
    dist = n[0] * a + n[1] * b + n[2] * c - n[3]  # [face][particle], >= 0 inside
    outside = np.maximum(-dist.min(axis=0), 0.0)
    k0 = t["knode"][t["tet"][0, it]]
    v = t["vt"][it]
    e_band = v[:, 3] + v[:, 0] * (a - k0[:, 0]) + v[:, 1] * (b - k0[:, 1]) + v[:, 2] * (c - k0[:, 2])
    de = np.abs(p["energy"] - e_band)
    m = eng.mesh
    pos_out = 0.0
    for axis, nodes, idx in (("x", m.lx, p["i"]), ("y", m.ly, p["j"]), ("z", m.lz, p["k"])):
        lo, hi = nodes[idx], nodes[idx + 1]
        pos_out = np.maximum(pos_out, np.maximum(lo - p[axis], p[axis] - hi))
    band_ok = bool(np.all(t["ibt"][it] >= 0))
    return {
        "k_outside_max": float(outside.max()) if len(it) else 0.0,
        "k_outside_frac_1e-4": float((outside > 1e-4).mean()) if len(it) else 0.0,
        "energy_err_max": float(de.max()) if len(it) else 0.0,
        "energy_err_rms": float(np.sqrt((de ** 2).mean())) if len(it) else 0.0,
        "energy_err_rel_max": float((de / np.maximum(np.abs(p["energy"]), 1e-3)).max()) if len(it) else 0.0,
        "position_outside_max": float(np.max(pos_out)) if len(it) else 0.0,
        "band_ok": band_ok,
    }
