"""The engine's host-built full-band tables against the reference's own
Band::IELEC (run inside the CPU oracle): bit-exact, table by table."""
import numpy as np
import pytest

import mcb200
from oracle_bridge import Oracle

# (engine name, oracle name, dtype, how to cut the oracle's fixed-size array)
NT_TABLES = ["gamtet", "vgt", "faclow", "facmedium", "fachigh"]


@pytest.fixture(scope="module")
def pair(oracle_tables):
    orc = Oracle()
    orc.build_band_only(300.0)
    eng = mcb200.Engine(table_dir=oracle_tables, kelvin=300.0, device=-1, max_particles=1)
    yield orc, eng
    eng.close()


def same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    assert a.dtype == b.dtype
    if a.dtype.kind == "f":
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), f"{np.sum(a != b)} entries differ"
    else:
        assert np.array_equal(a, b), f"{np.sum(a != b)} entries differ"


def test_sizes(pair):
    orc, eng = pair
    assert len(eng.table("gamtet", np.float64)) == int(orc.band_scalar("nt")) == 55320
    assert len(eng.table("xkk", np.float64)) == int(orc.band_scalar("nk")) == 12619


@pytest.mark.parametrize("name", NT_TABLES)
def test_per_tet(pair, name):
    orc, eng = pair
    nt = int(orc.band_scalar("nt"))
    same(eng.table(name, np.float64), orc.band(name)[:nt])


def test_kgrid_and_topology(pair):
    orc, eng = pair
    nk, nt = int(orc.band_scalar("nk")), int(orc.band_scalar("nt"))
    for n in ("xkk", "ykk", "zkk", "eek"):
        same(eng.table(n, np.float64), orc.band(n)[:nk])
    same(eng.table("tet", np.int32).reshape(4, nt), orc.band("tet")[:, :nt])
    same(eng.table("NeibrTet", np.int32).reshape(4, nt), orc.band("NeibrTet")[:, :nt])
    same(eng.table("ibt", np.int32), orc.band("ibt")[:nt])
    same(eng.table("vt", np.float64), orc.band("vt")[:4 * nt])
    same(eng.table("datantlin", np.float64).reshape(4, 4, nt), orc.band("datantlin")[:, :, :nt])


def test_symmetry(pair):
    orc, eng = pair
    same(eng.table("matsym", np.int32).reshape(6, 48), orc.band("matsym"))
    same(eng.table("indmat", np.int32)[orc.band("indmat") != 0], orc.band("indmat")[orc.band("indmat") != 0])
    same(eng.table("newisym", np.int32).reshape(5, 48), orc.band("newisym"))
    for n in ("xbz", "ybz", "zbz"):
        same(eng.table(n, np.float64).reshape(5, 48), orc.band(n))


def test_tet_lists(pair):
    orc, eng = pair
    for n in ("ntlist", "ptlist", "nslist", "pslist"):
        same(eng.table(n, np.int32).reshape(325, 8), orc.band(n))
    for n in ("ntlists", "ptlists"):
        same(eng.table(n, np.int32).reshape(60, 8), orc.band(n))
    for n, cap in (("tlist", 470000), ("slist", 16000), ("tlists", 101000)):
        e = eng.table(n, np.int32)
        same(e, orc.band(n)[:len(e)])


def test_dos_and_rates(pair):
    orc, eng = pair
    same(eng.table("energy", np.float64), orc.band("energy"))
    same(eng.table("dos", np.float64).reshape(8, 7501), orc.band("dos"))
    same(eng.table("sumdos", np.float64).reshape(7501, 3), orc.band("sumdos"))
    same(eng.table("dostetmax", np.float64).reshape(8, 7501), orc.band("dostetmax"))
    same(eng.table("scatte", np.float64).reshape(14, 4, 4), orc.band("scatte"))
    same(eng.table("dose", np.float64).reshape(14, 4, 7501), orc.band("dose"))
    same(eng.table("scattiie", np.float64).reshape(4, 4, 7501), orc.band("scattiie"))
    same(eng.table("scatth", np.float64).reshape(4, 3, 3), orc.band("scatth"))
    same(eng.table("dosh", np.float64).reshape(4, 3, 7501), orc.band("dosh"))
    same(eng.table("scattiih", np.float64).reshape(3, 3, 7501), orc.band("scattiih"))
    same(eng.table("sumscatt", np.float64).reshape(7501, 8), orc.band("sumscatt"))


def test_units(pair):
    orc, eng = pair
    u = eng.units()
    for k, o in (("a0pi", "a0pi"), ("sieg", "sieg"), ("eV0", "eV0"), ("spr0", "spr0"), ("time0", "time0"),
                 ("conc0", "conc0"), ("field0", "field0"), ("eps_silicon", "eps_si"), ("scrt0", "scrt0")):
        assert u[k] == orc.scalar(o), k
