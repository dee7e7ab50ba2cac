"""The C ABI library loads without a GPU and exports every entry point its
public headers declare (no compute calls here)."""
import ctypes
import os
import re

import mcb200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h") or h == "mcb200_rng.h":  # the RNG header is inline-only
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(mcb200_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(mcb200.LIB_PATH)
    names = declared_functions()
    assert {"mcb200_create", "mcb200_step", "mcb200_destroy"} <= names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_context_builds_tables(oracle_tables):
    eng = mcb200.Engine(table_dir=oracle_tables, device=-1, max_particles=1)
    assert eng.table("gamtet", float).size == 55320
    try:
        eng.set_mesh([0, 1], [0, 1], [0, 1])
        raised = False
    except mcb200.EngineError:
        raised = True
    assert raised, "a host-only context must refuse device work"
    eng.close()


def test_bad_table_dir_reports_io_error():
    try:
        mcb200.Engine(table_dir="/nonexistent", device=-1, max_particles=1)
    except mcb200.EngineError as e:
        assert "cannot open" in str(e)
    else:
        raise AssertionError("expected an error")
