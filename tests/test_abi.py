"""The C ABI library loads, exports every symbol include/necsim_b200.h
declares, and its host-only entry points agree with the oracle (CPU)."""
import os
import re

import numpy as np


def declared_symbols():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    names = set()
    for fn in os.listdir(os.path.join(root, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(root, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(necsim_\w+)\s*\(", text, re.M))
    return names


def test_exports_every_declared_symbol(nb):
    L = nb.lib()
    decl = declared_symbols()
    assert {"necsim_gpu_create", "necsim_gpu_simulate", "necsim_gpu_simulate_batch"} <= decl
    for name in decl:
        assert hasattr(L, name), name
    assert set(nb.SYMBOLS) <= decl


def test_seed_from_u64_matches_oracle(nb, oracle, kat):
    for s, v in kat["seed_from_u64"].items():
        assert nb.seed_from_u64(int(s)) == v == oracle.seed_from_u64(int(s))


def test_origins_match_oracle(nb, oracle, syn, kat):
    hab = syn.habitat_map(9, 7, 0.3, 4, 8)
    descs = [dict(kind=0, speciation_probability=0.1, width=7, height=3, deme=4),
             dict(kind=1, speciation_probability=0.1, width=11, height=2, deme=3, meta_width=50,
                  meta_height=2, meta_deme=2, migration_probability=0.2),
             dict(kind=2, speciation_probability=0.1, sigma=2.0, radius=9, centre_x=5,
                  centre_y=0xFFFFFFFF - 3),
             dict(kind=3, speciation_probability=0.1, width=9, height=7, habitat=hab,
                  dispersal=syn.dispersal_map(hab, 1.0))]
    for d in descs:
        a = nb.enumerate_origins(syn.to_scenario(d))
        b = oracle.enumerate_origins(d)
        for f in ("gref", "x", "y", "index"):
            assert np.array_equal(a[f], b[f]), (d["kind"], f)
    for case in kat["circle_origins"]:
        sc = nb.AlmostInfinite(nb.Circle(case["radius"], tuple(case["centre"])), nb.Normal(1.0))
        o = nb.enumerate_origins(sc)
        assert [[int(x), int(y)] for x, y in zip(o["x"], o["y"])] == case["locations"]


def test_invalid_arguments_fail_cleanly(nb):
    import pytest
    with pytest.raises(nb.NecsimError) as e:
        nb.Simulation(nb.NonSpatial((0, 5), 1), 0.1)
    assert e.value.code == -1
    with pytest.raises(nb.NecsimError):
        nb.Simulation(nb.NonSpatial((5, 5), 1), 0.0)
    with pytest.raises(nb.NecsimError):
        nb.Simulation(nb.SpatiallyImplicit((5, 1), 1, (10, 1), 1, 0.0), 0.1)


def test_scenario_layout_matches_ctypes_mirrors(nb, oracle, tmp_path):
    """necsim_scenario (include/necsim_b200.h) and oracle_scenario have the
    field offsets of the package's and the oracle's ctypes structures."""
    import ctypes
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    fields = [f[0] for f in nb.CScenario._fields_]
    ofields = [f[0] for f in oracle.OracleScenario._fields_]
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "include/necsim_b200.h"',
           '#include "oracle/necsim_oracle.h"', 'int main(void) {',
           '  printf("%zu %zu\\n", sizeof(necsim_scenario), sizeof(oracle_scenario));']
    src += ['  printf("%%zu\\n", offsetof(necsim_scenario, %s));' % f for f in fields]
    src += ['  printf("%%zu\\n", offsetof(oracle_scenario, %s));' % f for f in ofields]
    src += ['  return 0;', '}']
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", root, "-o", str(exe), str(c)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert [int(v) for v in out[:2]] == [ctypes.sizeof(nb.CScenario), ctypes.sizeof(oracle.OracleScenario)]
    got = [int(v) for v in out[2:]]
    assert got[:len(fields)] == [getattr(nb.CScenario, f).offset for f in fields]
    assert got[len(fields):] == [getattr(oracle.OracleScenario, f).offset for f in ofields]
