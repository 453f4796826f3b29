"""CPU tests of the C ABI library: it loads, exports every entry point the
header declares, derives the reference's displacement tables, and fails loudly
(no CPU fallback) where no CUDA device is present. No kernel runs here."""
import json
import os
import re

import numpy as np
import pytest

import pyro_cmc_b200 as pc
from pyro_cmc_b200 import _lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(REPO, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(REPO, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(pc_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    names = declared_symbols()
    assert len(names) > 40
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert declared_symbols() <= set(_lib._SIGNATURES)


def test_version():
    assert _lib.lib().pc_version() >= 100


def test_displacement_tables_match_reference_tables(golden_dir):
    g = json.load(open(os.path.join(golden_dir, "geometry_tables.json")))
    for kind, name in ((1, "nn1_dist"), (2, "nn2_dist"), (3, "nn3a_dist"), (4, "nn3b_dist")):
        for p in range(4):
            got = pc.displacements(kind, p)
            assert len(got) == len(g[name][p])
            assert sorted(map(tuple, got.tolist())) == sorted(map(tuple, g[name][p]))
    for mu, nu in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)):
        t = g["nn1_pair_%d%d" % (mu, nu)]
        assert sorted(map(tuple, pc.displacements(10 + nu, mu).tolist())) == sorted(map(tuple, t[mu]))
        assert sorted(map(tuple, pc.displacements(10 + mu, nu).tolist())) == sorted(map(tuple, t[nu]))


def test_sublattice_offsets_match_reference_cell(golden_dir):
    g = json.load(open(os.path.join(golden_dir, "geometry_tables.json")))
    r = pc.sublattice_offsets()
    for sl in range(16):
        f, p = divmod(sl, 4)
        assert (r[sl] == np.array(g["PyroCubicCell_R_fcc"][f]) + np.array(g["PyroCubicCell_link_positions"][p])).all()


def test_displacement_errors_are_invalid_argument():
    with pytest.raises(pc.InvalidArgument):
        pc.displacements(7, 0)
    with pytest.raises(pc.InvalidArgument):
        pc.displacements(1, 4)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure mode")
def test_no_gpu_fails_loudly():
    with pytest.raises(pc.PyroCMCError) as e:
        pc.System(2)
    assert e.value.code == _lib.ERR_CUDA
