"""CPU: the oracle's and the library's tables against the golden file
generated from the reference's sources (tests/golden/make_golden.py)."""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from oracle.fd_oracle import template

GOLDEN = json.loads((Path(__file__).parent / "golden" / "templates.json").read_text())["templates"]
RED = json.loads((Path(__file__).parent / "golden" / "templates.json").read_text())["reduction_known_answers"]


def library_lattice(q):
    from asl_b200 import _lib as L
    lib = L.load()
    c, w, inv = (C.c_int * (3 * q))(), (C.c_double * q)(), (C.c_int * q)()
    L.check(lib.aslb_lattice(q, c, w, inv), "aslb_lattice")
    return np.array(c[:]).reshape(q, 3), np.array(w[:]), np.array(inv[:])


@pytest.mark.parametrize("q", [15, 19, 27])
def test_velocity_sets_match_reference_tables(oracle_mod, q):
    want = np.array(GOLDEN["d3q%d" % q]["vectors"])
    for c, w, inv in (oracle_mod.lattice(q), library_lattice(q)):
        assert np.array_equal(c, want)
        assert np.array_equal(c[inv], -c)  # opposite-direction table
        if q != 27:  # weights = LC / 6 + [i == 0] (aslTemplates.cxx:55-68)
            lc = np.array(GOLDEN["d3q%d" % q]["lc"])
            assert np.allclose(w, lc / 6 + (np.arange(q) == 0), rtol=0, atol=1e-15)
        else:  # the reference's d3q27 has no coefficients: standard weights
            assert "lc" not in GOLDEN["d3q27"]
            assert abs(w.sum() - 1) < 1e-15 and abs(w[0] - 8 / 27) < 1e-15


@pytest.mark.parametrize("q", [7, 15, 19])
def test_fd_templates_match_reference_tables(oracle_mod, q):
    e, lc, gc = template(q)
    ref = GOLDEN["d3q%d" % q]
    assert np.array_equal(e, np.array(ref["vectors"]))
    assert np.allclose(lc, ref["lc"], rtol=0, atol=1e-15)
    assert np.allclose(gc, ref["gc"], rtol=0, atol=1e-15)


def test_reduction_known_answers_from_reference(oracle_mod):
    assert [r["sum"] for r in RED] == [202.0, 600006.0]
    for r in RED:
        factor = r["sum"] / r["n"]
        assert oracle_mod.load().orc_sum((C.c_double * r["n"])(*([factor] * r["n"])), r["n"]) == r["sum"]
