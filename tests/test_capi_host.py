"""CPU checks of the C ABI: libdevil_b200.so loads, exports every entry point
include/devil_b200.h declares, and its host-side entry points (cluster
handling, mirroring R/main.R:190-196 and R/group_data.R:38-69) behave like
R's factor / is.unsorted / rle / order.  No GPU compute is called here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def header_symbols():
    text = open(os.path.join(ROOT, "include", "devil_b200.h")).read()
    return sorted(set(re.findall(r"DEVIL_API[^;(]*?\b(devil_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = header_symbols()
    assert "devil_fit" in syms and "devil_test_de" in syms and len(syms) >= 20


def test_library_exports_every_declared_symbol(dv):
    out = subprocess.run(["nm", "-D", "--defined-only", dv.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = [s for s in header_symbols() if s not in exported]
    assert not missing, missing
    from devil_b200._lib import EXPORTS
    assert set(EXPORTS) == set(header_symbols())


def test_ctypes_resolves_every_symbol(dv):
    L = dv.load_library()
    for s in header_symbols():
        assert getattr(L, s) is not None


def test_version_string(dv):
    assert b"sm_100a" in dv.load_library().devil_version()


def test_cluster_blocks_first_appearance(dv, orc):
    cl = np.array([7, 7, 3, 3, 3, 9, 9, 1])
    levels, ends = dv.cluster_blocks(cl)
    np.testing.assert_array_equal(levels, [1, 1, 2, 2, 2, 3, 3, 4])
    np.testing.assert_array_equal(ends, [2, 5, 7, 8])
    lev_o, nl = orc.factor_first_appearance(cl)
    np.testing.assert_array_equal(levels, lev_o)
    np.testing.assert_array_equal(ends, orc.cluster_blocks(lev_o))


def test_cluster_blocks_string_labels(dv):
    levels, ends = dv.cluster_blocks(np.array(["P2", "P2", "P1", "P1"]))
    np.testing.assert_array_equal(ends, [2, 4])


def test_cluster_blocks_unsorted_errors(dv):
    with pytest.raises(ValueError, match="grouped in blocks of patients"):
        dv.cluster_blocks(np.array([1, 2, 1]))


def test_group_data_order_is_stable_and_bit_exact(dv, orc):
    rng = np.random.default_rng(0)
    cl = rng.choice([5, 2, 8, 11], size=1000)
    Y = rng.poisson(3, (4, 1000)).astype(float)
    X = rng.normal(size=(1000, 2))
    g = dv.group_data(Y, X, cl)
    lev, nl = orc.factor_first_appearance(cl)
    ordr = orc.group_order(lev, nl)
    np.testing.assert_array_equal(g["input_matrix"], Y[:, ordr])
    np.testing.assert_array_equal(g["design_matrix"], X[ordr])
    np.testing.assert_array_equal(g["clusters"], lev[ordr].astype(float))
    # numpy's stable sort of the first-appearance codes gives the same order
    np.testing.assert_array_equal(ordr, np.argsort(lev, kind="stable"))
    # the grouped clusters are sorted, so fit_devil accepts them
    dv.cluster_blocks(g["clusters"])


def test_group_data_dimension_errors(dv):
    with pytest.raises(ValueError, match="ncol"):
        dv.group_data(np.zeros((2, 3)), np.zeros((4, 1)), [1, 1, 1])
    with pytest.raises(ValueError, match="length"):
        dv.group_data(np.zeros((2, 3)), np.zeros((3, 1)), [1, 1])


def test_argument_errors_before_gpu(dv):
    with pytest.raises(ValueError, match="Unknown overdispersion"):
        dv.api._od_mode("bogus")
    assert dv.api._od_mode("new") == dv.api._od_mode("I") == 3
    with pytest.raises(ValueError, match="should be one of"):
        dv.api._sf_mode("bogus", 3)
    with pytest.raises(RuntimeError, match="edgeR"):
        dv.api._sf_mode("edgeR", 3)
    with pytest.raises(ValueError, match="older version"):
        dv.test_de({"beta": np.zeros((2, 2))}, [0, 1])
    with pytest.raises(ValueError, match="precision must be one of"):
        dv.api._fit_opts("MOM", None, False, 0.0, 0, None, 200, 1e-3, False, "chosen", "fp16")
    opts = dv.api._fit_opts("MOM", None, False, 0.0, 0, None, 200, 1e-3, False, "chosen", "tc_tf32")
    assert opts.precision == 1 and opts.form == 0


def test_fit_opts_layout_matches_header():
    """The ctypes mirror of devil_fit_opts lists the header's fields in order."""
    import re
    from devil_b200 import _lib as L
    hdr = open(os.path.join(ROOT, "include", "devil_b200.h")).read()
    body = hdr[hdr.index("typedef struct devil_fit_opts {"):hdr.index("} devil_fit_opts;")]
    fields = re.findall(r"^\s+(?:const\s+)?\w+\s*\*?\s*(\w+);", body, re.M)
    assert fields == [f for f, _ in L.FitOpts._fields_]


def test_null_context_is_an_error_not_a_crash(dv):
    L = dv.load_library()
    assert L.devil_ctx_synchronize(None) != 0
    assert L.devil_fit(None, None, None, 0, None, 0, None, None) != 0
    n = C.c_int(0)
    assert L.devil_cluster_blocks(-1, None, None, None, C.byref(n)) != 0
