"""libhns.so loads, exports every entry point its headers declare, and rejects bad
arguments with status codes; none of these tests launches a kernel."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from hnanosolver_b200 import lib as hl
from hnanosolver_b200 import synth


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    return set(re.findall(r"HNS_API\s+[\w\s\*]+?\b(hns_\w+)\s*\(", src))


def test_library_exports_every_declared_symbol():
    names = declared("hns.h")
    assert len(names) > 20
    lib = ctypes.CDLL(hl.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_status_strings():
    assert hl.lib.hns_abi_version() == 1
    assert hl.lib.hns_status_string(0) == b"ok"
    assert hl.lib.hns_status_string(5) == b"invalid leaf layout"


def test_sort_leaves_matches_oracle(oracle):
    rng = np.random.default_rng(4)
    o = np.unique(rng.integers(-9000, 9000, size=(500, 3)) // 8 * 8, axis=0).astype(np.int32)
    rng.shuffle(o)
    assert np.array_equal(hl.sort_leaves_nanovdb(o), oracle.sort_leaves(o))
    assert np.array_equal(hl.sort_leaves_nanovdb(o), synth.sort_leaves_nanovdb(o))


def test_null_arguments_are_rejected():
    h = ctypes.c_void_p()
    assert hl.lib.hns_create(None, None, 0, 1.0, 0) == 1
    assert hl.lib.hns_create(ctypes.byref(h), None, 1, 1.0, 0) == 1
    assert b"null" in hl.lib.hns_last_error()
    assert hl.lib.hns_destroy(None) == 0
    assert hl.lib.hns_advect_vec3(None, None, None, 0.1) == 1
    assert hl.lib.hns_num_voxels(None) == 0


def test_non_leaf_dense_coordinates_are_a_layout_error():
    coords = synth.leaf_dense_coords(np.array([[0, 0, 0]], np.int32)).copy()
    coords[[3, 4]] = coords[[4, 3]]
    with pytest.raises(hl.HnsError) as e:
        hl.Grid(coords=coords, voxel_size=0.1)
    assert e.value.status == 5
    with pytest.raises(hl.HnsError) as e:
        hl.Grid(coords=coords[:100], voxel_size=0.1)
    assert e.value.status == 5


def test_bad_voxel_size_is_rejected():
    with pytest.raises(hl.HnsError) as e:
        hl.Grid(np.zeros((1, 3), np.int32), voxel_size=0.0)
    assert e.value.status == 1


def test_python_constants_mirror_the_header():
    """Every option, option value and solve flag the header defines has the same value in the
    Python binding (HNS_OPT_X -> OPT_X, HNS_SOLVE_X -> SOLVE_X, value names without the prefix)."""
    src = open(os.path.join(ROOT, "include", "hns.h")).read()
    defs = dict((m.group(1), int(m.group(2))) for m in
                re.finditer(r"^#define HNS_((?:OPT|RBGS|INNER|SPLIT|COARSE|SOLVE)_\w+)\s+(\d+)u?\b", src, re.M))
    assert "OPT_COARSE_SOLVE" in defs and "OPT_L2_PERSIST" in defs and "SOLVE_MULTIGRID" in defs
    for name, value in defs.items():
        assert getattr(hl, name) == value, name


def test_set_option_without_a_context_is_rejected():
    for opt in (hl.OPT_RBGS_KERNEL, hl.OPT_INNER_LAYOUT, hl.OPT_WAIT_POLLS, hl.OPT_SPLIT_SOLVE,
                hl.OPT_COARSE_SOLVE, hl.OPT_L2_PERSIST):
        assert hl.lib.hns_set_option(None, opt, 0) == 1
