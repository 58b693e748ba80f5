"""Host side of the per-N-bucket autotuner (molscat_b200/autotune.py): the
committed B200 tables are well formed and self-consistent, and applying them
only records kernel-family overrides in the library (no device call), so this
runs without a GPU."""
import json
import os

import pytest

from molscat_b200 import _lib, autotune

PROPS = ("LDMD", "LDJ")


@pytest.fixture(scope="module")
def lib():
    from molscat_b200.build import build
    build()
    L = _lib.load()
    yield L
    _lib.set_family_for_n(-1, -1, -1)  # leave no overrides behind


@pytest.mark.parametrize("prop", PROPS)
def test_committed_table_is_consistent(prop):
    path = autotune.default_path(prop)
    assert os.path.exists(path), path
    with open(path) as f:
        t = json.load(f)
    assert t["prop"] == prop
    assert [(r["lo"], r["hi"]) for r in t["ranges"]] == list(autotune.RANGES)
    for r in t["ranges"]:
        cands = autotune.candidates(r["hi"], prop)
        measured = {int(k): v for k, v in r["tflops"].items()}
        assert r["family"] in cands, r
        assert set(measured) <= set(cands), r
        # the tuner keeps the fastest family it measured for the range
        assert r["family"] == max(measured, key=measured.get), r


@pytest.mark.parametrize("prop", PROPS)
def test_apply_records_overrides_without_a_device(lib, prop):
    path = autotune.default_path(prop)
    with open(path) as f:
        t = json.load(f)
    expected = sum(1 for r in t["ranges"] if r["family"] != _lib.FAMILY_DMMA)
    assert autotune.apply(path) == expected
    _lib.set_family_for_n(-1, -1, -1, prop)


def test_family_override_arguments_are_checked(lib):
    with pytest.raises(ValueError):
        _lib.set_family_for_n(10, 5, _lib.FAMILY_BIG)       # empty range
    with pytest.raises(ValueError):
        _lib.set_family_for_n(1, 8, 3)                      # no such family
    with pytest.raises(ValueError):
        _lib.set_family_for_n(0, 8, _lib.FAMILY_DMMA)       # N starts at 1
    _lib.set_family_for_n(41, 64, _lib.FAMILY_TILE4, "LDMD")
    _lib.set_family_for_n(-1, -1, -1, "LDMD")               # clearing always succeeds
