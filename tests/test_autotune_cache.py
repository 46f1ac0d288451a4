"""Autotuner cache (host logic only, no GPU): a stored choice is found again
under its key, other keys and unreadable files give no hit, and a cache hit
is applied to the solver without timing anything."""
import importlib
import json

import pytest


@pytest.fixture()
def at(monkeypatch, tmp_path):
    mod = importlib.import_module("geos-chem-gpu-hybrid_b200.autotune")
    monkeypatch.setenv("GCCHEM_B200_TUNE_CACHE", str(tmp_path / "sub" / "autotune.json"))
    monkeypatch.setattr(mod, "_key",
                        lambda solver, tag="default": f"B200|{solver.mech}|{solver.variant}|{tag}")
    return mod


class _FakeSolver:
    def __init__(self, mech="fullchem", variant="fma"):
        self.mech, self.variant = mech, variant
        self.launch = None
        self.chunk = None

    def set_launch(self, mode, threads, blocks_per_sm):
        self.launch = (mode, threads, blocks_per_sm)

    def set_chunk(self, cells):
        self.chunk = cells

    def set_row_scratch(self, shared):
        self.shared = shared


def test_store_and_reload(at):
    s = _FakeSolver()
    assert at.load_cached(s) is None
    entry = {"mode": "persistent", "threads": 256, "blocks_per_sm": 0, "cells_per_s": 1.0}
    at._store(s, entry)
    assert at.load_cached(s) == entry
    assert at.load_cached(_FakeSolver(variant="nofma")) is None
    at._store(_FakeSolver(variant="nofma"), dict(entry, threads=64))
    assert at.load_cached(s)["threads"] == 256
    assert at.load_cached(_FakeSolver(variant="nofma"))["threads"] == 64


def test_unreadable_cache_is_a_miss(at):
    s = _FakeSolver()
    at._store(s, {"mode": "plain", "threads": 128, "blocks_per_sm": 0})
    with open(at.cache_path(), "w") as fh:
        fh.write("{not json")
    assert at.load_cached(s) is None


def test_cache_hit_is_applied_without_timing(at, pkg):
    s = _FakeSolver()
    at._store(s, {"mode": "plain", "threads": 64, "blocks_per_sm": 0, "cells_per_s": 5.0})
    got = at.tune(s, batch=None)
    assert got["cached"] is True
    assert s.launch == (pkg.PLAIN, 64, 0)
    assert s.chunk == 0
    with open(at.cache_path()) as fh:
        assert json.load(fh)["B200|fullchem|fma|default"]["threads"] == 64


def test_chunked_candidates_keep_their_own_entry(at, pkg):
    """The large-grid candidate set (layout and chunk size) is cached under
    its own tag, and a hit sets the chunk size too."""
    s = _FakeSolver()
    at._store(s, {"mode": "plain_fused", "threads": 128, "blocks_per_sm": 0,
                  "chunk": 131072, "cells_per_s": 9.0}, "chunked")
    assert at.load_cached(s) is None
    got = at.tune(s, batch=None, candidates=at.CHUNKED, tag="chunked")
    assert got["cached"] is True
    assert s.launch == (pkg.PLAIN_FUSED, 128, 0) and s.chunk == 131072
    assert {c[3] for c in at.CHUNKED} >= {0, 32768, 65536, 131072}
    assert s.shared is False


def test_persistent_kernel_preferred_at_near_equal_speed(at):
    """A plain candidate must beat the persistent kernel by PREFER_PERSISTENT."""
    p = {"mode": "persistent", "cells_per_s": 100.0}
    assert at._score({"mode": "plain_fused", "cells_per_s": 104.0}) < at._score(p)
    assert at._score({"mode": "plain_fused", "cells_per_s": 106.0}) > at._score(p)
    assert {c[4] for c in at.CANDIDATES} == {"global", "shared"}
