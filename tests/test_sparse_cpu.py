"""Pins the oracle's restatement of PNanoVDB (oracle/vpt_oracle.cpp, `Nano` and the HDDA) to the
reference's own NanoVDB code: tests/golden/sparse_grids.npz holds NanoVDB buffers built by the
reference's GridBuilder from the fixture grids, and the reference accessor's and HDDA's outputs on
them (tests/golden/make_sparse_golden.py).  Integer traversal results are compared bit for bit."""
import numpy as np
import pytest

from oracle import bridge
from tests.harness import SPARSE_GRIDS, sparse_golden

GOLD = sparse_golden()


@pytest.mark.parametrize("name", SPARSE_GRIDS)
def test_oracle_accessor_matches_reference(name):
    g = GOLD[name]
    val, dim, act = bridge.nanovdb_query(g["buf"], g["ijk"])
    assert np.array_equal(val.view(np.uint32), g["value"].view(np.uint32))
    assert np.array_equal(dim, g["dim"])
    assert np.array_equal(act, g["active"])


@pytest.mark.parametrize("name", SPARSE_GRIDS)
def test_oracle_hdda_walk_matches_reference(name):
    g = GOLD[name]
    assert len(g["walks"]) > 40
    for origin, direction, lowest, ref in g["walks"]:
        got = bridge.nanovdb_hdda_walk(g["buf"], origin, direction, lowest)
        assert got is not None
        for f in ("voxel", "dim", "active", "box", "t"):
            a, b = got[f], ref[f]
            assert a.shape == b.shape, (f, a.shape, b.shape)
            if a.dtype == np.float32:
                assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f
            else:
                assert np.array_equal(a, b), f
        # node level as the tracker sees it (only meaningful for active cells)
        assert np.array_equal(np.where(got["active"] == 1, got["level"], 0), np.where(ref["active"] == 1, ref["level"], 0))


def test_fixture_covers_every_node_kind():
    """Leaves, lower-node tiles (8), upper-node tiles (128) and the background (4096) all occur, and
    some cells classify as active tiles, so every branch of the accessor and the HDDA is exercised."""
    dims = np.concatenate([GOLD[n]["dim"] for n in SPARSE_GRIDS])
    assert set(np.unique(dims)) >= {1, 8, 128, 4096}
    levels = np.concatenate([w["level"][w["active"] == 1] for n in SPARSE_GRIDS for (_, _, lv, w) in GOLD[n]["walks"]
                             if lv == 8])
    assert {0, 1, 2} <= set(np.unique(levels))
