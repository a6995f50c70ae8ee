"""The oracle's supervoxel builders against the reference's own (SuperVoxelGrid.cpp and
DensityField.cpp compiled unmodified; fixture tests/golden/supervoxel_grids.npz): normalisation by
getDataFloatAtNorm, per-supervoxel min / max (one-voxel halo unless nearest, zero border),
occupancy, and the residual ratio tracking controls (mu_c, mu_r_bar) - all bit for bit."""
import numpy as np
import pytest

from oracle import bridge
from tests.harness import supervoxel_golden, supervoxel_size

GOLD = supervoxel_golden()


@pytest.mark.parametrize("key", sorted(GOLD))
def test_oracle_supervoxels_match_reference(key):
    g = GOLD[key]
    raw = g["raw"]
    nz, ny, nx = raw.shape
    sv = supervoxel_size(nx, ny, nz)
    assert [-(-nx // sv), -(-ny // sv), -(-nz // sv), sv] == g["dims"]
    vmin, vmax = bridge.minmax(raw)
    dens = bridge.normalize(raw, vmin, vmax)
    mn, mx, avg, occ = bridge.supervoxel_stats(dens, sv, 0 if g["interp"] == 0 else 1)
    assert np.array_equal(mn.view(np.uint32), g["minmax"][0::2].view(np.uint32))
    assert np.array_equal(mx.view(np.uint32), g["minmax"][1::2].view(np.uint32))
    assert np.array_equal(occ, g["occ_decomposition"])
    assert np.array_equal(occ, g["occ_rrt"])
    pairs = bridge.rrt_params(mn, mx, avg, g["extinction"], sv)
    assert np.array_equal(pairs.view(np.uint32), g["rrt"].view(np.uint32))
