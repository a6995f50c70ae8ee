""".xyz volume files (CloudData::loadFromXyzFile, CloudData.cpp:236-317): header of three u32 grid sizes
and three f64 voxel sizes, then the values with z fastest; the loader transposes them to x fastest and
applies the min-max normalisation whose minimum starts at 0 (sgl::reduceFloatArrayMinMax with the
initial pair (0, lowest)).  The expected grids are restated here with plain loops."""
import struct

import numpy as np
import pytest

from cloudrendering_b200 import vpt


def write_xyz(path, values_zfast, sizes, voxel=(1.0, 1.0, 1.0)):
    xs, ys, zs = sizes
    with open(path, "wb") as f:
        f.write(struct.pack("<3I", xs, ys, zs))
        f.write(struct.pack("<3d", *voxel))
        f.write(np.asarray(values_zfast, "<f4").tobytes())


def reference_grid(file_values, sizes):
    """The loader's loops: densityFieldFloat[x + (y + z * Y) * X] = file[z + (y + x * Y) * Z], then
    (v - min) / (max - min) with min <= 0 when max - min > 1e-6."""
    xs, ys, zs = sizes
    out = np.empty(xs * ys * zs, np.float32)
    for z in range(zs):
        for y in range(ys):
            for x in range(xs):
                out[x + (y + z * ys) * xs] = file_values[z + (y + x * ys) * zs]
    lo = np.float32(min(0.0, float(out.min())))
    hi = np.float32(out.max())
    if hi - lo > np.float32(1e-6):
        out = (out - lo) / (hi - lo)
    return out.reshape(zs, ys, xs)


@pytest.mark.parametrize("sizes,offset", [((5, 3, 4), 0.0), ((2, 7, 3), 0.5), ((4, 4, 4), -2.0)])
def test_xyz_values_transposed_and_normalised(tmp_path, sizes, offset):
    rng = np.random.default_rng(sum(sizes))
    n = int(np.prod(sizes))
    values = (rng.random(n).astype(np.float32) * 3.0 + np.float32(offset)).astype(np.float32)
    path = str(tmp_path / "grid.xyz")
    write_xyz(path, values, sizes, voxel=(0.5, 0.25, 2.0))
    got = vpt._read_xyz(path)
    want = reference_grid(values, sizes)
    assert got.shape == want.shape and got.dtype == np.float32
    assert np.array_equal(got, want)


def test_xyz_constant_grid_is_not_normalised(tmp_path):
    sizes = (3, 3, 3)
    path = str(tmp_path / "const.xyz")
    write_xyz(path, np.zeros(27, np.float32), sizes)
    assert np.array_equal(vpt._read_xyz(path), np.zeros((3, 3, 3), np.float32))


def test_xyz_header_voxel_sizes(tmp_path):
    path = str(tmp_path / "vox.xyz")
    write_xyz(path, np.arange(8, dtype=np.float32), (2, 2, 2), voxel=(0.5, 0.25, 2.0))
    with open(path, "rb") as f:
        assert struct.unpack_from("<3d", f.read(36), 12) == (0.5, 0.25, 2.0)
