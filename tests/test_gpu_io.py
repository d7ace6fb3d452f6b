"""Field::Save / Field::Read in raw binary (se_field_save / se_field_read):
the file's layout, a bit-exact round trip through the GPU field, and the
refusals (another mesh or size, a missing or truncated file)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def read_raw(path):
    with open(path, "rb") as f:
        magic = f.read(8)
        dims = np.frombuffer(f.read(4), "<i4")[0]
        res = np.frombuffer(f.read(8), "<i4")
        rows = np.frombuffer(f.read(8), "<i8")[0]
        cols = np.frombuffer(f.read(4), "<i4")[0]
        data = np.frombuffer(f.read(), "<f8").reshape(rows, cols)
    return magic, dims, res, rows, cols, data


@pytest.mark.parametrize("ndofs", [1, 2])
def test_save_read_round_trip(segpu, tmp_path, ndofs):
    m = segpu.Mesh("m", [5, 3], "legendre", 4, [0, 0], [1, 1], [True, False])
    nv = 21 * 13
    vals = np.random.default_rng(ndofs).standard_normal((nv, ndofs))
    f = segpu.Field("phi", m, ndofs, None)
    f.vals = vals if ndofs == 2 else vals[:, 0]
    stem = str(tmp_path / "phi")
    f.Save(7, stem)
    path = stem + ".00007.seb"
    magic, dims, res, rows, cols, data = read_raw(path)
    assert magic == b"SEFIELD1" and dims == 2 and list(res) == [20, 12]
    assert rows == nv and cols == ndofs
    assert np.array_equal(data, vals)
    g = segpu.Field("phi", m, ndofs, None)
    g.Read(7, stem)
    got = g.vals.reshape(nv, ndofs)
    assert np.array_equal(got, vals)


def test_read_refuses_mismatches(segpu, tmp_path):
    m = segpu.Mesh("m", [5, 3], "legendre", 4, [0, 0], [1, 1], [True, False])
    f = segpu.Field("phi", m, 1, None)
    f.vals = np.arange(21 * 13, dtype=np.float64)
    stem = str(tmp_path / "phi")
    f.Save(0, stem)
    other = segpu.Mesh("o", [4, 3], "legendre", 4, [0, 0], [1, 1], [True, False])
    with pytest.raises(segpu.SEError):
        segpu.Field("phi", other, 1, None).Read(0, stem)
    with pytest.raises(segpu.SEError):
        segpu.Field("phi", m, 2, None).Read(0, stem)
    with pytest.raises(segpu.SEError):
        f.Read(1, stem)  # no such file
    path = stem + ".00000.seb"
    with open(path, "r+b") as fh:
        fh.truncate(os.path.getsize(path) - 8)
    with pytest.raises(segpu.SEError):
        f.Read(0, stem)
