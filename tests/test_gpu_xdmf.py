"""Mesh::Save and the XDMF writers (src/base/Mesh.cpp:366-489,
src/base/Utils.cpp:53-229) with raw binary in place of HDF5
(se_mesh_save, se_write_xdmf_*): the mesh file's layout and connectivity,
and XDMF files whose Binary DataItems (file, byte offset, dimensions) lead
to the mesh's and the fields' values."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def read_binary_item(item, base):
    """The array a Binary DataItem of these files names."""
    dims = [int(d) for d in item.get("Dimensions").split()]
    dtype = "<f8" if item.get("NumberType") == "Float" else "<i4"
    assert item.get("Format") == "Binary" and item.get("Endian") == "Little"
    with open(base / item.text.strip(), "rb") as f:
        f.seek(int(item.get("Seek")))
        return np.frombuffer(f.read(int(np.prod(dims)) * np.dtype(dtype).itemsize),
                             dtype).reshape(dims)


def slab_column(slab, base):
    """Column selected by a HyperSlab DataItem (start, stride, count)."""
    sel, data = list(slab)
    start = [int(v) for v in sel.text.split()[:2]]
    return read_binary_item(data, base)[:, start[1]]


def test_mesh_save_layout(segpu, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    m = segpu.Mesh("mesh", [4, 3], "legendre", 5, [-1.0, 0.0], [1.0, 1.5], [True, False])
    m.Save()
    raw = (tmp_path / "mesh.seb").read_bytes()
    assert raw[:8] == b"SEMESH01"
    dims = np.frombuffer(raw[8:16], "<i4")
    res = np.frombuffer(raw[16:24], "<i4")
    mn, mx = np.frombuffer(raw[24:40], "<f8"), np.frombuffer(raw[40:56], "<f8")
    nv, nq = np.frombuffer(raw[56:72], "<i8")
    assert dims[0] == 2 and list(res) == [20, 15]
    assert list(mn) == [-1.0, 0.0] and list(mx) == [1.0, 1.5]
    assert nv == m.nVertsTotal and nq == 20 * 15
    verts = np.frombuffer(raw[72:72 + 16 * nv], "<f8").reshape(nv, 2)
    assert np.array_equal(verts, m.verts)
    conn = np.frombuffer(raw[72 + 16 * nv:], "<i4").reshape(nq, 4)
    e = np.arange(nq)
    first = e + e // 20  # Mesh::Save's linear quads
    want = np.stack([first, first + 1, first + 1 + m.nVerts[0], first + m.nVerts[0]], 1)
    assert np.array_equal(conn, want)


def test_xdmf_files_reference_the_data(segpu, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    m = segpu.Mesh("vMesh", [5, 4], "legendre", 4, [0.0, 0.0], [2.0, 1.0], [True, False])
    m.Save()
    rng = np.random.default_rng(3)
    phi = segpu.Field("phi", m, 1, None)
    vel = segpu.Field("velocity", m, 2, None)
    phi.vals = rng.standard_normal(m.nVertsTotal)
    vel.vals = rng.standard_normal((m.nVertsTotal, 2))
    segpu.WriteXDMFHeader(7)
    segpu.WriteXDMF([phi, vel], 2, 7, 0.35, 0.05)
    segpu.WriteXDMFFooter(7)
    segpu.WriteXDMFTemporal(10, 7)
    assert (tmp_path / "time.00007.ts").read_text() == "time step:\t7\ttime:\t0.35\tdt:\t0.05\n"
    root = ET.parse(tmp_path / "XDMF.00007.xmf").getroot()
    grid = root.find("Domain/Grid")
    assert grid.get("Name") == "FEM_Grid_vMesh"
    assert grid.find("Time").get("Value") == "0.35"
    topo = grid.find("Topology")
    nq = (m.nVerts[0] - 1) * (m.nVerts[1] - 1)
    assert topo.get("NumberOfElements") == str(nq)
    conn = read_binary_item(topo.find("DataItem"), tmp_path)
    assert conn.shape == (nq, 4) and conn[0, 0] == 0 and conn[0, 2] == m.nVerts[0] + 1
    xy = [slab_column(s, tmp_path) for s in grid.find("Geometry/DataItem")]
    assert np.array_equal(np.stack(xy, 1), m.verts)
    attrs = {a.get("Name"): a for a in grid.findall("Attribute")}
    assert attrs["phi"].get("Type") == "Scalar"
    assert np.array_equal(slab_column(attrs["phi"].find("DataItem"), tmp_path), phi.vals)
    assert attrs["velocity"].get("Type") == "Vector"
    uv = [slab_column(s, tmp_path) for s in attrs["velocity"].find("DataItem")]
    assert np.array_equal(np.stack(uv, 1), vel.vals)
    files = ET.parse(tmp_path / "XDMF.FilesField.xdmf").getroot()
    hrefs = [e.get("href") for e in files.iter() if e.get("href")]
    assert hrefs == ["XDMF.00000.xmf", "XDMF.00007.xmf"]
    for f in ("XDMF.temporalAll.xmf", "XDMF.temporalFields.xmf"):
        ET.parse(tmp_path / f)  # well-formed
    with pytest.raises(segpu.SEError):
        segpu.WriteXDMFTemporal(10, 0)
