"""Field output in the VTK XML parallel structured-grid format (row f4).

The reference's io::VTKWriter<Cartesian<Dim>> (IO/VTKWriter.inl:34-86,
Grid/Cartesian/VTKOptions_Cartesian.h:146-323, IO/VTKPXMLStructuredGridWriter.cpp:32-45)
writes, for one grid on one rank, <base>/<grid>_<step>.pvts and one piece in
the subdirectory <grid>_<step>/: the ghosted local grid (extent 0 .. n + 2g
per active dimension, a one-cell-high pseudo-2-D grid for 1-D), Float32 node
coordinates x_i = dx i - g dx, one Float64 cell array per field in VTK's
x-fastest order, and "TimeValue" when time >= 0.  Its own test
(IO/test/test_VTKWriter.cpp) only checks that Write returns true; these tests
decode the files and check every item above.  They need no GPU (the host-array
entry point writes the same files as the device one).
"""
import base64
import os
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import dare_b200 as D


def _decode(text, dtype):
    """VTK inline binary: base64(UInt64 byte count) + base64(data)."""
    text = text.strip()
    nbytes = struct.unpack("<Q", base64.b64decode(text[:12]))[0]
    data = base64.b64decode(text[12:])
    assert len(data) == nbytes
    return np.frombuffer(data, dtype=dtype)


CASES = [((10,), (1.0,)), ((10, 11), (1.0, 2.0)), ((10, 11, 12), (1.0, 2.0, 3.0)), ((5, 3, 7), (0.5, 0.3, 2.1))]


@pytest.mark.parametrize("n,size", CASES)
def test_vtk_structured_grid_files(tmp_path, n, size):
    dim, g = len(n), 2
    rng = np.random.default_rng(dim)
    gn = [x + 2 * g for x in n] + [1] * (3 - dim)
    a = rng.normal(size=int(np.prod(gn)))
    b = rng.normal(size=int(np.prod(gn)))
    base = str(tmp_path / "out")
    grid_name = f"Cartesian{dim}D"
    D.write_vtk_host(n, size, g, [a, b], ["phi", "analytical"], base, grid_name, 100 * dim, time=0.25 * dim)

    stem = f"{grid_name}_{100 * dim}"
    pvts = os.path.join(base, stem + ".pvts")
    vts = os.path.join(base, stem, stem + "_0.vts")
    assert os.path.isfile(pvts) and os.path.isfile(vts)

    ext = [0, gn[0], 0, gn[1] if dim > 1 else 1, 0, gn[2] if dim > 2 else 0]
    ext_s = " ".join(str(e) for e in ext)

    root = ET.parse(pvts).getroot()
    assert root.get("type") == "PStructuredGrid" and root.get("header_type") == "UInt64"
    pg = root.find("PStructuredGrid")
    assert pg.get("WholeExtent") == ext_s and pg.get("GhostLevel") == str(g)
    assert [x.get("Name") for x in pg.find("PCellData")] == ["phi", "analytical"]
    assert all(x.get("type") == "Float64" for x in pg.find("PCellData"))
    pp = pg.find("PPoints/PDataArray")
    assert pp.get("type") == "Float32" and pp.get("NumberOfComponents") == "3"
    piece = pg.find("Piece")
    assert piece.get("Source") == f"{stem}/{stem}_0.vts" and piece.get("Extent") == ext_s
    # attribute order of the reference's WritePPieceAttributes: Source, then Extent
    raw = open(pvts).read()
    assert raw.index('Source="') < raw.index('Extent="', raw.index("<Piece"))

    root = ET.parse(vts).getroot()
    sg = root.find("StructuredGrid")
    assert sg.get("WholeExtent") == ext_s and sg.find("Piece").get("Extent") == ext_s
    tv = sg.find("FieldData/DataArray")
    assert tv.get("Name") == "TimeValue" and _decode(tv.text, "<f8")[0] == 0.25 * dim

    cells = {x.get("Name"): _decode(x.text, "<f8") for x in sg.find("Piece/CellData")}
    ncell = int(np.prod(gn))
    for name, src in (("phi", a), ("analytical", b)):
        got = cells[name]
        assert got.size == ncell
        # VTK id i + j cx + k cx cy  <->  grid ordinal (i gn1 + j) gn2 + k
        np.testing.assert_array_equal(got, src.reshape(gn).transpose(2, 1, 0).reshape(-1))

    pts = _decode(sg.find("Piece/Points/DataArray").text, "<f4").reshape(-1, 3)
    px, py, pz = ext[1] + 1, ext[3] + 1, ext[5] + 1
    assert pts.shape[0] == px * py * pz
    dn = [size[d] / n[d] for d in range(dim)] + [0.0] * (3 - dim)
    off = [0.0 - g * dn[d] for d in range(dim)] + [0.0] * (3 - dim)
    if dim == 1:
        dn[1] = dn[0]     # pseudo 2-D grid, offset 0 in y
    k, j, i = np.meshgrid(np.arange(pz), np.arange(py), np.arange(px), indexing="ij")
    want = np.stack([(dn[0] * i + off[0]).astype(np.float32), (dn[1] * j + off[1]).astype(np.float32),
                     (dn[2] * k + off[2]).astype(np.float32)], axis=-1).reshape(-1, 3)
    np.testing.assert_array_equal(pts, want)


def test_vtk_without_time_and_bad_args(tmp_path):
    n = (4, 5, 6)
    a = np.zeros(int(np.prod([x + 4 for x in n])))
    D.write_vtk_host(n, (1.0, 1.0, 1.0), 2, [a], ["phi"], str(tmp_path), "g", 0, time=-1.0)
    root = ET.parse(os.path.join(str(tmp_path), "g_0", "g_0_0.vts")).getroot()
    assert root.find("StructuredGrid/FieldData") is None
    with pytest.raises(D.DareError):
        D.write_vtk_host(n, (1.0, 1.0, 1.0), 2, [a], [""], str(tmp_path), "g", 0)
    with pytest.raises(D.DareError):
        D.write_vtk_host(n, (1.0, 1.0, 1.0), 2, [a], ["phi"], str(tmp_path / "missing" / "deeper"), "g", 0)
