"""The .vti writer (clb_vti_write) on the CPU: the file is VTK ImageData XML that an independent
reader (here: xml + base64 + numpy) turns back into the interior x-planes of the arrays, x fastest,
components side by side, in the stored type."""
import base64
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest


def read_vti(path):
    root = ET.parse(path).getroot()
    assert root.get("type") == "ImageData" and root.get("header_type") == "UInt64"
    img = root.find("ImageData")
    ext = [int(v) for v in img.get("WholeExtent").split()]
    dims = (ext[1] - ext[0] + 1, ext[3] - ext[2] + 1, ext[5] - ext[4] + 1)
    out = {}
    for da in img.find("Piece").find("PointData").findall("DataArray"):
        text = da.text.strip()
        nbytes = np.frombuffer(base64.b64decode(text[:12]), dtype="<u8")[0]
        raw = base64.b64decode(text[12:])
        assert len(raw) == nbytes
        dt = {"Float32": "<f4", "Float64": "<f8"}[da.get("type")]
        comps = int(da.get("NumberOfComponents"))
        out[da.get("Name")] = (np.frombuffer(raw, dtype=dt), comps, da.get("type"))
    return dims, out


def test_vti_round_trip(clb, tmp_path):
    nx, ny, nz = 7, 5, 4
    N = nx * ny * nz
    rng = np.random.default_rng(0)
    scal = rng.random(N)
    vec = rng.random((3, N)).astype(np.float32)
    path = os.path.join(tmp_path, "f_0000042.vti")
    clb.vti_write(path, (nx, ny, nz), {"Density": scal, "velocity": vec})
    dims, arrays = read_vti(path)
    assert dims == (nx - 2, ny, nz)
    d, comps, typ = arrays["Density"]
    assert comps == 1 and typ == "Float64"
    # interior planes x = 1..nx-2, x fastest in the file
    want = scal.reshape(nx, ny, nz)[1:-1].transpose(2, 1, 0).ravel()
    np.testing.assert_array_equal(d, want)
    v, comps, typ = arrays["velocity"]
    assert comps == 3 and typ == "Float32"
    want = vec.reshape(3, nx, ny, nz)[:, 1:-1].transpose(3, 2, 1, 0).reshape(-1)
    np.testing.assert_array_equal(v, want)


def test_vti_rejects_bad_arguments(clb, tmp_path):
    with pytest.raises(clb.ClbError):
        clb.vti_write(os.path.join(tmp_path, "x.vti"), (2, 3, 3), {"a": np.zeros(18)})
    with pytest.raises(clb.ClbError):
        clb.vti_write(os.path.join(tmp_path, "no", "such", "dir.vti"), (4, 3, 3), {"a": np.zeros(36)})
