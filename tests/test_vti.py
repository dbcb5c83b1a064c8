"""VTI geometry reader (fm_vti_read) against the reference's own readVTI.

The reference's header-only readVTI (include/vti/VTIReader.hpp:35-160) is
compiled for the host into oracle/_ref/libfmref_vti.so (oracle/build_oracle.py);
every ASCII case below is read by both and the dimensions and masks must be
identical, and every malformed file must fail in both with the same message.
The binary encodings the reference cannot read are checked against the values
that were written.  Runs on the CPU (no lattice is created).
"""
import base64
import ctypes as C
import os
import struct

import numpy as np
import pytest

from fluidmaxxer_b200 import vti
from fluidmaxxer_b200._abi import FM_ERR_ARG, FM_ERR_UNSUPPORTED, FmError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libfmref_vti.so")


def _ref():
    if not os.path.exists(REF_LIB):
        pytest.skip("reference readVTI not built (reference tree absent)")
    lib = C.CDLL(REF_LIB)
    lib.ref_vti_read.argtypes = [C.c_char_p, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.c_void_p, C.c_longlong]
    lib.ref_vti_error.restype = C.c_char_p
    return lib


def ref_read(path, thr=0.5):
    lib = _ref()
    nx, ny, nz = C.c_int(), C.c_int(), C.c_int()
    if lib.ref_vti_read(str(path).encode(), thr, C.byref(nx), C.byref(ny), C.byref(nz), None, 0):
        raise RuntimeError(lib.ref_vti_error().decode())
    mask = np.zeros(max(nx.value * ny.value * nz.value, 1), np.uint8)
    assert lib.ref_vti_read(str(path).encode(), thr, C.byref(nx), C.byref(ny), C.byref(nz), mask.ctypes.data,
                            mask.size) == 0
    return nx.value, ny.value, nz.value, mask[: nx.value * ny.value * nz.value]


def ascii_vti(path, extent, tokens, ext_attr="WholeExtent", comps=1, per_line=7):
    body = "\n".join(" ".join(tokens[i:i + per_line]) for i in range(0, len(tokens), per_line))
    path.write_text(
        '<?xml version="1.0"?>\n<VTKFile type="ImageData" version="0.1">\n'
        f'  <ImageData {ext_attr}="{extent}" Origin="0 0 0" Spacing="1 1 1">\n'
        f'    <Piece Extent="{extent}">\n      <CellData Scalars="geom">\n'
        f'        <DataArray type="Float32" Name="geom" NumberOfComponents="{comps}" format="ascii">\n'
        f"{body}\n        </DataArray>\n      </CellData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n")
    return path


def _fmt(rng, vals):
    out = []
    for i, v in enumerate(vals):
        k = i % 5
        out.append([f"{v:.9g}", f"{v:.3e}", f"+{abs(v):.4f}" if v >= 0 else f"{v:.4f}", repr(float(v)), f"{v:g}"][k])
    return out


CASES = {
    "scalar": (5, 4, 3, 1, "0 4 0 3 0 2", "WholeExtent"),
    "offset_extent": (6, 3, 2, 1, "2 7 10 12 -1 0", "WholeExtent"),
    "extent_only": (4, 4, 4, 1, "0 3 0 3 0 3", "Extent"),
    "vector": (4, 3, 3, 3, "0 3 0 2 0 2", "WholeExtent"),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("thr", [0.5, 0.0, 0.9])
def test_ascii_matches_reference_readvti(tmp_path, name, thr):
    nx, ny, nz, comps, ext, attr = CASES[name]
    rng = np.random.default_rng(hash(name) % 2**32)
    vals = rng.uniform(-1.0, 1.5, nx * ny * nz * comps)
    vals[::7] = 0.5                                    # exactly at the threshold
    path = ascii_vti(tmp_path / f"{name}.vti", ext, _fmt(rng, vals), attr, comps)
    rx, ry, rz, rmask = ref_read(path, thr)
    got = vti.read_vti(path, thr)
    assert (got.Nx, got.Ny, got.Nz) == (rx, ry, rz) == (nx, ny, nz)
    assert np.array_equal(got.mask, rmask)
    # the per-cell values: the parsed numbers (or magnitudes)
    parsed = np.array([float(t) for t in _fmt(rng, vals)])
    expect = parsed if comps == 1 else np.sqrt((parsed.reshape(-1, 3) ** 2).sum(1))
    assert np.array_equal(got.values, expect)


@pytest.mark.parametrize("count", [10, 200])
def test_count_mismatch_keeps_the_first_values(tmp_path, count):
    path = ascii_vti(tmp_path / "short.vti", "0 4 0 4 0 2", [str(v) for v in np.linspace(0, 1, count)])
    rx, ry, rz, rmask = ref_read(path)
    got = vti.read_vti(path)
    assert (got.Nx, got.Ny, got.Nz) == (rx, ry, rz)
    assert np.array_equal(got.mask, rmask)


def test_stops_at_the_first_non_number_like_the_stream(tmp_path):
    toks = ["0.7"] * 10 + ["abc"] + ["0.9"] * 17
    path = ascii_vti(tmp_path / "junk.vti", "0 2 0 2 0 2", toks)
    assert np.array_equal(vti.read_vti(path).mask, ref_read(path)[3])


BROKEN = {
    "no_extent": '<VTKFile><ImageData><Piece><CellData><DataArray format="ascii">1 2</DataArray></CellData></Piece></ImageData></VTKFile>',
    "bad_extent": '<VTKFile><ImageData WholeExtent="0 1 a 2 0 1"><DataArray format="ascii">1</DataArray></ImageData></VTKFile>',
    "no_dataarray": '<VTKFile><ImageData WholeExtent="0 1 0 1 0 1"></ImageData></VTKFile>',
    "no_close": '<VTKFile><ImageData WholeExtent="0 1 0 1 0 1"><DataArray format="ascii">1 1 1',
    "empty": '<VTKFile><ImageData WholeExtent="0 1 0 1 0 1"><DataArray format="ascii">  </DataArray></ImageData></VTKFile>',
}


@pytest.mark.parametrize("name", sorted(BROKEN))
def test_errors_carry_the_reference_messages(tmp_path, name):
    path = tmp_path / f"{name}.vti"
    path.write_text(BROKEN[name])
    with pytest.raises(RuntimeError) as ref:
        ref_read(path)
    with pytest.raises(FmError) as got:
        vti.read_vti(path)
    assert got.value.code == FM_ERR_ARG
    assert str(ref.value) in str(got.value)


def test_missing_file(tmp_path):
    with pytest.raises(RuntimeError) as ref:
        ref_read(tmp_path / "nope.vti")
    with pytest.raises(FmError) as got:
        vti.read_vti(tmp_path / "nope.vti")
    assert str(ref.value) in str(got.value)


def _binary_vti(path, vals, vtype, header="UInt32", appended=None):
    raw = vals.astype({"Float32": "<f4", "Float64": "<f8", "UInt8": "u1", "Int32": "<i4", "UInt16": "<u2"}[vtype]).tobytes()
    hdr = struct.pack("<I" if header == "UInt32" else "<Q", len(raw))
    head = (f'<?xml version="1.0"?>\n<VTKFile type="ImageData" version="1.0" byte_order="LittleEndian" '
            f'header_type="{header}">\n<ImageData WholeExtent="0 3 0 2 0 1">\n<Piece Extent="0 3 0 2 0 1">\n'
            f'<CellData>\n')
    if appended is None:
        data = base64.b64encode(hdr + raw).decode()
        text = head + f'<DataArray type="{vtype}" Name="s" format="binary">\n{data}\n</DataArray>\n' \
            '</CellData></Piece></ImageData></VTKFile>\n'
        path.write_bytes(text.encode())
    elif appended == "base64":
        data = base64.b64encode(hdr + raw).decode()
        text = head + f'<DataArray type="{vtype}" Name="s" format="appended" offset="0"/>\n' \
            f'</CellData></Piece></ImageData>\n<AppendedData encoding="base64">\n_{data}\n</AppendedData></VTKFile>\n'
        path.write_bytes(text.encode())
    else:
        text = head + f'<DataArray type="{vtype}" Name="s" format="appended" offset="0"/>\n' \
            '</CellData></Piece></ImageData>\n<AppendedData encoding="raw">\n_'
        path.write_bytes(text.encode() + hdr + raw + b"\n</AppendedData></VTKFile>\n")
    return path


@pytest.mark.parametrize("vtype", ["Float32", "Float64", "UInt8", "Int32", "UInt16"])
@pytest.mark.parametrize("enc", [None, "base64", "raw"])
@pytest.mark.parametrize("header", ["UInt32", "UInt64"])
def test_binary_encodings(tmp_path, vtype, enc, header):
    rng = np.random.default_rng(3)
    vals = rng.uniform(0, 3, 24)
    if vtype != "Float32" and vtype != "Float64":
        vals = np.floor(vals)
    path = _binary_vti(tmp_path / "b.vti", vals, vtype, header, enc)
    got = vti.read_vti(path, 0.5)
    stored = vals.astype(np.float32).astype(np.float64) if vtype == "Float32" else vals
    assert (got.Nx, got.Ny, got.Nz) == (4, 3, 2)
    assert np.array_equal(got.values, stored)
    assert np.array_equal(got.mask, (stored > 0.5).astype(np.uint8))


def test_compressed_is_rejected(tmp_path):
    path = tmp_path / "z.vti"
    path.write_text('<VTKFile type="ImageData" compressor="vtkZLibDataCompressor"><ImageData WholeExtent="0 1 0 1 0 1">'
                    '<DataArray type="Float32" format="binary">AAAA</DataArray></ImageData></VTKFile>')
    with pytest.raises(FmError) as e:
        vti.read_vti(path)
    assert e.value.code == FM_ERR_UNSUPPORTED


@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("comps", [1, 3])
def test_writer_round_trip_and_reference_reads_ascii(tmp_path, binary, comps):
    rng = np.random.default_rng(9)
    nx, ny, nz = 7, 5, 3
    vals = rng.normal(size=nx * ny * nz * comps) * 1e-3 + 0.5
    path = tmp_path / "w.vti"
    vti.write_vti(path, nx, ny, nz, vals, binary=binary)
    got = vti.read_vti(path)
    expect = vals if comps == 1 else np.sqrt((vals.reshape(-1, 3) ** 2).sum(1))
    assert np.array_equal(got.values, expect)
    if not binary:
        rx, ry, rz, rmask = ref_read(path)
        assert (rx, ry, rz) == (nx, ny, nz)
        assert np.array_equal(rmask, got.mask)


def test_geometry_file_drives_a_problem(tmp_path):
    """A sphere-pack geometry written as VTI and read back gives the same mask."""
    from fluidmaxxer_b200 import synth

    solid = synth.bernoulli(24, 12, 10, 0.3, 7, fluid_lo=2, fluid_hi=2, walls=True)
    path = tmp_path / "geometry.vti"
    vti.write_vti(path, 24, 12, 10, solid.astype(np.float64), name="solid", binary=False)
    got = vti.read_vti(path, 0.5)
    assert np.array_equal(got.mask, solid)
    assert np.array_equal(ref_read(path)[3], solid)
