"""Reader of VTK files restating the parsing steps of the reference's `read_vtk`
(src/VtkReader/VtkReader.jl): pvtu -> piece sources relative to the pvtu's directory
(:250-269); appended raw data after `<AppendedData encoding="raw">` and the next "_", up to
"\\n  </AppendedData>" (:50-83); per DataArray (format "appended", type Float64 / Int64 /
UInt8, NumberOfComponents, offset) four UInt64 header words, the fourth the compressed size,
then a zlib block (:213-222); Points, PointData and FieldData arrays (:95-110, :224-247).
Test infrastructure: checks that files written by pdcuda.vtk parse the way the reference's
reader parses them."""
import os
import re
import xml.etree.ElementTree as ET
import zlib

import numpy as np

TYPES = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}


def _raw(file):
    data = open(file, "rb").read()
    m = data.find(b'<AppendedData encoding="raw">')
    assert m >= 0, "no raw appended data"
    begin = data.find(b"_", m) + 1
    end = data.find(b"\n  </AppendedData>", begin)
    assert end > begin
    xml = data[:begin - 1] + data[end:]
    return xml.decode(), data[begin:end]


def _array(da, raw):
    assert da.attrib["format"] == "appended"
    t = TYPES[da.attrib["type"]]
    ncomp = int(da.attrib["NumberOfComponents"])
    off = int(da.attrib["offset"])
    head = np.frombuffer(raw[off:off + 32], dtype="<u8")
    nbytes = int(head[3])
    a = np.frombuffer(zlib.decompress(raw[off + 32:off + 32 + nbytes]), dtype=t)
    return a if ncomp == 1 else a.reshape(-1, ncomp).T   # ncomp x n, as the reference returns


def read_vtu(file):
    xml, raw = _raw(file)
    root = ET.fromstring(xml[xml.index("<VTKFile"):])
    grid = root.find("UnstructuredGrid")
    piece = grid.find("Piece")
    d = {"position": _array(piece.find("Points").find("DataArray"), raw)}
    pdata = piece.find("PointData")
    if pdata is not None:
        for da in pdata:
            d[da.attrib["Name"]] = _array(da, raw)
    fdata = grid.find("FieldData")
    if fdata is not None:
        for da in fdata:
            d[da.attrib["Name"]] = _array(da, raw)
    return d


def read_vtk(file):
    if file.endswith(".vtu"):
        return read_vtu(file)
    root = ET.parse(file).getroot()
    pieces = [os.path.join(os.path.dirname(file), p.attrib["Source"])
              for p in root.find("PUnstructuredGrid").findall("Piece")]
    parts = [read_vtu(p) for p in pieces]
    out = {}
    for k in parts[0]:
        vals = [p[k] for p in parts]
        out[k] = vals[0] if k == "time" else np.concatenate(vals, axis=-1)
    return out


def find_vtk_files(path):
    """pvtu files sorted by time step (process_each_export.jl:148-155)."""
    files = [os.path.join(path, f) for f in os.listdir(path) if f.endswith(".pvtu")]
    return sorted(files, key=lambda f: int(re.findall(r"_(\d+)\.pvtu$", f)[0]))
