"""VTK export of device fields in the reference's file layout.

`Job(path=..., freq=..., fields=...)` of the reference writes, at step 0 and at every step n
with n % freq == 0, `<path>/vtk/timestep_<n>.pvtu` with one piece
`<path>/vtk/timestep_<n>/timestep_<n>_1.vtu` (WriteVTK's `pvtk_grid`, src/auxiliary/io.jl:
141-186): an UnstructuredGrid of vertex cells at the current positions, the exported fields as
point data and the time as field data. The data arrays are appended raw binary, each a
zlib-compressed block behind four UInt64 header words (blocks, block size, last block size,
compressed size): the form the reference's own reader `read_vtk` parses
(src/VtkReader/VtkReader.jl). Default fields: displacement and damage (io.jl,
default_export_fields).
"""
from __future__ import annotations

import os
import zlib

import numpy as np

DEFAULT_FIELDS = ("displacement", "damage")
_VTK_TYPE = {np.dtype(np.float64): "Float64", np.dtype(np.int64): "Int64", np.dtype(np.uint8): "UInt8"}


def _block(a):
    raw = np.ascontiguousarray(a).tobytes()
    comp = zlib.compress(raw)
    head = np.array([1, len(raw), len(raw), len(comp)], dtype="<u8").tobytes()
    return head + comp


def _as_points(a, n):
    """(n, c) C-order array of a field given as (c, n) / (n,) like the reference's 3 x N."""
    a = np.asarray(a)
    if a.ndim == 2 and a.shape[0] != n:
        a = a.T
    return np.ascontiguousarray(a)


def write_vtu(filename, position, point_data, time):
    """One piece: position (n, 3) or (3, n); point_data {name: (n,), (n, c) or (c, n)}."""
    n = np.asarray(position).size // 3
    pos = _as_points(np.asarray(position, np.float64), n).reshape(n, 3)
    arrays, blobs, off = [], [], 0

    def add(kind, name, a, ncomp):
        nonlocal off
        a = np.asarray(a)
        t = _VTK_TYPE.get(a.dtype)
        if t is None:
            a = a.astype(np.float64)
            t = "Float64"
        b = _block(a)
        arrays.append((kind, f'<DataArray type="{t}" Name="{name}" NumberOfComponents="{ncomp}" '
                             f'format="appended" offset="{off}"/>'))
        blobs.append(b)
        off += len(b)

    add("field", "time", np.array([float(time)]), 1)
    add("points", "Points", pos, 3)
    add("cells", "connectivity", np.arange(n, dtype=np.int64), 1)
    add("cells", "offsets", np.arange(1, n + 1, dtype=np.int64), 1)
    add("cells", "types", np.ones(n, dtype=np.uint8), 1)  # VTK_VERTEX
    for name, a in point_data.items():
        a = _as_points(a, n)
        add("point", name, a, 1 if a.ndim == 1 else a.shape[1])
    sect = lambda k: "\n".join("        " + x for kk, x in arrays if kk == k)
    xml = (
        '<?xml version="1.0" encoding="utf-8"?>\n'
        '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" '
        'header_type="UInt64" compressor="vtkZLibDataCompressor">\n'
        '  <UnstructuredGrid>\n'
        '    <FieldData>\n' + sect("field").replace("        ", "      ") + '\n    </FieldData>\n'
        f'    <Piece NumberOfPoints="{n}" NumberOfCells="{n}">\n'
        '      <Points>\n' + sect("points") + '\n      </Points>\n'
        '      <Cells>\n' + sect("cells") + '\n      </Cells>\n'
        '      <PointData>\n' + sect("point") + '\n      </PointData>\n'
        '    </Piece>\n'
        '  </UnstructuredGrid>\n'
        '  <AppendedData encoding="raw">\n   _')
    with open(filename, "wb") as f:
        f.write(xml.encode())
        for b in blobs:
            f.write(b)
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")


def write_pvtu(filebase, position, point_data, time):
    """`<filebase>.pvtu` with the single piece `<filebase>/<name>_1.vtu`."""
    name = os.path.basename(filebase)
    os.makedirs(filebase, exist_ok=True)
    write_vtu(os.path.join(filebase, f"{name}_1.vtu"), position, point_data, time)
    n = np.asarray(position).size // 3
    pd_lines = []
    for fname, a in point_data.items():
        a = _as_points(a, n)
        t = _VTK_TYPE.get(a.dtype, "Float64")
        c = 1 if a.ndim == 1 else a.shape[1]
        pd_lines.append(f'      <PDataArray type="{t}" Name="{fname}" NumberOfComponents="{c}"/>')
    xml = ('<?xml version="1.0" encoding="utf-8"?>\n'
           '<VTKFile type="PUnstructuredGrid" version="1.0" byte_order="LittleEndian" '
           'header_type="UInt64">\n'
           '  <PUnstructuredGrid GhostLevel="0">\n'
           '    <PPointData>\n' + "\n".join(pd_lines) + '\n    </PPointData>\n'
           '    <PPoints>\n      <PDataArray type="Float64" Name="Points" NumberOfComponents="3"/>\n'
           '    </PPoints>\n'
           f'    <Piece Source="{name}/{name}_1.vtu"/>\n'
           '  </PUnstructuredGrid>\n'
           '</VTKFile>\n')
    with open(filebase + ".pvtu", "w") as f:
        f.write(xml)
    return filebase + ".pvtu"


class VtkExport:
    """Callable export(step, t, dev) of a Job with a path: the reference's export cadence
    (step 0 and every step n with n % freq == 0) and file names (body name "" ->
    `timestep_<n>`)."""

    def __init__(self, path, freq, fields=None):
        if fields is None:
            fields = DEFAULT_FIELDS
        self.root = os.path.join(path, "vtk")
        self.freq = int(freq)
        self.fields = tuple(fields)
        os.makedirs(self.root, exist_ok=True)
        self.written = []

    def __call__(self, step, t, dev):
        if step != 0 and (self.freq <= 0 or step % self.freq != 0):
            return
        data = {f: dev.field(f) for f in self.fields}
        fb = os.path.join(self.root, f"timestep_{step}")
        self.written.append(write_pvtu(fb, dev.field("position"), data, t))
