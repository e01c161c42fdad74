"""Utilities kept from the reference (src/utilites.py:18-34)."""
from __future__ import annotations

import os

import numpy as np

__all__ = ["get_index", "write_fields_xdmf"]


def get_index(N, n, rank):
    """Slab bounds of ``rank`` among ``n`` ranks (remainder to the first ranks)."""
    batch_size = N // n
    remaining = N % n
    if rank < remaining:
        return (rank * (batch_size + 1), (rank + 1) * (batch_size + 1))
    return (rank * batch_size + remaining, (rank + 1) * batch_size + remaining)


def write_fields_xdmf(prefix, fields, spacing, time=0.0):
    """Write physical fields as raw little-endian float64 files
    ``{prefix}_{name}.raw`` (C order, x slowest) plus ``{prefix}.xdmf``, an
    XDMF description that ParaView and VisIt open directly.

    Stands in for the reference's HDF5 dumps and their XDMF sidecars
    (mpi4py_fft.HDF5File in src/SM_solver.py:280-302, generate_xdmf in
    src/utilites.py:27-34), which need h5py.  ``fields`` maps names to arrays
    of one shape (2D or 3D); ``spacing`` is the grid spacing dx.
    Returns the list of files written.
    """
    arrs = {k: np.ascontiguousarray(np.asarray(v, dtype="<f8")) for k, v in fields.items()}
    shape = next(iter(arrs.values())).shape
    if any(a.shape != shape for a in arrs.values()) or len(shape) not in (2, 3):
        raise ValueError("fields must share one 2D or 3D shape")
    dims = " ".join(str(n) for n in shape)
    nd = len(shape)
    topo = "3DCoRectMesh" if nd == 3 else "2DCoRectMesh"
    geo = "ORIGIN_DXDYDZ" if nd == 3 else "ORIGIN_DXDY"
    base = os.path.basename(prefix)
    written = []
    attrs = []
    for name, a in arrs.items():
        fn = "%s_%s.raw" % (prefix, name)
        a.tofile(fn)
        written.append(fn)
        attrs.append('      <Attribute Name="%s" AttributeType="Scalar" Center="Node">\n'
                     '        <DataItem Format="Binary" Endian="Little" NumberType="Float" Precision="8" '
                     'Dimensions="%s">%s_%s.raw</DataItem>\n      </Attribute>' % (name, dims, base, name))
    xml = ('<?xml version="1.0" ?>\n<Xdmf Version="3.0">\n  <Domain>\n'
           '    <Grid Name="%s" GridType="Uniform">\n'
           '      <Time Value="%.17g"/>\n'
           '      <Topology TopologyType="%s" Dimensions="%s"/>\n'
           '      <Geometry GeometryType="%s">\n'
           '        <DataItem Format="XML" NumberType="Float" Dimensions="%d">%s</DataItem>\n'
           '        <DataItem Format="XML" NumberType="Float" Dimensions="%d">%s</DataItem>\n'
           '      </Geometry>\n%s\n    </Grid>\n  </Domain>\n</Xdmf>\n'
           % (base, time, topo, dims, geo, nd, " ".join(["0"] * nd), nd, " ".join(["%.17g" % spacing] * nd),
              "\n".join(attrs)))
    fx = prefix + ".xdmf"
    with open(fx, "w") as f:
        f.write(xml)
    written.append(fx)
    return written
