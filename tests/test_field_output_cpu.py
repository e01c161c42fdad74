"""The field writer that stands in for the reference's HDF5 dumps: raw
float64 files and an XDMF description that names them (no GPU needed)."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from sles.utilites import write_fields_xdmf


@pytest.mark.parametrize("shape", [(6, 5, 4), (8, 7)])
def test_fields_round_trip_through_xdmf(tmp_path, shape):
    rng = np.random.default_rng(1)
    fields = {"u": rng.standard_normal(shape), "v": rng.standard_normal(shape).astype(np.float32)}
    files = write_fields_xdmf(str(tmp_path / "dump3"), fields, spacing=0.25, time=1.5)
    assert sorted(p.split("/")[-1] for p in files) == ["dump3.xdmf", "dump3_u.raw", "dump3_v.raw"]
    root = ET.parse(tmp_path / "dump3.xdmf").getroot()
    grid = root.find("Domain/Grid")
    assert float(grid.find("Time").get("Value")) == 1.5
    assert grid.find("Topology").get("Dimensions") == " ".join(map(str, shape))
    for att in grid.findall("Attribute"):
        item = att.find("DataItem")
        a = np.fromfile(tmp_path / item.text, dtype="<f8").reshape(shape)
        assert np.array_equal(a, np.asarray(fields[att.get("Name")], dtype=np.float64))


def test_mismatched_shapes_are_rejected(tmp_path):
    with pytest.raises(ValueError):
        write_fields_xdmf(str(tmp_path / "d"), {"u": np.zeros((4, 4, 4)), "v": np.zeros((4, 4))}, spacing=1.0)
