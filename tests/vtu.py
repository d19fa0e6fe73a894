"""Reader for the files DataWriter_t writes (test helper): a parallel
unstructured grid summary (.pvtu-style XML) and its piece with inline base64
arrays (format="binary", UInt64 headers)."""
from __future__ import annotations

import base64
import os
import xml.etree.ElementTree as ET

import numpy as np

DTYPES = {"Float64": np.float64, "Int64": np.int64, "UInt64": np.uint64, "Int32": np.int32, "UInt8": np.uint8}


def _array(el) -> np.ndarray:
    raw = base64.b64decode(el.text.strip())
    n = int(np.frombuffer(raw[:8], dtype=np.uint64)[0])
    vals = np.frombuffer(raw[8:8 + n], dtype=DTYPES[el.get("type")])
    comps = int(el.get("NumberOfComponents", "1"))
    return vals.reshape(-1, comps) if comps > 1 else vals


def read_grid(summary_path: str) -> dict:
    """Summary file -> {"summary": {...}, "points", "connectivity", "offsets",
    "types", "point_data": {name: array}, "cell_data": {name: array}}."""
    summary = ET.parse(summary_path).getroot()
    assert summary.get("type") == "PUnstructuredGrid"
    pug = summary.find("PUnstructuredGrid")
    pieces = [p.get("Source") for p in pug.findall("Piece")]
    assert len(pieces) == 1
    out = {
        "summary_point_data": [(a.get("Name"), a.get("type"), int(a.get("NumberOfComponents", "1"))) for a in pug.find("PPointData")],
        "summary_cell_data": [(a.get("Name"), a.get("type"), int(a.get("NumberOfComponents", "1"))) for a in pug.find("PCellData")],
        "piece_file": pieces[0],
    }
    root = ET.parse(os.path.join(os.path.dirname(summary_path), pieces[0])).getroot()
    assert root.get("type") == "UnstructuredGrid" and root.get("header_type") == "UInt64"
    piece = root.find("UnstructuredGrid").find("Piece")
    out["n_points"] = int(piece.get("NumberOfPoints"))
    out["n_cells"] = int(piece.get("NumberOfCells"))
    out["point_data"] = {a.get("Name"): _array(a) for a in piece.find("PointData")}
    out["cell_data"] = {a.get("Name"): _array(a) for a in piece.find("CellData")}
    out["points"] = _array(piece.find("Points").find("DataArray"))
    cells = {a.get("Name"): _array(a) for a in piece.find("Cells")}
    out.update(connectivity=cells["connectivity"], offsets=cells["offsets"], types=cells["types"])
    return out
