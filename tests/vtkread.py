"""A reader of the VTK XML files with raw appended data and UInt64 headers
that the library writes (test infrastructure)."""
from __future__ import annotations

import re
import xml.etree.ElementTree as ET

import numpy as np

TYPES = {"Float64": np.float64, "UInt64": np.uint64, "Int64": np.int64, "Int32": np.int32, "UInt8": np.uint8}


def read(path):
    """(xml root, {array name: numpy array (tuples, components)}, raw header text)."""
    data = open(path, "rb").read()
    marker = b'<AppendedData encoding="raw">\n_'
    at = data.index(marker)
    head = data[:at].decode() + '<AppendedData encoding="raw"/>\n</VTKFile>\n'
    root = ET.fromstring(head)
    payload = data[at + len(marker):]
    tail = b"\n  </AppendedData>\n</VTKFile>\n"
    assert payload.endswith(tail)
    payload = payload[:-len(tail)]
    arrays = {}
    for el in root.iter("DataArray"):
        if el.get("format") != "appended":
            continue
        off = int(el.get("offset"))
        nbytes = int(np.frombuffer(payload[off:off + 8], dtype=np.uint64)[0])
        a = np.frombuffer(payload[off + 8:off + 8 + nbytes], dtype=TYPES[el.get("type")])
        comps = int(el.get("NumberOfComponents", "1"))
        arrays[el.get("Name")] = a.reshape(-1, comps) if comps > 1 else a
    return root, arrays, head


def field_data(root) -> dict:
    out = {}
    fd = root.find(".//FieldData")
    for el in fd:
        name = el.get("Name")
        text = el.text.strip()
        if el.get("type") == "String":
            codes = [int(x) for x in text.split()]
            assert codes[-1] == 0
            out[name] = bytes(codes[:-1]).decode()
        elif el.get("type") == "Float64":
            out[name] = float(text)
        else:
            out[name] = int(text)
    return out
