"""Minimal reader of legacy VTK files in BINARY encoding (big-endian words), for the tests."""
import numpy as np


def read_vtk(path):
    """Returns (header dict, arrays dict).  Handles the sections the library writes."""
    data = open(path, "rb").read()
    pos = 0

    def line():
        nonlocal pos
        e = data.index(b"\n", pos)
        s = data[pos:e].decode()
        pos = e + 1
        return s

    def words(n, dt):
        nonlocal pos
        a = np.frombuffer(data, dtype=dt, count=n, offset=pos).copy()
        pos += 4 * n
        assert data[pos:pos + 1] == b"\n"
        pos += 1
        return a

    head = {"version": line(), "title": line(), "encoding": line(), "dataset": line().split()[1]}
    arrays = {}
    while pos < len(data):
        parts = line().split()
        if not parts:
            continue
        key = parts[0]
        if key in ("DIMENSIONS", "ORIGIN", "SPACING"):
            head[key] = [float(x) for x in parts[1:]]
        elif key in ("POINT_DATA", "CELL_DATA"):
            head[key] = int(parts[1])
        elif key == "POINTS":
            arrays["POINTS"] = words(3 * int(parts[1]), ">f4").reshape(-1, 3)
        elif key in ("CELLS", "VERTICES"):
            arrays[key] = words(int(parts[2]), ">i4")
        elif key == "CELL_TYPES":
            arrays[key] = words(int(parts[1]), ">i4")
        elif key == "SCALARS":
            name, dtype = parts[1], parts[2]
            assert line().startswith("LOOKUP_TABLE")
            n = head.get("POINT_DATA", head.get("CELL_DATA"))
            arrays[name] = words(n, ">f4" if dtype == "float" else ">i4")
        elif key == "VECTORS":
            arrays[parts[1]] = words(3 * head["POINT_DATA"], ">f4").reshape(-1, 3)
        else:
            raise ValueError(f"unexpected VTK line {parts}")
    return head, arrays
