"""Shared helpers for the parity tests: scene set-up and contact-list canonicalisation."""
import numpy as np


def dense_ellipsoid_scene(scenes, n=64, n_nodes=300, n_grid=16, spacing=8.0e-3, seed=7, floor=True, vel_sigma=0.05,
                          box=None):
    """Ellipsoids (5, 4, 3 mm) on a cubic lattice closer than two bounding radii, so that many
    surface nodes are inside neighbours; lowest layer overlapping the floor wall at z = 0."""
    m = int(np.ceil(n ** (1.0 / 3.0)))
    box = box or (m * spacing + 0.01, m * spacing + 0.01, m * spacing + 0.02)
    sc = scenes.ellipsoid_falling(n=n, n_nodes=n_nodes, n_grid=n_grid, packing=spacing, box=box, seed=seed,
                                  vel_sigma=vel_sigma)
    sc["pos"][:, 2] -= sc["pos"][:, 2].min() - 3.5e-3  # bottom layer centres at 3.5 mm: cut the floor at z = 0
    if not floor:
        sc["floor"] = None
    rng = np.random.default_rng(seed + 1)
    sc["angvel"] = rng.normal(0.0, 5.0, size=(n, 3))
    return sc


def load_scene(lsdem, scenes, sc, precision=0, **cap):
    sv = lsdem.Solver()
    scenes.load_into(sv, sc)
    if "angvel" in sc:
        sv.set_state(angvel=sc["angvel"])
    if cap:
        sv.set_capacity(**cap)
    sv.set_precision(precision)
    sv.set_record_contacts(True)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    return sv


def canon(c, keys=("node", "partner")):
    """Contacts sorted by (node, partner[, image]) for comparison with the reference order."""
    cols = [np.asarray(c[k]) for k in keys]
    order = np.lexsort(cols[::-1])
    return order


def history_from_gpu(c, n_nodes_total):
    """The reference's per-node history arrays (inclusive prefix, partner, spring) of a contact list."""
    node = np.asarray(c["node"], np.int64)
    order = np.argsort(node, kind="stable")
    cnt = np.bincount(node, minlength=n_nodes_total)
    return {"prefix": np.cumsum(cnt).astype(np.int32), "partner": np.asarray(c["partner"], np.int32)[order],
            "spring": np.asarray(c["spring"])[order]}


def read_vtu(path):
    """Arrays of a VTK XML UnstructuredGrid file with inline base64 binary arrays (UInt64 byte-count
    header) or ascii arrays: {"TIME", "STEP", "points", "connectivity", "offsets", "types", and the
    PointData arrays by name}."""
    import base64
    import xml.etree.ElementTree as ET

    types = {"Float32": np.float32, "Float64": np.float64, "Int32": np.int32, "Int64": np.int64, "UInt8": np.uint8}
    root = ET.parse(path).getroot()
    out = {}
    piece = root.find("UnstructuredGrid/Piece")
    out["n_points"] = int(piece.get("NumberOfPoints"))
    out["n_cells"] = int(piece.get("NumberOfCells"))
    for da in root.iter("DataArray"):
        dt = types[da.get("type")]
        nc = int(da.get("NumberOfComponents", "1"))
        text = (da.text or "").strip()
        if da.get("format") == "binary":
            raw = base64.b64decode(text)
            nbytes = int(np.frombuffer(raw[:8], "<u8")[0])
            assert len(raw) == 8 + nbytes, (path, da.get("Name"), len(raw), nbytes)
            a = np.frombuffer(raw[8:8 + nbytes], dt)
        else:
            a = np.array(text.split(), dt)
        if nc > 1:
            a = a.reshape(-1, nc)
        name = da.get("Name")
        out[name if name else "points"] = a
    return out
