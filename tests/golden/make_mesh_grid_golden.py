"""Generates tests/golden/mesh_grid.npz by running the reference's own level-set
generator (FunDEM/kernel/helper/LevelSetObjectGenerator.h, a host-only header)
through oracle/_ref/mesh_grid_ref, which oracle/build_ref.sh compiles against it.
Runs on the host; needs no CUDA device.

    python tests/golden/make_mesh_grid_golden.py [OUT.npz]

Cases (arrays prefixed with the case name):
  * superellipsoids built by LevelSetObject::Superellipsoid: the mesh
    (vertices, triangles), the class's own grid (analytic F / |grad F|,
    "<case>_analytic") and the grid of a TriangleMeshParticle made from that
    mesh ("<case>_mesh": nearest-triangle distance with the solid-angle sign);
  * a torus mesh (non-convex, made here) through TriangleMeshParticle.
Every grid is stored with its origin, node counts and spacing as the reference
chose them (buildGrid's padded, snapped box).
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
REF = ROOT / "oracle" / "_ref" / "mesh_grid_ref"

SUPER = {
    # name: (rx, ry, rz, ee, en, subdivision level, spacing, padding layers)
    "super_p4": (1.0, 0.8, 0.6, 0.5, 0.5, 2, 0.1, 2),
    "super_mixed": (0.9, 1.1, 0.7, 0.4, 1.3, 3, 0.12, 2),
    "ellipsoid": (0.5, 0.4, 0.3, 1.0, 1.0, 1, 0.07, 1),
}


def torus_mesh(R=1.0, r=0.35, nu=24, nv=12):
    """Closed torus around z, quads split in two, outward winding."""
    u = 2 * np.pi * np.arange(nu) / nu
    v = 2 * np.pi * np.arange(nv) / nv
    U, V = np.meshgrid(u, v, indexing="ij")
    X = np.stack([(R + r * np.cos(V)) * np.cos(U), (R + r * np.cos(V)) * np.sin(U), r * np.sin(V)], -1).reshape(-1, 3)
    tris = []
    for i in range(nu):
        for j in range(nv):
            a, b = i * nv + j, ((i + 1) % nu) * nv + j
            c, d = ((i + 1) % nu) * nv + (j + 1) % nv, i * nv + (j + 1) % nv
            tris += [(a, b, c), (a, c, d)]
    return X, np.array(tris, np.int32)


def _parse(path):
    lines = Path(path).read_text().split("\n")
    out = {}
    i = 0
    while i < len(lines):
        head = lines[i].split()
        if not head:
            i += 1
            continue
        if head[0] == "mesh":
            nv, nt = int(head[1]), int(head[2])
            out["verts"] = np.array([[float(x) for x in lines[i + 1 + k].split()] for k in range(nv)])
            out["tris"] = np.array([[int(x) for x in lines[i + 1 + nv + k].split()] for k in range(nt)], np.int32)
            i += 1 + nv + nt
        elif head[0] == "grid":
            name = head[1]
            size = np.array([int(head[2]), int(head[3]), int(head[4])], np.int32)
            n = int(np.prod(size))
            out[name] = np.array([float(lines[i + 1 + k]) for k in range(n)])
            out[name + "_size"] = size
            out[name + "_origin"] = np.array([float(head[5]), float(head[6]), float(head[7])])
            out[name + "_h"] = np.array(float(head[8]))
            i += 1 + n
        else:
            i += 1
    return out


def main(out_path):
    if not REF.exists():
        sys.exit(f"{REF} not built (oracle/build_ref.sh)")
    data = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, (rx, ry, rz, ee, en, level, h, pad) in SUPER.items():
            f = Path(tmp) / f"{name}.txt"
            subprocess.run([str(REF), "super", repr(rx), repr(ry), repr(rz), repr(ee), repr(en), str(level), repr(h),
                            str(pad), str(f)], check=True)
            r = _parse(f)
            data[f"{name}_params"] = np.array([rx, ry, rz, ee, en, level, h, pad])
            for k, v in r.items():
                data[f"{name}_{k}"] = v
        X, T = torus_mesh()
        mi = Path(tmp) / "torus_in.txt"
        mi.write_text(f"{len(X)} {len(T)}\n" + "\n".join(" ".join(repr(float(c)) for c in p) for p in X) + "\n" +
                      "\n".join(" ".join(str(int(c)) for c in t) for t in T) + "\n")
        f = Path(tmp) / "torus.txt"
        subprocess.run([str(REF), "mesh", str(mi), repr(0.1), "2", str(f)], check=True)
        r = _parse(f)
        data["torus_params"] = np.array([0.1, 2])
        for k, v in r.items():
            data[f"torus_{k}"] = v
    np.savez_compressed(out_path, **data)
    print("wrote", out_path, {k: v.shape for k, v in data.items() if v.ndim})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(Path(__file__).resolve().parent / "mesh_grid.npz"))
