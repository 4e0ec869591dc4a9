"""FP64 CPU oracle of the level-set DEM step — TEST INFRASTRUCTURE ONLY.

ctypes binding of oracle/liboracle.so (the C++ restatement of the reference
kernels in lsdem_oracle.cpp) and a step orchestrator that follows the
reference loop (FunDEM/kernel/LSSolver.h:1000-1128): half kick, drift of
particles and walls, hash + stable sort + cell ranges, per-node count /
inclusive scan / write with history carried over by partner id
(SolidInteraction.h:93-152), periodic wrap and ghost images
(PeriodicBoundary.h:215-303), zeroed forces, contact forces, bonds, external
hook, half kick.

Only tests/, __graft_entry__.smoke() (as the checker) and bench.py's CPU
baseline leg use this module. Parity of this oracle with the reference's own
kernels is pinned by the golden vectors under tests/golden/.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# LSDEM_ORACLE_LIB: another build of the same source (the benchmark's CPU baseline builds
# one with -march=native for the host it runs on)
LIB = Path(os.environ["LSDEM_ORACLE_LIB"]) if os.environ.get("LSDEM_ORACLE_LIB") else HERE / "liboracle.so"

FIX_GRADIENT = 1
FIX_SQRTF = 2


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


if not LIB.exists():
    build()
lib = C.CDLL(str(LIB))

DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)
LP = C.POINTER(C.c_longlong)


class Bodies(C.Structure):
    _fields_ = [("n", C.c_int), ("pos", DP), ("quat", DP), ("radius", DP), ("invh", DP), ("origin", DP),
                ("gsize", IP), ("sdf_off", LP), ("sdf", DP), ("sdf_scale", DP)]


class Nodes(C.Structure):
    _fields_ = [("np", C.c_int), ("node_base", LP), ("node_src", LP), ("node_local", DP), ("node_scale", DP)]


class Grid(C.Structure):
    _fields_ = [("min", C.c_double * 3), ("max", C.c_double * 3), ("inv", C.c_double * 3), ("size", C.c_int * 3),
                ("idx", IP), ("start", IP), ("end", IP)]


class Dyn(C.Structure):
    _fields_ = [("n", C.c_int), ("pos", DP), ("vel", DP), ("angvel", DP), ("invmass", DP), ("kn", DP), ("ks", DP),
                ("mu", DP), ("res", DP)]


def _d(a):
    return None if a is None else a.ctypes.data_as(DP)


def _i(a):
    return None if a is None else a.ctypes.data_as(IP)


def _l(a):
    return None if a is None else a.ctypes.data_as(LP)


def f64(a, shape=None):
    a = np.ascontiguousarray(a, np.float64)
    return a.reshape(shape) if shape is not None else a


def i32(a):
    return np.ascontiguousarray(a, np.int32)


def i64(a):
    return np.ascontiguousarray(a, np.int64)


lib.ora_grid_set.argtypes = [DP, DP, C.c_double, DP, IP, DP]
lib.ora_hash.argtypes = [C.c_int, DP, DP, DP, DP, IP, IP]
lib.ora_ghost_hash.argtypes = [C.c_int, DP, DP, DP, DP, IP, IP]
lib.ora_sort_ranges.argtypes = [C.c_int, IP, IP, C.c_int, IP, IP]
lib.ora_wrap.argtypes = [C.c_int, DP, DP, DP, C.c_int]
lib.ora_ghost_positions.argtypes = [C.c_int, DP, DP, DP, DP, C.c_int, DP]
lib.ora_detect_count.argtypes = [C.c_int, C.POINTER(Nodes), DP, DP, C.POINTER(Bodies), C.POINTER(Grid), C.c_int,
                                 C.c_int, IP]
lib.ora_detect_write.argtypes = [C.c_int, C.POINTER(Nodes), DP, DP, C.POINTER(Bodies), C.POINTER(Grid), C.c_int,
                                 C.c_int, IP, IP, IP, DP, C.c_int, DP, DP, DP, DP, LP, IP, IP]
lib.ora_contact_force.argtypes = [C.c_int, C.c_longlong, IP, IP, DP, DP, DP, DP, DP, DP, C.POINTER(Dyn),
                                  C.POINTER(Dyn), C.c_double, C.c_int, DP, DP, C.c_int]
lib.ora_bond_force.argtypes = [C.c_int, IP, DP, DP, DP, IP, DP, DP, DP, DP, DP]
lib.ora_kick.argtypes = [C.c_int, DP, DP, DP, DP, DP, DP, DP, DP, C.c_double]
lib.ora_drift.argtypes = [C.c_int, DP, DP, DP, DP, C.c_double]
lib.ora_mass_props.argtypes = [DP, C.c_int, C.c_int, C.c_int, DP, C.c_double, C.c_double, DP]
lib.ora_mesh_grid.argtypes = [DP, IP, C.c_int, DP, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, DP]
lib.ora_sector_wrap.argtypes = [C.c_int, DP, DP, DP, DP, DP, DP]
lib.ora_sector_ghosts.argtypes = [C.c_int, DP, DP, DP, DP, DP, DP, DP, DP]
lib.ora_set_threads.argtypes = [C.c_int]
lib.ora_num_threads.restype = C.c_int


def set_threads(n: int):
    lib.ora_set_threads(int(n))


def num_threads() -> int:
    return int(lib.ora_num_threads())


# ---------------------------------------------------------------------------
# Unit-level functions (each mirrors one reference launcher).


def grid_set(mn, mx, cell):
    inv = np.zeros(3)
    size = np.zeros(3, np.int32)
    mx_out = np.zeros(3)
    lib.ora_grid_set(_d(f64(mn)), _d(f64(mx)), float(cell), _d(inv), _i(size), _d(mx_out))
    return {"min": f64(mn).copy(), "max": mx_out, "inv": inv, "size": size}


def hash_keys(pos, g, ghost=False):
    pos = f64(pos, (-1, 3))
    key = np.zeros(len(pos), np.int32)
    f = lib.ora_ghost_hash if ghost else lib.ora_hash
    f(len(pos), _d(pos), _d(f64(g["min"])), _d(f64(g["max"])), _d(f64(g["inv"])), _i(i32(g["size"])), _i(key))
    return key


def sort_ranges(key, ncells):
    k = i32(key).copy()
    idx = np.zeros(len(k), np.int32)
    st = np.zeros(ncells, np.int32)
    en = np.zeros(ncells, np.int32)
    lib.ora_sort_ranges(len(k), _i(k), _i(idx), int(ncells), _i(st), _i(en))
    return {"sorted_key": k, "sorted_idx": idx, "start": st, "end": en}


def wrap(pos, g, axis):
    lib.ora_wrap(len(pos), _d(pos), _d(f64(g["min"])), _d(f64(g["max"])), int(axis))


def sector_wrap(pos, vel, quat, g, force=None, torque=None):
    """Sector wrap in place (mySpatialGrid.cu:58-85); force / torque, when given, turn with the particles."""
    lib.ora_sector_wrap(len(pos), _d(pos), _d(vel), _d(quat), _d(force), _d(torque), _d(f64(g["min"])))


def sector_ghosts(pos, vel, quat, g):
    """Sector image sets R90, R180, R270 (mySpatialGrid.cu:154-212): (pos, vel, quat), each 3 x n."""
    n = len(pos)
    gp, gv, gq = np.zeros((3 * n, 3)), np.zeros((3 * n, 3)), np.zeros((3 * n, 4))
    lib.ora_sector_ghosts(n, _d(f64(pos)), _d(f64(vel)), _d(f64(quat)), _d(f64(g["min"])), _d(f64(g["inv"])),
                          _d(gp), _d(gv), _d(gq))
    return gp.reshape(3, n, 3), gv.reshape(3, n, 3), gq.reshape(3, n, 4)


def ghost_positions(pos, g, mask):
    out = np.zeros_like(pos)
    lib.ora_ghost_positions(len(pos), _d(f64(pos)), _d(f64(g["min"])), _d(f64(g["max"])), _d(f64(g["inv"])),
                            int(mask), _d(out))
    return out


def mass_props(sdf, size, origin, h, density):
    out = np.zeros(16)
    lib.ora_mass_props(_d(f64(sdf)), int(size[0]), int(size[1]), int(size[2]), _d(f64(origin)), float(h),
                       float(density), _d(out))
    return out


def mesh_grid(verts, tris, origin, size, h, positive_inside=False):
    """Level-set grid of a closed triangle mesh (buildGrid over the mesh distance with the
    solid-angle sign, LevelSetObjectGenerator.h:122-224, 454-500, 758-802)."""
    v = f64(verts, (-1, 3))
    t = i32(np.reshape(tris, (-1, 3)))
    out = np.zeros(int(np.prod(np.asarray(size, np.int64))))
    lib.ora_mesh_grid(_d(v), _i(t), len(t), _d(f64(origin)), int(size[0]), int(size[1]), int(size[2]), float(h),
                      1 if positive_inside else 0, _d(out))
    return out


class BodySet:
    """SDF-side body arrays (particles, walls or ghost images) kept alive for ctypes."""

    def __init__(self, pos, quat, radius, invh, origin, gsize, sdf_off, sdf, sdf_scale=None):
        self.pos = f64(pos, (-1, 3))
        self.quat = f64(quat, (-1, 4))
        self.radius = f64(radius)
        self.invh = f64(invh)
        self.origin = f64(origin, (-1, 3))
        self.gsize = i32(gsize).reshape(-1, 3)
        self.sdf_off = i64(sdf_off)
        self.sdf = f64(sdf)
        self.sdf_scale = None if sdf_scale is None else f64(sdf_scale)
        self.s = Bodies(len(self.pos), _d(self.pos), _d(self.quat), _d(self.radius), _d(self.invh), _d(self.origin),
                        _i(self.gsize), _l(self.sdf_off), _d(self.sdf), _d(self.sdf_scale))


class NodeSet:
    def __init__(self, node_base, node_src, node_local, node_scale=None):
        self.node_base = i64(node_base)
        self.node_src = i64(node_src)
        self.node_local = f64(node_local, (-1, 3))
        self.node_scale = None if node_scale is None else f64(node_scale)
        self.s = Nodes(len(self.node_src), _l(self.node_base), _l(self.node_src), _d(self.node_local),
                       _d(self.node_scale))

    @property
    def total(self):
        return int(self.node_base[-1])


def make_grid(g, sorted_idx, start, end):
    G = Grid()
    for a in range(3):
        G.min[a], G.max[a], G.inv[a], G.size[a] = g["min"][a], g["max"][a], g["inv"][a], int(g["size"][a])
    keep = (i32(sorted_idx), i32(start), i32(end))
    G.idx, G.start, G.end = _i(keep[0]), _i(keep[1]), _i(keep[2])
    return G, keep


def detect(mode, nodes: NodeSet, ppos, pquat, B: BodySet, g, sorted_idx, start, end, old=None, flags=0, p0=0,
           p1=None):
    """Count + inclusive scan + write of one interaction list (reference order).

    old: dict(prefix, partner, spring) of the previous step of the same list (or None).
    Returns dict(count, prefix, node, partner, owner, point, normal, overlap, spring)."""
    ppos = f64(ppos, (-1, 3))
    pquat = f64(pquat, (-1, 4))
    p1 = nodes.s.np if p1 is None else p1
    nn = nodes.total
    G, keep = make_grid(g, sorted_idx, start, end)
    count = np.zeros(nn, np.int32)
    lib.ora_detect_count(int(mode), C.byref(nodes.s), _d(ppos), _d(pquat), C.byref(B.s), C.byref(G), int(p0), int(p1),
                         _i(count))
    prefix = np.cumsum(count, dtype=np.int64).astype(np.int32)
    nc = int(prefix[-1]) if nn else 0
    if old is None:
        old = {"prefix": np.zeros(nn, np.int32), "partner": np.zeros(1, np.int32), "spring": np.zeros((1, 3))}
    out = {"count": count, "prefix": prefix, "spring": np.zeros((nc, 3)), "point": np.zeros((nc, 3)),
           "normal": np.zeros((nc, 3)), "overlap": np.zeros(nc), "node": np.zeros(nc, np.int64),
           "partner": np.zeros(nc, np.int32), "owner": np.zeros(nc, np.int32)}
    op, opa, osp = i32(old["prefix"]), i32(old["partner"]), f64(old["spring"], (-1, 3))
    if len(opa) == 0:
        opa, osp = np.zeros(1, np.int32), np.zeros((1, 3))
    lib.ora_detect_write(int(mode), C.byref(nodes.s), _d(ppos), _d(pquat), C.byref(B.s), C.byref(G), int(p0), int(p1),
                         _i(prefix), _i(op), _i(opa), _d(osp), int(flags), _d(out["spring"]), _d(out["point"]),
                         _d(out["normal"]), _d(out["overlap"]), _l(out["node"]), _i(out["partner"]),
                         _i(out["owner"]))
    return out


class DynSet:
    def __init__(self, pos, vel, angvel, invmass=None, kn=None, ks=None, mu=None, res=None):
        n = len(pos)
        z = np.zeros(n)
        self.arrs = [f64(pos, (-1, 3)), f64(vel, (-1, 3)), f64(angvel, (-1, 3))] + \
                    [f64(z if a is None else a) for a in (invmass, kn, ks, mu, res)]
        self.s = Dyn(n, *[_d(a) for a in self.arrs])


def contact_force(kind, c, P: DynSet, J: DynSet, dt, force, torque, flags=0, nthreads=1):
    nc = len(c["overlap"])
    en_n = np.zeros(nc)
    en_s = np.zeros(nc)
    if nc:
        lib.ora_contact_force(int(kind), nc, _i(i32(c["owner"])), _i(i32(c["partner"])), _d(f64(c["point"])),
                              _d(f64(c["normal"])), _d(f64(c["overlap"])), _d(c["spring"]), _d(en_n), _d(en_s),
                              C.byref(P.s), C.byref(J.s), float(dt), int(flags), _d(force), _d(torque), int(nthreads))
    c["en_n"], c["en_s"] = en_n, en_s


def kick(vel, angvel, force, torque, invmass, quat, invI, g, h):
    lib.ora_kick(len(vel), _d(vel), _d(angvel), _d(f64(force)), _d(f64(torque)), _d(f64(invmass)), _d(f64(quat)),
                 _d(f64(invI)), _d(f64(g)), float(h))


def drift(pos, quat, vel, angvel, dt):
    lib.ora_drift(len(pos), _d(pos), _d(quat), _d(f64(vel)), _d(f64(angvel)), float(dt))


def bond_force(b, pos, quat, force, torque):
    nb = len(b["bonded"])
    if nb:
        lib.ora_bond_force(nb, _i(b["ids"]), _d(b["B"]), _d(b["geo"]), _d(b["frames"]), _i(b["bonded"]),
                           _d(b["state"]), _d(f64(pos)), _d(f64(quat)), _d(force), _d(torque))


# ---------------------------------------------------------------------------
# Whole-step orchestration.


class OracleSim:
    """A full system stepped by the oracle in the reference order.

    model: dict with
      shapes: list of dict(nodes, sdf, size, origin, spacing)
      particles: dict(shape, scale, pos, vel, angvel, quat, inv_mass, inv_inertia, radius, kn, ks, mu, e, origin,
                      invh) (origin/invh per particle as stored by the solver)
      walls: dict(shape, pos, vel, angvel, quat, radius, mu, e, origin, invh) or None
      bonds: dict(ids, B, geo, frames, bonded, state) or None
      domain: (min, max), gravity, periodic axes mask
      grid_cell (optional): particle grid cell size (default 2 x the largest radius)
    """

    def __init__(self, model, flags=0, nthreads=1, literal_wrap_arms=False):
        # literal_wrap_arms=True reproduces the reference's order exactly: particle-particle and
        # particle-wall contacts detected before the periodic wrap but their forces evaluated with
        # positions read after it (LSSolver.h:1104-1118). The default evaluates them with the
        # detection-time positions, as the CUDA step does.
        self.literal_wrap_arms = literal_wrap_arms
        self.flags = flags
        self.nthreads = nthreads
        shapes = model["shapes"]
        offs = np.cumsum([0] + [len(s["sdf"]) for s in shapes])
        self.sdf = np.concatenate([f64(s["sdf"]) for s in shapes]) if shapes else np.zeros(1)
        noffs = np.cumsum([0] + [len(s["nodes"]) for s in shapes])
        self.node_store = np.concatenate([f64(s["nodes"], (-1, 3)) for s in shapes]) if shapes else np.zeros((1, 3))
        self.shapes = shapes
        p = model["particles"]
        self.P = {k: np.array(v, copy=True) for k, v in p.items()}
        sh = i32(p["shape"])
        self.np_ = len(sh)
        self.sdf_off = offs[sh].astype(np.int64)
        self.gsize = np.array([shapes[s]["size"] for s in sh], np.int32).reshape(-1, 3)
        cnt = np.array([len(shapes[s]["nodes"]) for s in sh], np.int64)
        self.node_base = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
        self.nodes = NodeSet(self.node_base, noffs[sh].astype(np.int64), self.node_store, self.P.get("scale"))
        self.W = None if model.get("walls") is None else {k: np.array(v, copy=True) for k, v in model["walls"].items()}
        self.bonds = None if model.get("bonds") is None else {k: np.array(v, copy=True) for k, v in model["bonds"].items()}
        self.dmin, self.dmax = f64(model["domain"][0]), f64(model["domain"][1])
        self.gravity = f64(model.get("gravity", np.zeros(3)))
        self.periodic = int(model.get("periodic", 0))
        self.F = np.zeros((self.np_, 3))
        self.T = np.zeros((self.np_, 3))
        rp = float(np.max(self.P["radius"])) if self.np_ else 0.0
        # grid_cell: the cell size of a larger system this model is a part of (a spatial
        # sub-box keeps the whole system's grid, so keys and windows are the same)
        cell = float(model["grid_cell"]) if model.get("grid_cell") else (2.0 * rp if self.np_ else 0.0)
        self.pg = grid_set(self.dmin, self.dmax, cell)
        if self.W is not None and len(self.W["pos"]):
            self.wg = grid_set(self.dmin, self.dmax, 2.0 * float(np.max(self.W["radius"])))
            self.w_sdf_off = offs[i32(self.W["shape"])].astype(np.int64)
            self.w_gsize = np.array([shapes[s]["size"] for s in self.W["shape"]], np.int32).reshape(-1, 3)
        self.old = {}
        self.last = {}
        self.time = 0.0

    def _bodies(self, pos=None, quat=None):
        P = self.P
        return BodySet(P["pos"] if pos is None else pos, P["quat"] if quat is None else quat, P["radius"], P["invh"],
                       P["origin"], self.gsize, self.sdf_off, self.sdf, P.get("scale"))

    def _list(self, name, mode, B, g, key):
        sr = sort_ranges(key, int(np.prod(g["size"])))
        c = detect(mode, self.nodes, self.P["pos"], self.P["quat"], B, g, sr["sorted_idx"], sr["start"], sr["end"],
                   self.old.get(name), self.flags)
        self.old[name] = {"prefix": c["prefix"], "partner": c["partner"], "spring": c["spring"]}
        self.last[name] = c
        return c, sr

    def detect_all(self):
        """Hash + detection of all lists on the current state (no forces)."""
        P = self.P
        key = hash_keys(P["pos"], self.pg)
        self.last_hash = {"key": key}
        c, sr = self._list("pp", 0, self._bodies(), self.pg, key)
        self.last_hash.update(sr)
        if self.W is not None and len(self.W["pos"]):
            W = self.W
            WB = BodySet(W["pos"], W["quat"], W["radius"], W["invh"], W["origin"], self.w_gsize, self.w_sdf_off,
                         self.sdf)
            self._list("pw", 1, WB, self.wg, hash_keys(W["pos"], self.wg))
        if self.periodic:
            self._periodic_detect()

    def _periodic_detect(self):
        P = self.P
        g = self.pg
        self.pos_detect = P["pos"].copy()
        self.ghost_pos = {}
        self.ghost_vel, self.ghost_quat = {}, {}
        if self.periodic & 8:
            # sector: wrap (position, velocity, orientation), then the three turned image sets
            self.vel_detect = P["vel"].copy()
            self.quat_detect = P["quat"].copy()
            sector_wrap(P["pos"], P["vel"], P["quat"], g)
            gp, gv, gq = sector_ghosts(P["pos"], P["vel"], P["quat"], g)
            for s, m in enumerate((8, 16, 32)):
                self.ghost_pos[m], self.ghost_vel[m], self.ghost_quat[m] = gp[s], gv[s], gq[s]
                GB = self._bodies(pos=gp[s], quat=gq[s])
                self._list(f"g{m}", 1, GB, g, hash_keys(gp[s], g, ghost=True))
            return
        order = [1, 2, 4, 3, 5, 6, 7]
        sets = [m for m in order if (m & self.periodic) == m]
        for ax in range(3):
            if not (self.periodic >> ax) & 1:
                continue
            wrap(P["pos"], g, ax)
            for m in sets:
                if m == (1 << ax):
                    self.ghost_pos[m] = ghost_positions(P["pos"], g, m)
        for m in sets:
            if bin(m).count("1") >= 2:
                self.ghost_pos[m] = ghost_positions(P["pos"], g, m)
        for m in sets:
            gp = self.ghost_pos[m]
            GB = self._bodies(pos=gp)
            self._list(f"g{m}", 1, GB, g, hash_keys(gp, g, ghost=True))

    def forces(self, dt):
        P = self.P
        self.F[:] = 0.0
        self.T[:] = 0.0
        pos_pp = P["pos"]
        vel_pp = P["vel"]
        if self.periodic and not self.literal_wrap_arms:
            pos_pp = self.pos_detect
            if self.periodic & 8:
                vel_pp = self.vel_detect
        PD = DynSet(pos_pp, vel_pp, P["angvel"], P["inv_mass"], P["kn"], P["ks"], P["mu"], P["e"])
        contact_force(0, self.last["pp"], PD, PD, dt, self.F, self.T, self.flags, self.nthreads)
        if "pw" in self.last:
            W = self.W
            WD = DynSet(W["pos"], W["vel"], W["angvel"], None, None, None, W["mu"], W["e"])
            contact_force(1, self.last["pw"], PD, WD, dt, self.F, self.T, self.flags, self.nthreads)
        if self.periodic & 8 and not self.literal_wrap_arms:
            # the wrapped particles' forces and torques turn with them (same wrap, pre-wrap state)
            sector_wrap(self.pos_detect.copy(), self.vel_detect.copy(), self.quat_detect.copy(), self.pg,
                        self.F, self.T)
        if self.periodic:
            PW = DynSet(P["pos"], P["vel"], P["angvel"], P["inv_mass"], P["kn"], P["ks"], P["mu"], P["e"])
            for m, gp in self.ghost_pos.items():
                gv = self.ghost_vel.get(m, P["vel"])  # sector images: turned velocity; angular velocity not turned
                GD = DynSet(gp, gv, P["angvel"], P["inv_mass"], P["kn"], P["ks"], P["mu"], P["e"])
                contact_force(2, self.last[f"g{m}"], PW, GD, dt, self.F, self.T, self.flags, self.nthreads)
        if self.bonds is not None:
            bond_force(self.bonds, P["pos"], P["quat"], self.F, self.T)

    def step(self, dt, hook=None):
        P = self.P
        kick(P["vel"], P["angvel"], self.F, self.T, P["inv_mass"], P["quat"], P["inv_inertia"], self.gravity, 0.5 * dt)
        drift(P["pos"], P["quat"], P["vel"], P["angvel"], dt)
        if self.W is not None and len(self.W["pos"]):
            drift(self.W["pos"], self.W["quat"], self.W["vel"], self.W["angvel"], dt)
        self.detect_all()
        self.forces(dt)
        if hook is not None:
            hook(self, self.time)
        kick(P["vel"], P["angvel"], self.F, self.T, P["inv_mass"], P["quat"], P["inv_inertia"], self.gravity, 0.5 * dt)
        self.time += dt


def model_from_solver(sv, with_walls=True):
    """Snapshot of a lsdem Solver's model (same inputs for the oracle)."""
    pp = sv.particle_params()
    st = sv.state()
    nshape = sv.num(4)
    shapes = [sv.shape(k) for k in range(nshape)]
    particles = {"shape": pp["shape"], "scale": pp["scale"], "pos": st["pos"], "vel": st["vel"],
                 "angvel": st["angvel"], "quat": st["quat"], "inv_mass": pp["inv_mass"],
                 "inv_inertia": pp["inv_inertia"], "radius": pp["radius"], "kn": pp["kn"], "ks": pp["ks"],
                 "mu": pp["mu"], "e": pp["e"], "origin": pp["origin"], "invh": pp["invh"]}
    walls = None
    if with_walls and sv.n_walls:
        wp = sv.wall_params()
        ws = sv.wall_state()
        walls = {"shape": wp["shape"], "pos": ws["pos"], "vel": ws["vel"], "angvel": ws["angvel"], "quat": ws["quat"],
                 "radius": wp["radius"], "mu": wp["mu"], "e": wp["e"], "origin": wp["origin"], "invh": wp["invh"]}
    bonds = None
    if sv.num(2):
        b, bp = sv.bonds(), sv.bond_params()
        bonds = {"ids": b["ids"], "B": bp["B"], "geo": bp["geo"], "frames": bp["frames"], "bonded": b["bonded"],
                 "state": b["state"]}
    return {"shapes": shapes, "particles": particles, "walls": walls, "bonds": bonds}


def model_from_scene(sc):
    """The oracle model of a multi-template scene dict (the scenes module's layout), built on
    the host with the solver's set-up rules and no device: per-particle grid origin scaled
    and inverse spacing 1 / (scale h), bounding radius max |scale * node|
    (LSParticle.h:175-181), quaternions normalised, kn / ks / mu clamped at 0, restitution
    outside (0, 1] set to 1 (LSParticle.h:193-202); wall radius = largest vertex distance
    (LSSolver.h:255-271)."""
    T = sc["templates"]
    shapes = [{"nodes": f64(t["nodes"], (-1, 3)), "sdf": f64(t["sdf"]), "size": i32(t["size"]),
               "origin": f64(t["origin"]), "spacing": float(t["spacing"])} for t in T]
    sh = i32(sc["shape"])
    n = len(sh)
    scale = f64(sc["scale"])
    cache = {}

    def body_radius(s, c):
        if (s, c) not in cache:
            p = shapes[s]["nodes"] * c if c != 1.0 else shapes[s]["nodes"]
            cache[(s, c)] = float(np.max(np.sqrt(p[:, 0] * p[:, 0] + p[:, 1] * p[:, 1] + p[:, 2] * p[:, 2])))
        return cache[(s, c)]
    radius = np.array([body_radius(int(sh[i]), float(scale[i])) for i in range(n)])
    origin = np.array([shapes[s]["origin"] * (scale[i] if scale[i] != 1.0 else 1.0) for i, s in enumerate(sh)])
    invh = np.array([1.0 / (shapes[s]["spacing"] * scale[i] if scale[i] != 1.0 else shapes[s]["spacing"])
                     for i, s in enumerate(sh)])
    q = f64(sc["quat"], (-1, 4))
    q = q / np.sqrt((q ** 2).sum(axis=1))[:, None]
    full = lambda v: np.full(n, float(v)) if np.ndim(v) == 0 else f64(v)
    res = full(sc["e"])
    res = np.where((res <= 0.0) | (res > 1.0), 1.0, res)
    particles = {"shape": sh, "scale": scale, "pos": f64(sc["pos"], (-1, 3)).copy(),
                 "vel": f64(sc.get("vel", np.zeros((n, 3))), (-1, 3)).copy(),
                 "angvel": f64(sc.get("angvel", np.zeros((n, 3))), (-1, 3)).copy(), "quat": q,
                 "inv_mass": f64(sc["inv_mass"]), "inv_inertia": f64(sc["inv_inertia"], (-1, 6)),
                 "radius": radius, "kn": np.maximum(full(sc["kn"]), 0.0), "ks": np.maximum(full(sc["ks"]), 0.0),
                 "mu": np.maximum(full(sc["mu"]), 0.0), "e": res, "origin": origin, "invh": invh}
    walls = None
    if sc.get("walls"):
        W = sc["walls"]
        k0 = len(shapes)
        for w in W:
            shapes.append({"nodes": np.zeros((0, 3)), "sdf": f64(w["sdf"]), "size": i32(w["size"]),
                           "origin": f64(w["origin"]), "spacing": float(w["spacing"])})
        wq = np.array([f64(w["quat"]) / np.sqrt((f64(w["quat"]) ** 2).sum()) for w in W])
        walls = {"shape": np.arange(k0, k0 + len(W), dtype=np.int32),
                 "pos": np.array([f64(w["pos"]) for w in W]),
                 "vel": np.array([f64(w.get("vel", np.zeros(3)) if w.get("vel") is not None else np.zeros(3))
                                  for w in W]),
                 "angvel": np.array([f64(w.get("angvel", np.zeros(3)) if w.get("angvel") is not None
                                         else np.zeros(3)) for w in W]),
                 "quat": wq, "radius": np.array([float(np.max(np.sqrt((f64(w["verts"], (-1, 3)) ** 2).sum(1))))
                                                 for w in W]),
                 "mu": np.array([max(float(w["mu"]), 0.0) for w in W]),
                 "e": np.array([float(w["e"]) if 0.0 < float(w["e"]) <= 1.0 else 1.0 for w in W]),
                 "origin": np.array([f64(w["origin"]) for w in W]),
                 "invh": np.array([1.0 / float(w["spacing"]) for w in W])}
    return {"shapes": shapes, "particles": particles, "walls": walls, "bonds": None,
            "domain": (f64(sc["min"]), f64(sc["max"])), "gravity": f64(sc["gravity"]),
            "periodic": int(sc.get("periodic", 0))}
