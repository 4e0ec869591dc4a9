"""Python binding of the B200 level-set DEM step (ctypes over include/lsdem_b200.h).

The compute path is the CUDA library liblsdem_b200.so built from csrc/; there
is no CPU fallback: importing this module fails loudly when the library is
missing. The Solver class mirrors the reference solver's app-facing API
(FunDEM/kernel/LSSolver.h): add_ls_particle ~ addLSParticle, add_wall ~ addWall,
add_bond ~ addBondedInteraction, set_periodic ~ addPeriodicBoundary{XD,YD},
initialize + step ~ solve's upload and step loop.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "liblsdem_b200.so"

OK = 0
FIX_GRADIENT = 1
FIX_SQRTF = 2
CONTACT_PARTICLE, CONTACT_WALL, CONTACT_GHOST = 0, 1, 2
PREC_FP64, PREC_FP32_FP16, PREC_FP32_BF16 = 0, 1, 2

_ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "out of device memory", 4: "call out of order",
           5: "no CUDA device"}


class LSDEMError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"lsdem error {code} ({_ERRORS.get(code, '?')}): {msg}")
        self.code = code


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python lsdem2.0_b200/build.py` "
                          "(the CUDA library is the only compute path)")
    return C.CDLL(str(LIB_PATH))


lib = _load()

P = C.c_void_p
DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)
LP = C.POINTER(C.c_longlong)
FP = C.POINTER(C.c_float)
HOOK = C.CFUNCTYPE(None, C.c_void_p, C.c_double)

_SIGS = {
    "lsdem_create": (C.c_int, [C.c_int, P, C.POINTER(P)]),
    "lsdem_destroy": (None, [P]),
    "lsdem_last_error": (C.c_char_p, [P]),
    "lsdem_set_flags": (C.c_int, [P, C.c_int]),
    "lsdem_mass_properties": (C.c_int, [DP, IP, DP, C.c_double, C.c_double, DP]),
    "lsdem_add_shape": (C.c_int, [P, DP, C.c_int, DP, IP, DP, C.c_double, IP]),
    "lsdem_add_particles": (C.c_int, [P, C.c_int, IP, DP, DP, DP, DP, DP, DP, DP, DP, DP, DP, DP, IP]),
    "lsdem_add_ls_particle": (C.c_int, [P, DP, C.c_int, DP, IP, DP, C.c_double, DP, DP, DP, DP, C.c_double,
                                        C.c_double, C.c_double, C.c_double, C.c_double, IP]),
    "lsdem_add_wall": (C.c_int, [P, DP, C.c_int, DP, IP, DP, C.c_double, DP, DP, C.c_double, C.c_double, IP]),
    "lsdem_move_particle": (C.c_int, [P, C.c_int, DP]),
    "lsdem_move_wall": (C.c_int, [P, C.c_int, DP]),
    "lsdem_set_wall_velocity": (C.c_int, [P, C.c_int, DP]),
    "lsdem_set_wall_angular_velocity": (C.c_int, [P, C.c_int, DP]),
    "lsdem_add_bond": (C.c_int, [P, C.c_int, C.c_int, DP, DP, C.c_double, C.c_double, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_double]),
    "lsdem_create_bonds_from_contacts": (C.c_int, [P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                                   C.c_double, C.c_double]),
    "lsdem_set_periodic": (C.c_int, [P, C.c_int]),
    "lsdem_set_precision": (C.c_int, [P, C.c_int]),
    "lsdem_initialize": (C.c_int, [P, DP, DP, DP]),
    "lsdem_step": (C.c_int, [P, C.c_double, C.c_longlong, HOOK, P]),
    "lsdem_set_record_contacts": (C.c_int, [P, C.c_int]),
    "lsdem_set_capacity": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_longlong, C.c_int]),
    "lsdem_num": (C.c_longlong, [P, C.c_int]),
    "lsdem_time": (C.c_double, [P]),
    "lsdem_get_state": (C.c_int, [P, DP, DP, DP, DP, DP, DP]),
    "lsdem_get_wall_state": (C.c_int, [P, DP, DP, DP, DP]),
    "lsdem_set_state": (C.c_int, [P, DP, DP, DP, DP]),
    "lsdem_get_particle_params": (C.c_int, [P, DP, DP, DP, DP, DP, DP, DP, IP, DP, DP, DP, LP]),
    "lsdem_get_wall_params": (C.c_int, [P, DP, DP, DP, IP, DP, DP]),
    "lsdem_get_shape": (C.c_int, [P, C.c_int, DP, DP, IP, DP, DP, IP]),
    "lsdem_get_grid": (C.c_int, [P, DP, DP, DP, IP]),
    "lsdem_get_wall_grid": (C.c_int, [P, DP, DP, DP, IP]),
    "lsdem_get_hash": (C.c_int, [P, IP, IP, IP, IP, IP]),
    "lsdem_count_contacts": (C.c_int, [P, C.c_int, LP]),
    "lsdem_get_contacts": (C.c_int, [P, C.c_int, C.c_longlong, LP, IP, IP, DP, DP, DP, DP, DP, DP]),
    "lsdem_get_bonds": (C.c_int, [P, IP, IP, DP]),
    "lsdem_device_pointers": (C.c_int, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(P),
                                        C.POINTER(P)]),
    "lsdem_stream": (P, [P]),
    "lsdem_set_profiling": (C.c_int, [P, C.c_int]),
    "lsdem_get_profile": (C.c_int, [P, DP, LP]),
    "lsdem_step_stats": (C.c_int, [P, LP]),
    "lsdem_set_screen_stats": (C.c_int, [P, C.c_int]),
    "lsdem_set_step_timing": (C.c_int, [P, C.c_int, C.c_longlong]),
    "lsdem_get_bond_params": (C.c_int, [P, DP, DP, DP]),
    "lsdem_train_learned_sdf": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_ulonglong, DP, DP]),
    "lsdem_set_learned_sdf": (C.c_int, [P, C.c_int]),
    "lsdem_set_learned_training": (C.c_int, [P, C.c_double, C.c_double, C.c_double]),
    "lsdem_get_learned_sdf": (C.c_int, [P, C.c_int, FP, FP]),
    "lsdem_mlp_eval": (C.c_int, [P, C.c_int, C.c_int, DP, FP]),
    "lsdem_mlp_gradient": (C.c_int, [C.c_int, C.c_int, FP, FP, FP, FP, FP]),
    "lsdem_get_screen_stats": (C.c_int, [P, LP]),
    "lsdem_get_screen_queue": (C.c_int, [P, LP]),
    "lsdem_pack_rsa": (C.c_int, [C.c_int, DP, DP, DP, C.c_int, C.c_ulonglong, C.c_int, IP, DP]),
    "lsdem_cell_sort_static": (C.c_int, [P, C.c_int, DP, DP, DP, IP, P, P, P, P, P, P]),
    "lsdem_mesh_grid_box": (C.c_int, [DP, C.c_int, C.c_double, C.c_int, DP, IP]),
    "lsdem_set_triangles": (C.c_int, [P, C.c_int, C.c_int, IP, C.c_int]),
    "lsdem_set_graphs": (C.c_int, [P, C.c_int]),
    "lsdem_set_neighbour_lists": (C.c_int, [P, C.c_int]),
    "lsdem_write_vtu": (C.c_int, [P, C.c_char_p, C.c_ulonglong, C.c_ulonglong, C.c_double]),
    "lsdem_mesh_grid": (C.c_int, [DP, C.c_int, IP, C.c_int, DP, IP, C.c_double, C.c_int, DP, C.c_int]),
    "lsdem_mass_properties_gpu": (C.c_int, [DP, IP, DP, C.c_double, C.c_double, DP, C.c_int]),
    "lsdem_snapshot_save": (C.c_int, [P, C.c_char_p]),
    "lsdem_snapshot_load": (C.c_int, [P, C.c_char_p]),
}
for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = sorted(_SIGS)


def _d(a):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.ctypes.data_as(DP)


def _i(a):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a.ctypes.data_as(IP)


def _dp(a):  # pointer into a writable float64 array
    return None if a is None else a.ctypes.data_as(DP)


def _ip(a):
    return None if a is None else a.ctypes.data_as(IP)


MLP_PARAMS = 4484


def mlp_gradient(params, pts, device=0):
    """Loss (mean squared error), its gradient and the FP32 forward output of one network
    over points (n x 4: x, y, z, target; n a multiple of 128), from the training kernel."""
    params = np.ascontiguousarray(params, np.float32)
    pts = np.ascontiguousarray(pts, np.float32)
    loss = np.zeros(1, np.float32)
    grad = np.zeros(MLP_PARAMS, np.float32)
    y = np.zeros(len(pts), np.float32)
    rc = lib.lsdem_mlp_gradient(int(device), len(pts), params.ctypes.data_as(FP), pts.ctypes.data_as(FP),
                                loss.ctypes.data_as(FP), grad.ctypes.data_as(FP), y.ctypes.data_as(FP))
    if rc:
        raise LSDEMError(rc, "mlp_gradient")
    return float(loss[0]), grad, y


def pack_rsa(radius, lo, hi, periodic=False, seed=12345, max_tries=1000, keep=None, pos=None):
    """Random sequential addition of spheres with the given radii (placed in order); with `keep`,
    spheres where keep is nonzero stay at `pos` and the others are placed around them."""
    r = np.ascontiguousarray(radius, np.float64)
    out = np.zeros((len(r), 3)) if pos is None else np.array(pos, np.float64, copy=True, order="C")
    kp = None if keep is None else np.ascontiguousarray(keep, np.int32)
    rc = lib.lsdem_pack_rsa(len(r), _d(r), _d(lo), _d(hi), 1 if periodic else 0, int(seed), int(max_tries),
                            _ip(kp), _dp(out))
    if rc:
        raise LSDEMError(rc, "pack_rsa: could not place every sphere")
    return out


def mass_properties(sdf, size, origin, spacing, density):
    """Mass, centroid, inertia and inverse inertia by smoothed-Heaviside integration (LSSolver.h:66-135)."""
    sdf = np.ascontiguousarray(sdf, dtype=np.float64).ravel()
    out = np.zeros(16)
    rc = lib.lsdem_mass_properties(_d(sdf), _i(np.asarray(size, np.int32)), _d(origin), float(spacing),
                                   float(density), _dp(out))
    if rc:
        raise LSDEMError(rc, "mass_properties")
    return {"mass": out[0], "centroid": out[1:4].copy(), "inertia": out[4:10].copy(), "inv_inertia": out[10:16].copy()}


def mass_properties_gpu(sdf, size, origin, spacing, density, device=0):
    """mass_properties computed on the GPU (parallel sums; agrees with the host loop to rounding)."""
    sdf = np.ascontiguousarray(sdf, dtype=np.float64).ravel()
    out = np.zeros(16)
    rc = lib.lsdem_mass_properties_gpu(_d(sdf), _i(np.asarray(size, np.int32)), _d(origin), float(spacing),
                                       float(density), _dp(out), int(device))
    if rc:
        raise LSDEMError(rc, "mass_properties_gpu")
    return {"mass": out[0], "centroid": out[1:4].copy(), "inertia": out[4:10].copy(), "inv_inertia": out[10:16].copy()}


def mesh_grid_box(verts, spacing, pad=2):
    """Origin and node counts of the grid buildGrid(spacing, pad) puts around a mesh
    (LevelSetObjectGenerator.h:122-170)."""
    v = np.ascontiguousarray(verts, np.float64).reshape(-1, 3)
    origin = np.zeros(3)
    size = np.zeros(3, np.int32)
    rc = lib.lsdem_mesh_grid_box(_d(v), len(v), float(spacing), int(pad), _dp(origin), _ip(size))
    if rc:
        raise LSDEMError(rc, "mesh_grid_box")
    return origin, size


def mesh_grid(verts, tris, spacing, pad=2, positive_inside=False, device=0, origin=None, size=None):
    """Level-set grid of a closed triangle mesh computed on the GPU (buildGrid over the mesh
    distance with the solid-angle sign, LevelSetObjectGenerator.h:122-224, 454-500, 758-802).
    Returns (sdf, size, origin) with sdf in the order ix + nx (iy + ny iz)."""
    v = np.ascontiguousarray(verts, np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
    if origin is None or size is None:
        origin, size = mesh_grid_box(v, spacing, pad)
    origin = np.ascontiguousarray(origin, np.float64)
    size = np.ascontiguousarray(size, np.int32)
    out = np.zeros(int(np.prod(size.astype(np.int64))))
    rc = lib.lsdem_mesh_grid(_d(v), len(v), _i(t), len(t), _d(origin), _i(size), float(spacing),
                             1 if positive_inside else 0, _dp(out), int(device))
    if rc:
        raise LSDEMError(rc, "mesh_grid")
    return out, size, origin


class Solver:
    """One level-set DEM system on one GPU (owner of an lsdem_solver handle)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        h = P()
        rc = lib.lsdem_create(int(device), P(stream) if stream else None, C.byref(h))
        if rc:
            raise LSDEMError(rc, "create")
        self.h = h
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            lib.lsdem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, what=""):
        if rc:
            raise LSDEMError(rc, f"{what}: {lib.lsdem_last_error(self.h).decode()}")

    # ---- model ---------------------------------------------------------------
    def set_flags(self, flags: int):
        self._chk(lib.lsdem_set_flags(self.h, int(flags)), "set_flags")

    def add_shape(self, nodes, sdf, size, origin, spacing) -> int:
        nodes = np.ascontiguousarray(nodes, np.float64).reshape(-1, 3)
        sid = C.c_int(-1)
        self._chk(lib.lsdem_add_shape(self.h, _d(nodes), len(nodes), _d(np.ravel(sdf)), _i(size), _d(origin),
                                      float(spacing), C.byref(sid)), "add_shape")
        return sid.value

    def add_particles(self, shape, pos, quat, inv_mass, inv_inertia, kn, ks, mu, e, vel=None, angvel=None,
                      scale=None) -> int:
        shape = np.ascontiguousarray(shape, np.int32).ravel()
        n = len(shape)
        bc = lambda v: np.ascontiguousarray(np.broadcast_to(np.asarray(v, np.float64), (n,)))
        first = C.c_int(-1)
        self._chk(lib.lsdem_add_particles(
            self.h, n, _i(shape), _d(scale), _d(np.reshape(pos, (n, 3))), _d(None if vel is None else np.reshape(vel, (n, 3))),
            _d(None if angvel is None else np.reshape(angvel, (n, 3))), _d(np.reshape(quat, (n, 4))), _d(bc(inv_mass)),
            _d(np.reshape(inv_inertia, (n, 6))), _d(bc(kn)), _d(bc(ks)), _d(bc(mu)), _d(bc(e)), C.byref(first)),
            "add_particles")
        return first.value

    def add_ls_particle(self, nodes, sdf, size, origin, spacing, pos, vel, angvel, quat, kn, ks, mu, e, density) -> int:
        nodes = np.ascontiguousarray(nodes, np.float64).reshape(-1, 3)
        idx = C.c_int(-1)
        self._chk(lib.lsdem_add_ls_particle(self.h, _d(nodes), len(nodes), _d(np.ravel(sdf)), _i(size), _d(origin),
                                            float(spacing), _d(pos), _d(vel), _d(angvel), _d(quat), float(kn),
                                            float(ks), float(mu), float(e), float(density), C.byref(idx)),
                  "add_ls_particle")
        return idx.value

    def add_wall(self, verts, sdf, size, origin, spacing, pos, quat, mu, e=1.0) -> int:
        verts = np.ascontiguousarray(verts, np.float64).reshape(-1, 3)
        idx = C.c_int(-1)
        self._chk(lib.lsdem_add_wall(self.h, _d(verts), len(verts), _d(np.ravel(sdf)), _i(size), _d(origin),
                                     float(spacing), _d(pos), _d(quat), float(mu), float(e), C.byref(idx)), "add_wall")
        return idx.value

    def set_wall_velocity(self, i, v):
        self._chk(lib.lsdem_set_wall_velocity(self.h, int(i), _d(v)), "set_wall_velocity")

    def set_wall_angular_velocity(self, i, w):
        self._chk(lib.lsdem_set_wall_angular_velocity(self.h, int(i), _d(w)), "set_wall_angular_velocity")

    def add_bond(self, master, slave, point, normal, radius, length, youngs, poisson, tensile=0.0, cohesion=0.0,
                 mu=0.0):
        self._chk(lib.lsdem_add_bond(self.h, int(master), int(slave), _d(point), _d(normal), float(radius),
                                     float(length), float(youngs), float(poisson), float(tensile), float(cohesion),
                                     float(mu)), "add_bond")

    def create_bonds_from_contacts(self, radius, length, youngs, poisson, tensile=0.0, cohesion=0.0, mu=0.0):
        self._chk(lib.lsdem_create_bonds_from_contacts(self.h, float(radius), float(length), float(youngs),
                                                       float(poisson), float(tensile), float(cohesion), float(mu)),
                  "create_bonds_from_contacts")

    def set_precision(self, mode: int):
        """PREC_FP64 (default), PREC_FP32_FP16 or PREC_FP32_BF16; takes effect at initialize."""
        self._chk(lib.lsdem_set_precision(self.h, int(mode)), "set_precision")

    def set_periodic(self, axes: int):
        self._chk(lib.lsdem_set_periodic(self.h, int(axes)), "set_periodic")

    def set_graphs(self, on=True):
        """Replay steps from a CUDA graph (default) or launch every kernel."""
        self._chk(lib.lsdem_set_graphs(self.h, 1 if on else 0), "set_graphs")

    def set_neighbour_lists(self, on=True):
        """Reuse per-particle neighbour lists between steps (default; exact), sorting the
        cells only when lists are rebuilt, or sort and walk the 27 cells every step."""
        self._chk(lib.lsdem_set_neighbour_lists(self.h, 1 if on else 0), "set_neighbour_lists")

    def snapshot_save(self, path):
        """Writes the dynamic state and contact history to a binary snapshot file."""
        self._chk(lib.lsdem_snapshot_save(self.h, str(path).encode()), "snapshot_save")

    def snapshot_load(self, path):
        """Restores a snapshot into this (initialized, same-model) solver."""
        self._chk(lib.lsdem_snapshot_load(self.h, str(path).encode()), "snapshot_load")

    def set_triangles(self, kind, index, tris):
        """Triangles of a body's nodes (kind 0 particle, 1 wall) for the mesh output files."""
        t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
        self._chk(lib.lsdem_set_triangles(self.h, int(kind), int(index), _i(t), len(t)), "set_triangles")

    def write_vtu(self, directory, frame, step, time):
        """The reference's output files of one frame under `directory` (LSSolver::output)."""
        self._chk(lib.lsdem_write_vtu(self.h, str(directory).encode(), int(frame), int(step), float(time)),
                  "write_vtu")

    def set_capacity(self, pp=0, wall=0, ghost=0, contacts=0, batch=0):
        self._chk(lib.lsdem_set_capacity(self.h, int(pp), int(wall), int(ghost), int(contacts), int(batch)),
                  "set_capacity")

    def set_record_contacts(self, on=True):
        self._chk(lib.lsdem_set_record_contacts(self.h, 1 if on else 0), "set_record_contacts")

    # ---- run -----------------------------------------------------------------
    def initialize(self, dmin, dmax, gravity=(0.0, 0.0, 0.0)):
        self._chk(lib.lsdem_initialize(self.h, _d(dmin), _d(dmax), _d(gravity)), "initialize")

    def step(self, dt: float, nsteps: int = 1, hook=None):
        """hook(time) is called after the contact/bond forces of each step, before the second half kick."""
        if hook is None:
            cb = HOOK()
        else:
            cb = HOOK(lambda _u, t: hook(t))
        self._keep = [cb]
        self._chk(lib.lsdem_step(self.h, float(dt), int(nsteps), cb, None), "step")

    # ---- queries -------------------------------------------------------------
    def num(self, what: int) -> int:
        return int(lib.lsdem_num(self.h, what))

    @property
    def n_particles(self):
        return self.num(0)

    @property
    def n_walls(self):
        return self.num(1)

    @property
    def time(self):
        return float(lib.lsdem_time(self.h))

    def state(self):
        n = self.n_particles
        out = {k: np.zeros((n, 3)) for k in ("pos", "vel", "angvel", "force", "torque")}
        out["quat"] = np.zeros((n, 4))
        self._chk(lib.lsdem_get_state(self.h, _dp(out["pos"]), _dp(out["vel"]), _dp(out["angvel"]),
                                      _dp(out["quat"]), _dp(out["force"]), _dp(out["torque"])), "get_state")
        return out

    def wall_state(self):
        n = self.n_walls
        out = {k: np.zeros((n, 3)) for k in ("pos", "vel", "angvel")}
        out["quat"] = np.zeros((n, 4))
        self._chk(lib.lsdem_get_wall_state(self.h, _dp(out["pos"]), _dp(out["vel"]), _dp(out["angvel"]),
                                           _dp(out["quat"])), "get_wall_state")
        return out

    def set_state(self, pos=None, vel=None, angvel=None, quat=None):
        self._chk(lib.lsdem_set_state(self.h, _d(pos), _d(vel), _d(angvel), _d(quat)), "set_state")

    def particle_params(self):
        n = self.n_particles
        o = {k: np.zeros(n) for k in ("inv_mass", "radius", "kn", "ks", "mu", "e", "scale", "invh")}
        o["inv_inertia"] = np.zeros((n, 6))
        o["origin"] = np.zeros((n, 3))
        o["shape"] = np.zeros(n, np.int32)
        o["node_base"] = np.zeros(n, np.int64)
        self._chk(lib.lsdem_get_particle_params(
            self.h, _dp(o["inv_mass"]), _dp(o["inv_inertia"]), _dp(o["radius"]), _dp(o["kn"]), _dp(o["ks"]),
            _dp(o["mu"]), _dp(o["e"]), _ip(o["shape"]), _dp(o["scale"]), _dp(o["origin"]), _dp(o["invh"]),
            o["node_base"].ctypes.data_as(LP)), "get_particle_params")
        return o

    def wall_params(self):
        n = self.n_walls
        o = {k: np.zeros(n) for k in ("radius", "mu", "e", "invh")}
        o["origin"] = np.zeros((n, 3))
        o["shape"] = np.zeros(n, np.int32)
        self._chk(lib.lsdem_get_wall_params(self.h, _dp(o["radius"]), _dp(o["mu"]), _dp(o["e"]), _ip(o["shape"]),
                                            _dp(o["origin"]), _dp(o["invh"])), "get_wall_params")
        return o

    def shape(self, sid: int):
        size = np.zeros(3, np.int32)
        origin = np.zeros(3)
        h = C.c_double()
        nn = C.c_int()
        self._chk(lib.lsdem_get_shape(self.h, sid, None, None, _ip(size), _dp(origin), C.byref(h), C.byref(nn)),
                  "get_shape")
        nodes = np.zeros((nn.value, 3))
        sdf = np.zeros(int(np.prod(size)))
        self._chk(lib.lsdem_get_shape(self.h, sid, _dp(nodes), _dp(sdf), None, None, None, None), "get_shape")
        return {"nodes": nodes, "sdf": sdf, "size": size, "origin": origin, "spacing": h.value}

    def grid(self, walls=False):
        mn, mx, inv = np.zeros(3), np.zeros(3), np.zeros(3)
        size = np.zeros(3, np.int32)
        f = lib.lsdem_get_wall_grid if walls else lib.lsdem_get_grid
        self._chk(f(self.h, _dp(mn), _dp(mx), _dp(inv), _ip(size)), "get_grid")
        return {"min": mn, "max": mx, "inv": inv, "size": size}

    def hash(self):
        n = self.n_particles
        g = self.grid()
        nc = int(np.prod(g["size"]))
        o = {"key": np.zeros(n, np.int32), "sorted_idx": np.zeros(n, np.int32), "sorted_key": np.zeros(n, np.int32),
             "start": np.zeros(nc, np.int32), "end": np.zeros(nc, np.int32)}
        self._chk(lib.lsdem_get_hash(self.h, _ip(o["key"]), _ip(o["sorted_idx"]), _ip(o["sorted_key"]),
                                     _ip(o["start"]), _ip(o["end"])), "get_hash")
        return o

    def contacts(self, kind=CONTACT_PARTICLE, geometry=False):
        n = C.c_longlong()
        self._chk(lib.lsdem_count_contacts(self.h, kind, C.byref(n)), "count_contacts")
        m = n.value
        o = {"node": np.zeros(m, np.int64), "partner": np.zeros(m, np.int32), "image": np.zeros(m, np.int32),
             "spring": np.zeros((m, 3))}
        g = {}
        if geometry:
            g = {"point": np.zeros((m, 3)), "normal": np.zeros((m, 3)), "overlap": np.zeros(m), "en_n": np.zeros(m),
                 "en_s": np.zeros(m)}
            o.update(g)
        self._chk(lib.lsdem_get_contacts(self.h, kind, m, o["node"].ctypes.data_as(LP), _ip(o["partner"]),
                                         _ip(o["image"]), _dp(o["spring"]), _dp(g.get("point")), _dp(g.get("normal")),
                                         _dp(g.get("overlap")), _dp(g.get("en_n")), _dp(g.get("en_s"))),
                  "get_contacts")
        return o

    def bond_params(self):
        nb = self.num(2)
        o = {"B": np.zeros((nb, 4)), "geo": np.zeros((nb, 5)), "frames": np.zeros((nb, 24))}
        self._chk(lib.lsdem_get_bond_params(self.h, _dp(o["B"]), _dp(o["geo"]), _dp(o["frames"])), "get_bond_params")
        return o

    def bonds(self):
        nb = self.num(2)
        ids = np.zeros((nb, 2), np.int32)
        bonded = np.zeros(nb, np.int32)
        state = np.zeros((nb, 9))
        self._chk(lib.lsdem_get_bonds(self.h, _ip(ids), _ip(bonded), _dp(state)), "get_bonds")
        return {"ids": ids, "bonded": bonded, "state": state}

    PHASES = ("kick_drift_keys", "cell_sort", "candidates", "narrowphase", "periodic", "ghost_narrowphase", "bonds",
              "kick", "contact_pass", "step", "network")

    def set_step_timing(self, on=True, l2_flush_bytes=0):
        """Per-step CUDA events (profile()["step"]), optionally with an L2 flush before each step."""
        self._chk(lib.lsdem_set_step_timing(self.h, 1 if on else 0, int(l2_flush_bytes)), "set_step_timing")

    def set_profiling(self, on=True):
        self._chk(lib.lsdem_set_profiling(self.h, 1 if on else 0), "set_profiling")

    def profile(self):
        ms = np.zeros(len(self.PHASES))
        calls = np.zeros(len(self.PHASES), np.int64)
        self._chk(lib.lsdem_get_profile(self.h, _dp(ms), calls.ctypes.data_as(LP)), "get_profile")
        return {k: (float(ms[i]), int(calls[i])) for i, k in enumerate(self.PHASES)}

    def step_stats(self):
        o = np.zeros(4, np.int64)
        self._chk(lib.lsdem_step_stats(self.h, o.ctypes.data_as(LP)), "step_stats")
        return {"pairs_particle": int(o[0]), "pairs_wall": int(o[1]), "pairs_ghost": int(o[2]), "contacts": int(o[3])}

    # ---- learned per-shape SDF ---------------------------------------------------
    def set_learned_training(self, clip_lo=-0.25, clip_hi=0.5, near_fraction=0.5):
        """Training options of the learned SDF: target clip range (units of R) and the share
        of samples drawn near the surface."""
        self._chk(lib.lsdem_set_learned_training(self.h, float(clip_lo), float(clip_hi), float(near_fraction)))

    def train_learned_sdf(self, iterations=3000, batch=4096, samples=1 << 18, lr=3e-3, seed=12345):
        """Trains one network per shape template; returns (loss, err) per shape (err in template units)."""
        ns = self.num(4)
        loss, err = np.zeros(ns), np.zeros(ns)
        self._chk(lib.lsdem_train_learned_sdf(self.h, int(iterations), int(batch), int(samples), float(lr), int(seed),
                                              _dp(loss), _dp(err)), "train_learned_sdf")
        return loss, err

    def set_learned_sdf(self, on=True):
        self._chk(lib.lsdem_set_learned_sdf(self.h, 1 if on else 0), "set_learned_sdf")

    def learned_sdf(self, shape):
        params = np.zeros(MLP_PARAMS, np.float32)
        norm = np.zeros(8, np.float32)
        self._chk(lib.lsdem_get_learned_sdf(self.h, int(shape), params.ctypes.data_as(FP), norm.ctypes.data_as(FP)),
                  "get_learned_sdf")
        return params, {"centre": norm[:3].astype(np.float64), "R": float(norm[3]), "err": float(norm[4]),
                        "threshold_h": float(norm[5]), "err_in": float(norm[6]), "delta": float(norm[7])}

    def mlp_eval(self, shape, pts):
        pts = np.ascontiguousarray(pts, np.float64)
        phi = np.zeros(len(pts), np.float32)
        self._chk(lib.lsdem_mlp_eval(self.h, int(shape), len(pts), _dp(pts), phi.ctypes.data_as(FP)), "mlp_eval")
        return phi

    SCREEN_COUNTERS = ("pairs", "clusters", "clusters_kept", "grid_lookups", "node_tests", "nodes_queued",
                       "net_evals", "subclusters_kept")

    def set_screen_stats(self, on=True):
        self._chk(lib.lsdem_set_screen_stats(self.h, 1 if on else 0), "set_screen_stats")

    def screen_stats(self):
        o = np.zeros(8, np.int64)
        self._chk(lib.lsdem_get_screen_stats(self.h, o.ctypes.data_as(LP)), "get_screen_stats")
        q = np.zeros(3, np.int64)
        self._chk(lib.lsdem_get_screen_queue(self.h, q.ctypes.data_as(LP)), "get_screen_queue")
        out = dict(zip(self.SCREEN_COUNTERS, (int(v) for v in o)))
        out.update(queued_particle=int(q[0]), queued_wall=int(q[1]), queued_image=int(q[2]))
        return out

    def device_pointers(self):
        ptrs = [P() for _ in range(6)]
        self._chk(lib.lsdem_device_pointers(self.h, *[C.byref(p) for p in ptrs]), "device_pointers")
        return dict(zip(("force", "torque", "vel", "angvel", "pos", "quat"), [p.value for p in ptrs]))
