"""Generates the golden vectors of tests/golden/ by running the reference's own
CUDA kernels (oracle/_ref/libfundem_ref.so, built by oracle/build_ref.sh from
the reference sources) on seeded inputs. Needs a CUDA device.

    python tests/golden/make_golden.py OUTDIR

Each .npz holds the inputs handed to a reference launcher (in the reference's
data layout: one SDF copy per body addressed by an inclusive prefix sum, one
surface-node list with a particle id per node) and the launcher's outputs.
tests/test_oracle_golden.py replays the inputs through the CPU oracle.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "tests"))
from conftest import load_package  # noqa: E402

DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)


def d(a):
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(DP)


def ip(a):
    return np.ascontiguousarray(a, np.int32).ctypes.data_as(IP)


def lib():
    L = C.CDLL(str(ROOT / "oracle" / "_ref" / "libfundem_ref.so"))
    for f in ("fref_hash_sort", "fref_detect", "fref_force", "fref_bond", "fref_kick", "fref_drift", "fref_wrap",
              "fref_ghost_pos"):
        getattr(L, f).restype = C.c_int
    return L


def grid_params(mn, mx, cell):
    """spatialGrid::set (FunDEM/kernel/CUDAKernelFunction/myUtility/mySpatialGrid.h:212-240)."""
    mx = np.array(mx, np.float64)
    mn = np.array(mn, np.float64)
    size = np.zeros(3, np.int32)
    inv = np.zeros(3)
    for a in range(3):
        dd = mx[a] - mn[a]
        size[a] = int(dd / cell) if dd > 2.0 * cell else 2
        inv[a] = size[a] / dd
    return mn, mx, inv, size


def hash_case(L, rng, ghost):
    mn, mx, inv, size = grid_params([0.0, 0.0, -0.01], [0.2, 0.1, 0.3], 0.01)
    n = 700
    pos = rng.uniform(-0.02, 0.32, size=(n, 3))
    pos[:50, 0] = mn[0]        # exactly on the lower face
    pos[50:80, 2] = mx[2]      # exactly on the upper face (outside)
    pos[80:120] = pos[200:240]  # duplicates -> equal keys, order must be stable
    if ghost:
        pos[:, 2] = rng.uniform(0.05, 0.3, size=n)  # z above max.y exercises the ghost-key z test
    nc = int(np.prod(size))
    key, idx, st, en = (np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(nc, np.int32), np.zeros(nc, np.int32))
    assert L.fref_hash_sort(int(ghost), n, d(pos), d(mn), d(mx), d(inv), ip(size), nc, ip(key), ip(idx), ip(st),
                            ip(en)) == 0
    return dict(pos=pos, min=mn, max=mx, inv=inv, size=size, key=key, idx=idx, start=st, end=en)


def shapes(scenes):
    return [scenes.make_ellipsoid(ax, n_grid=12, n_nodes=160) for ax in
            ((5e-3, 4e-3, 3e-3), (4.5e-3, 4.5e-3, 2.5e-3), (5e-3, 3e-3, 3e-3))]


def particle_layout(shp, which):
    """Reference layout of particles using templates `which` (per-particle copies)."""
    nodes, pid, sdf, prefix, origin, invh, size, rad = [], [], [], [], [], [], [], []
    tot = 0
    for i, k in enumerate(which):
        s = shp[k]
        nodes.append(s["nodes"])
        pid.append(np.full(len(s["nodes"]), i, np.int32))
        sdf.append(s["sdf"])
        tot += len(s["sdf"])
        prefix.append(tot)
        origin.append(s["origin"])
        invh.append(1.0 / s["spacing"])
        size.append(s["size"])
        rad.append(np.max(np.linalg.norm(s["nodes"], axis=1)))
    return dict(node_local=np.concatenate(nodes), node_pid=np.concatenate(pid), sdf=np.concatenate(sdf),
                prefix=np.array(prefix, np.int32), origin=np.array(origin), invh=np.array(invh),
                gsize=np.array(size, np.int32), radius=np.array(rad))


def detect(L, mode, nodes, pos, quat, bodies, bpos, bquat, grid, old=None):
    mn, inv, size, hidx, st, en = grid
    nn = len(nodes["node_pid"])
    nb = len(bpos)
    nc_cells = int(np.prod(size))
    if old is None:
        old = dict(prefix=np.zeros(nn, np.int32), partner=np.zeros(1, np.int32), spring=np.zeros((1, 3)))
    cap = 200000
    out = dict(count=np.zeros(nn, np.int32), prefix=np.zeros(nn, np.int32), spring=np.zeros((cap, 3)),
               point=np.zeros((cap, 3)), normal=np.zeros((cap, 3)), overlap=np.zeros(cap),
               node=np.zeros(cap, np.int32), partner=np.zeros(cap, np.int32))
    ncon = C.c_int()
    rc = L.fref_detect(mode, nn, d(nodes["node_local"]), ip(nodes["node_pid"]), len(pos), d(pos), d(quat), nb,
                       d(bpos), d(bquat), d(bodies["radius"]), d(bodies["invh"]), d(bodies["origin"]),
                       ip(bodies["gsize"]), ip(bodies["prefix"]), C.c_longlong(len(bodies["sdf"])), d(bodies["sdf"]),
                       d(mn), d(inv), ip(size), nc_cells, ip(hidx), ip(st), ip(en), ip(old["prefix"]),
                       len(old["partner"]), ip(old["partner"]), d(old["spring"]), cap, ip(out["count"]),
                       ip(out["prefix"]), C.byref(ncon), d(out["spring"]), d(out["point"]), d(out["normal"]),
                       d(out["overlap"]), ip(out["node"]), ip(out["partner"]))
    assert rc == 0, rc
    k = ncon.value
    for key in ("spring", "point", "normal", "overlap", "node", "partner"):
        out[key] = out[key][:k].copy()
    return out


def main(outdir):
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    L = lib()
    lsdem = load_package()
    from lsdem_b200 import scenes
    rng = np.random.default_rng(20240601)

    np.savez_compressed(out / "hash_sort.npz", **hash_case(L, rng, ghost=False))
    np.savez_compressed(out / "ghost_hash_sort.npz", **hash_case(L, rng, ghost=True))

    # --- particle-particle and particle-wall narrowphase + forces -----------------
    shp = shapes(scenes)
    m = 4
    n = m ** 3
    which = rng.integers(0, 3, size=n)
    lay = particle_layout(shp, which)
    spacing = 7.5e-3
    ijk = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
    pos = 0.006 + ijk * spacing + rng.uniform(-4e-4, 4e-4, size=(n, 3))
    pos[:, 2] -= pos[:, 2].min() - 3.2e-3
    quat = scenes.random_quaternions(rng, n)
    dmin, dmax = np.zeros(3), np.array([0.04, 0.04, 0.05])
    cell = 2.0 * lay["radius"].max()
    mn, mx, inv, size = grid_params(dmin, dmax, cell)
    nc = int(np.prod(size))
    key, hidx, st, en = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(nc, np.int32), np.zeros(nc, np.int32)
    assert L.fref_hash_sort(0, n, d(pos), d(mn), d(mx), d(inv), ip(size), nc, ip(key), ip(hidx), ip(st), ip(en)) == 0
    grid = (mn, inv, size, hidx, st, en)
    nodes = dict(node_local=lay["node_local"], node_pid=lay["node_pid"])
    # first detection without history, then a second one from slightly moved poses with that history
    first = detect(L, 0, nodes, pos, quat, lay, pos, quat, grid)
    first["spring"] = rng.normal(0, 1e-5, size=first["spring"].shape)
    pos2 = pos + rng.normal(0, 5e-5, size=pos.shape)
    q2 = quat + rng.normal(0, 2e-3, size=quat.shape)
    q2 /= np.linalg.norm(q2, axis=1, keepdims=True)
    assert L.fref_hash_sort(0, n, d(pos2), d(mn), d(mx), d(inv), ip(size), nc, ip(key), ip(hidx), ip(st), ip(en)) == 0
    grid2 = (mn, inv, size, hidx.copy(), st.copy(), en.copy())
    pp = detect(L, 0, nodes, pos2, q2, lay, pos2, q2, grid2,
                old=dict(prefix=first["prefix"], partner=first["partner"], spring=first["spring"]))
    # floor wall (phi = z) in its own grid
    fl = scenes.make_plane_wall((0.04, 0.04), h=0.02)
    wl = dict(radius=np.array([np.max(np.linalg.norm(fl["verts"], axis=1))]), invh=np.array([1.0 / fl["spacing"]]),
              origin=fl["origin"][None], gsize=fl["size"][None].astype(np.int32),
              prefix=np.array([len(fl["sdf"])], np.int32), sdf=fl["sdf"])
    wpos = np.array([[0.02, 0.02, 0.0]])
    wq = np.array([[1.0, 0.0, 0.0, 0.0]])
    wmn, wmx, winv, wsize = grid_params(dmin, dmax, 2.0 * wl["radius"][0])
    wnc = int(np.prod(wsize))
    wk, wi, wst, wen = np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(wnc, np.int32), np.zeros(wnc, np.int32)
    assert L.fref_hash_sort(0, 1, d(wpos), d(wmn), d(wmx), d(winv), ip(wsize), wnc, ip(wk), ip(wi), ip(wst),
                            ip(wen)) == 0
    pw = detect(L, 1, nodes, pos2, q2, wl, wpos, wq, (wmn, winv, wsize, wi, wst, wen))
    # forces
    vel = rng.normal(0, 0.05, size=(n, 3))
    angvel = rng.normal(0, 5.0, size=(n, 3))
    mass = 2500 * 4 / 3 * np.pi * 5e-3 * 4e-3 * 3e-3
    invm = np.full(n, 1.0 / mass)
    invm[5] = 0.0  # a fixed particle
    kn = rng.uniform(5e4, 2e5, size=n)
    ks = 0.8 * kn
    mu = rng.uniform(0.2, 0.6, size=n)
    res = rng.uniform(0.3, 1.0, size=n)
    dt = 1e-6

    def force2(kind, c, jpos=None, jvel=None, jang=None, jmu=None, jres=None):
        nc_ = len(c["overlap"])
        sp = np.ascontiguousarray(c["spring"], np.float64).copy()
        en_n, en_s = np.zeros(max(nc_, 1)), np.zeros(max(nc_, 1))
        F = np.ascontiguousarray(rng.normal(0, 1e-3, size=(n, 3)))
        T = np.ascontiguousarray(rng.normal(0, 1e-6, size=(n, 3)))
        F0, T0 = F.copy(), T.copy()
        nj = 0 if jpos is None else len(jpos)
        z = np.zeros((1, 3))
        args = [np.ascontiguousarray(a, np.float64) for a in
                (c["point"], c["normal"], c["overlap"], pos2, vel, angvel, invm, kn, ks, mu, res,
                 z if jpos is None else jpos, z if jvel is None else jvel, z if jang is None else jang,
                 np.zeros(1) if jmu is None else jmu, np.zeros(1) if jres is None else jres)]
        ints = [np.ascontiguousarray(a, np.int32) for a in (c["node"], c["partner"], lay["node_pid"])]
        rc = L.fref_force(kind, nc_, sp.ctypes.data_as(DP), en_n.ctypes.data_as(DP), en_s.ctypes.data_as(DP),
                          args[0].ctypes.data_as(DP), args[1].ctypes.data_as(DP), args[2].ctypes.data_as(DP),
                          ints[0].ctypes.data_as(IP), ints[1].ctypes.data_as(IP), len(lay["node_pid"]),
                          ints[2].ctypes.data_as(IP), n, *[a.ctypes.data_as(DP) for a in args[3:11]], nj,
                          *[a.ctypes.data_as(DP) for a in args[11:16]], C.c_double(dt), F.ctypes.data_as(DP),
                          T.ctypes.data_as(DP))
        assert rc == 0
        return dict(spring_out=sp, en_n=en_n[:nc_], en_s=en_s[:nc_], force_in=F0, torque_in=T0, force_out=F,
                    torque_out=T)

    fpp = force2(0, pp)
    wvel = np.array([[0.01, -0.02, 0.0]])
    wang = np.array([[0.0, 0.0, 0.5]])
    fpw = force2(1, pw, wpos, wvel, wang, np.array([0.4]), np.array([0.5]))
    # ghost forces: partner positions shifted by one box length in x (images), velocities copied
    gpos = pos2 + np.array([0.04, 0.0, 0.0])
    fpg = force2(2, pp, gpos, vel)
    np.savez_compressed(
        out / "narrowphase.npz", which=which, node_local=lay["node_local"], node_pid=lay["node_pid"], sdf=lay["sdf"],
        prefix=lay["prefix"], origin=lay["origin"], invh=lay["invh"], gsize=lay["gsize"], radius=lay["radius"],
        pos=pos2, quat=q2, grid_min=mn, grid_max=mx, grid_inv=inv, grid_size=size, hidx=grid2[3], hstart=grid2[4],
        hend=grid2[5], old_prefix=first["prefix"], old_partner=first["partner"], old_spring=first["spring"],
        **{f"pp_{k}": v for k, v in pp.items()},
        wall_sdf=wl["sdf"], wall_origin=wl["origin"], wall_invh=wl["invh"], wall_gsize=wl["gsize"],
        wall_radius=wl["radius"], wall_pos=wpos, wall_quat=wq, wgrid_min=wmn, wgrid_max=wmx, wgrid_inv=winv,
        wgrid_size=wsize, whidx=wi, whstart=wst, whend=wen, **{f"pw_{k}": v for k, v in pw.items()},
        vel=vel, angvel=angvel, invm=invm, kn=kn, ks=ks, mu=mu, res=res, dt=dt,
        wall_vel=wvel, wall_angvel=wang, wall_mu=np.array([0.4]), wall_res=np.array([0.5]), ghost_pos=gpos,
        **{f"fpp_{k}": v for k, v in fpp.items()}, **{f"fpw_{k}": v for k, v in fpw.items()},
        **{f"fpg_{k}": v for k, v in fpg.items()})

    # --- bonds -------------------------------------------------------------------
    nbond = 200
    ids = np.stack([rng.integers(0, n, nbond), rng.integers(0, n, nbond)], 1).astype(np.int32)
    ids[ids[:, 0] == ids[:, 1], 1] = (ids[ids[:, 0] == ids[:, 1], 1] + 1) % n
    Bk = np.abs(rng.normal(1.0, 0.3, size=(nbond, 4))) * np.array([1e4, 1e-2, 1e-2, 1e-2])
    geo = np.stack([np.full(nbond, 1e-3), np.full(nbond, 2e-4), rng.uniform(0, 2e5, nbond), rng.uniform(0, 2e5, nbond),
                    rng.uniform(0, 0.5, nbond)], 1)
    geo[::3, 2:4] = 0.0  # zero tensile strength and cohesion: no failure check, these bonds survive
    frames = rng.normal(0, 1, size=(nbond, 8, 3))
    for a in (0, 1, 2, 4, 5, 6):
        frames[:, a] /= np.linalg.norm(frames[:, a], axis=1, keepdims=True)
    frames[:, 3] *= 2e-3
    frames[:, 7] *= 2e-3
    bonded = (rng.random(nbond) > 0.1).astype(np.int32)
    state = rng.normal(0, 1, size=(nbond, 9))
    F = rng.normal(0, 1e-3, size=(n, 3))
    T = rng.normal(0, 1e-6, size=(n, 3))
    b_in = dict(ids=ids, Bk=Bk, geo=geo, frames=frames.reshape(nbond, 24), bonded=bonded.copy(), state=state.copy(),
                force=F.copy(), torque=T.copy())
    bonded_o, state_o, F_o, T_o = bonded.copy(), np.ascontiguousarray(state.copy()), F.copy(), T.copy()
    fr = np.ascontiguousarray(frames.reshape(nbond, 24))
    assert L.fref_bond(nbond, ip(ids), d(Bk), d(geo), fr.ctypes.data_as(DP), bonded_o.ctypes.data_as(IP),
                       state_o.ctypes.data_as(DP), n, d(pos2), d(q2), F_o.ctypes.data_as(DP),
                       T_o.ctypes.data_as(DP)) == 0
    np.savez_compressed(out / "bonds.npz", pos=pos2, quat=q2, **{f"in_{k}": v for k, v in b_in.items()},
                        bonded_out=bonded_o, state_out=state_o, force_out=F_o, torque_out=T_o)

    # --- integration ----------------------------------------------------------------
    invI = np.abs(rng.normal(1.0, 0.2, size=(n, 6))) * np.array([1e9, 1e9, 1e9, 1e7, 1e7, 1e7])
    v, w = np.ascontiguousarray(vel.copy()), np.ascontiguousarray(angvel.copy())
    F = rng.normal(0, 1e-2, size=(n, 3))
    T = rng.normal(0, 1e-6, size=(n, 3))
    g = np.array([0.0, 0.0, -9.81])
    assert L.fref_kick(n, v.ctypes.data_as(DP), w.ctypes.data_as(DP), d(F), d(T), d(invm), d(q2), d(invI), d(g),
                       C.c_double(5e-7)) == 0
    p3, q3 = np.ascontiguousarray(pos2.copy()), np.ascontiguousarray(q2.copy())
    assert L.fref_drift(n, p3.ctypes.data_as(DP), q3.ctypes.data_as(DP), d(v), d(w), C.c_double(1e-6)) == 0
    np.savez_compressed(out / "integration.npz", vel=vel, angvel=angvel, force=F, torque=T, invm=invm, quat=q2,
                        invI=invI, g=g, h=5e-7, dt=1e-6, pos=pos2, vel_out=v, angvel_out=w, pos_out=p3, quat_out=q3)

    # --- periodic wrap and images ------------------------------------------------
    mn, mx, inv, size = grid_params([0.0, 0.0, 0.0], [0.1, 0.08, 0.05], 0.01)
    P = rng.uniform(-0.005, 0.105, size=(400, 3))
    P[:, 1] = rng.uniform(-0.005, 0.085, 400)
    P[:, 2] = rng.uniform(0.0, 0.05, 400)
    wx = np.ascontiguousarray(P.copy())
    assert L.fref_wrap(400, wx.ctypes.data_as(DP), d(mn), d(mx), 0) == 0
    gx = np.zeros((400, 3))
    assert L.fref_ghost_pos(400, d(wx), d(mn), d(mx), d(inv), ip(size), 1, gx.ctypes.data_as(DP)) == 0
    wy = np.ascontiguousarray(wx.copy())
    assert L.fref_wrap(400, wy.ctypes.data_as(DP), d(mn), d(mx), 1) == 0
    gy = np.zeros((400, 3))
    gxy = np.zeros((400, 3))
    assert L.fref_ghost_pos(400, d(wy), d(mn), d(mx), d(inv), ip(size), 2, gy.ctypes.data_as(DP)) == 0
    assert L.fref_ghost_pos(400, d(wy), d(mn), d(mx), d(inv), ip(size), 3, gxy.ctypes.data_as(DP)) == 0
    np.savez_compressed(out / "periodic.npz", pos=P, min=mn, max=mx, inv=inv, size=size, wrap_x=wx, wrap_xy=wy,
                        ghost_x=gx, ghost_y=gy, ghost_xy=gxy)
    print("golden vectors written to", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py OUTPUT_DIR  (the fixtures are then copied into tests/golden/)")
    main(sys.argv[1])
