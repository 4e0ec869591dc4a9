"""Contact parity with the FP64 oracle at the benchmark configurations' own sizes.

The other parity tests use small scenes; the certified FP32 screen's rounding margins
depend on each template's Lipschitz bound, grid and node count, so these tests replay
one step of the full benchmark scenes through the oracle (the reference's per-node
27-cell detection, LSParticleContactDetectionKernel.cu:4-297, and its force kernels,
contactKernel.cu:46-271), in the FP32 screen on BF16 templates and in the learned
form (BF16 network in front of the same screen):

* precision configuration: 100,000 particles of 4 templates (48^3 grids, 2,000 nodes),
  triply periodic, the whole scene: cell keys, sorted order and cell ranges, the
  particle contact list and each of the 7 image sets;
* drum: 500,000 particles of 64 superquadrics (64^3 grids, 1,500 nodes, exponents up to
  8) in the rotating drum, replayed on the slab |y| < 1 cm through the drum's axis
  (particles and drum wall);
* scale: 2,000,000 particles of 16 superquadrics (48^3 grids, 1,500 nodes), periodic in x
  and y with floor and ceiling, replayed on the column 0.3 L <= x, y < 0.42 L over the
  full height (particles, floor, ceiling).

For a slab or column the oracle gets the particles of the region plus every particle
within 2.05 largest bounding radii of it (so every partner of a region particle is
present) on the whole scene's cell grid; the contacts compared are those with a region
particle as owner or partner, and forces and torques are compared on region particles.

Each replay runs three steps, takes the second step's contacts as history and the
third step's state in the external-force hook, and checks: the (node, partner) pairs of
every list equal the oracle's (bit-exact), springs 1e-7 of the largest, forces and
torques 1e-7 of the largest.
"""
import importlib.util

import numpy as np
import pytest

from conftest import ROOT, load_oracle
from helpers import canon

pytestmark = pytest.mark.gpu

RTOL = 1e-7
STEPS = 3


def _bench():
    spec = importlib.util.spec_from_file_location("lsdem_bench_cfg", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def bench():
    return _bench()


def _run(lsdem, bench, sc, workload, learned):
    """Steps the scene STEPS times; returns the hook state of the last step, the
    contacts of the step before it (history) and of the last step, per list."""
    sv = bench.load(lsdem, sc, workload, 0, 2, learned=learned, record=True)
    kinds = {"pp": lsdem.CONTACT_PARTICLE, "pw": lsdem.CONTACT_WALL, "pg": lsdem.CONTACT_GHOST}
    prev = None
    box = {}
    for k in range(STEPS):
        if k == STEPS - 1:
            prev = {n: sv.contacts(v) for n, v in kinds.items()}
            box["pos_before"] = sv.state()["pos"]

            def hook(t):
                box.update(sv.state())
            sv.step(sc["dt"], 1, hook=hook)
        else:
            sv.step(sc["dt"], 1)
    cur = {n: sv.contacts(v, geometry=True) for n, v in kinds.items()}
    model = load_oracle().model_from_solver(sv)
    hh = sv.hash() if workload == "polydisperse" else None
    grid = sv.grid()
    sv.close()
    return box, prev, cur, model, hh, grid


def _owner(node_base, node):
    return np.searchsorted(node_base, node, side="right") - 1


def _history(c, sub_of, nb_full, nb_sub, n_sub_nodes, partner_is_particle=True):
    """The reference's per-node history arrays (prefix, partner, spring) of the GPU
    contacts whose owner (and particle partner) lie in the oracle's model, in the
    model's numbering."""
    node = np.asarray(c["node"], np.int64)
    own = _owner(nb_full, node)
    so = sub_of[own]
    keep = so >= 0
    part = np.asarray(c["partner"], np.int64)
    if partner_is_particle:
        sp = sub_of[part]
        keep &= sp >= 0
        part = sp
    node_s = nb_sub[so[keep]] + (node[keep] - nb_full[own[keep]])
    order = np.argsort(node_s, kind="stable")
    cnt = np.bincount(node_s, minlength=n_sub_nodes)
    return {"prefix": np.cumsum(cnt).astype(np.int32), "partner": part[keep].astype(np.int32)[order],
            "spring": np.asarray(c["spring"])[keep][order]}


def _compare(label, gpu, orc, sel_gpu, sel_orc, gpu_node, orc_node, gpu_partner, orc_partner):
    g = {"node": gpu_node[sel_gpu], "partner": gpu_partner[sel_gpu]}
    o = {"node": orc_node[sel_orc], "partner": orc_partner[sel_orc]}
    og, oo = canon(g), canon(o)
    assert len(og) == len(oo), f"{label}: {len(og)} GPU contacts vs {len(oo)} oracle"
    assert np.array_equal(g["node"][og], o["node"][oo]), f"{label}: node ids differ"
    assert np.array_equal(g["partner"][og], o["partner"][oo]), f"{label}: partners differ"
    return len(og)


def _replay(lsdem, bench, sc, workload, learned, region=None):
    ora = load_oracle()
    box, prev, cur, model, hh, grid = _run(lsdem, bench, sc, workload, learned)
    P = model["particles"]
    n = len(P["pos"])
    for k in ("pos", "vel", "angvel", "quat"):
        P[k] = box[k].copy()
    if sc["periodic"]:
        # The hook sees positions after the step's periodic wrap; detection ran before it
        # (the reference's order, which the oracle follows). A body that crossed a face in
        # this step is put back across it: the drift from the state before the step tells
        # which did.
        drifted = box["pos_before"] + sc["dt"] * box["vel"]
        L = np.asarray(sc["max"]) - np.asarray(sc["min"])
        for ax in range(3):
            if (sc["periodic"] >> ax) & 1:
                up, dn = drifted[:, ax] >= sc["max"][ax], drifted[:, ax] < sc["min"][ax]
                P["pos"][up, ax] += L[ax]
                P["pos"][dn, ax] -= L[ax]
    counts = np.array([len(model["shapes"][s]["nodes"]) for s in P["shape"]], np.int64)
    nb_full = np.concatenate([[0], np.cumsum(counts)])
    rmax = float(P["radius"].max())
    if region is None:
        sub = np.arange(n)
        inner = np.ones(n, bool)
    else:
        lo, hi = region
        halo = 2.05 * rmax
        x = box["pos"]
        sub = np.nonzero(((x >= lo - halo) & (x < hi + halo)).all(axis=1))[0]
        inner = ((x[sub] >= lo) & (x[sub] < hi)).all(axis=1)
        model["particles"] = {k: np.asarray(v)[sub] for k, v in P.items()}
    sub_of = np.full(n, -1, np.int64)
    sub_of[sub] = np.arange(len(sub))
    model.update(domain=(sc["min"], sc["max"]), gravity=sc["gravity"], grid_cell=2.0 * rmax,
                 periodic=sc["periodic"] if region is None else 0)
    sim = ora.OracleSim(model, nthreads=ora.num_threads())
    nb_sub = sim.node_base
    n_sub_nodes = sim.nodes.total
    sim.old["pp"] = _history(prev["pp"], sub_of, nb_full, nb_sub, n_sub_nodes)
    if sim.W is not None:
        sim.old["pw"] = _history(prev["pw"], sub_of, nb_full, nb_sub, n_sub_nodes, partner_is_particle=False)
    if region is None and sc["periodic"]:
        for m in range(1, 8):
            if (m & sc["periodic"]) == m:
                sel = prev["pg"]["image"] == m
                sim.old[f"g{m}"] = _history({k: v[sel] for k, v in prev["pg"].items()}, sub_of, nb_full, nb_sub,
                                            n_sub_nodes)
    sim.detect_all()
    assert np.array_equal(sim.pg["inv"], grid["inv"]) and np.array_equal(sim.pg["size"], grid["size"])
    if hh is not None:
        for k in ("key", "sorted_idx", "sorted_key", "start", "end"):
            assert np.array_equal(hh[k], sim.last_hash[k]), f"hash: {k} differs"
    inner_full = np.zeros(n, bool)
    inner_full[sub[inner]] = True

    def orc_ids(c, particle_partner=True):
        own = np.asarray(c["owner"], np.int64)
        node = nb_full[sub[own]] + (np.asarray(c["node"], np.int64) - nb_sub[own])
        part = sub[np.asarray(c["partner"], np.int64)] if particle_partner else np.asarray(c["partner"], np.int64)
        return own, node, part

    total = 0
    lists = [("pp", "pp", None, True)]
    if sim.W is not None:
        lists.append(("pw", "pw", None, False))
    if region is None and sc["periodic"]:
        lists += [(f"g{m}", "pg", m, True) for m in range(1, 8) if (m & sc["periodic"]) == m]
    for name, gk, image, ppart in lists:
        g = cur[gk]
        gsel = np.ones(len(g["node"]), bool) if image is None else g["image"] == image
        gnode = np.asarray(g["node"], np.int64)
        gown = _owner(nb_full, gnode)
        gpart = np.asarray(g["partner"], np.int64)
        c = sim.last[name]
        oown, onode, opart = orc_ids(c, ppart)
        g_in = inner_full[gown] | (inner_full[gpart] if ppart else False)
        o_in = inner_full[sub[oown]] | (inner_full[opart] if ppart else False)
        total += _compare(f"{workload} {name}", g, c, gsel & g_in, o_in, gnode, onode, gpart, opart)
    assert total > 100, f"{workload}: only {total} contacts compared"
    sim.forces(sc["dt"])
    # springs after the force update, particle list
    c = sim.last["pp"]
    oown, onode, opart = orc_ids(c)
    o_in = inner_full[sub[oown]] | inner_full[opart]
    g = cur["pp"]
    gnode = np.asarray(g["node"], np.int64)
    gpart = np.asarray(g["partner"], np.int64)
    g_in = inner_full[_owner(nb_full, gnode)] | inner_full[gpart]
    og = canon({"node": gnode[g_in], "partner": gpart[g_in]})
    oo = canon({"node": onode[o_in], "partner": opart[o_in]})
    s_ref = np.asarray(c["spring"])[o_in][oo]
    s_gpu = np.asarray(g["spring"])[g_in][og]
    assert np.abs(s_gpu - s_ref).max() <= RTOL * max(np.abs(s_ref).max(), 1e-300)
    fi = inner
    for k, ref in (("force", sim.F), ("torque", sim.T)):
        a, b = box[k][sub[fi]], ref[fi]
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= RTOL * scale, f"{workload} {k}: {np.abs(a - b).max() / scale:.2e}"
    return total


@pytest.fixture(scope="module")
def polydisperse(lsdem, bench):
    sc, _ = bench.build_scene(lsdem, "polydisperse", 0)
    return sc


@pytest.fixture(scope="module")
def drum(lsdem, bench):
    sc, _ = bench.build_scene(lsdem, "drum", 0)
    return sc


@pytest.fixture(scope="module")
def scale(lsdem, bench):
    sc, _ = bench.build_scene(lsdem, "scale", 0)
    return sc


@pytest.mark.parametrize("learned", [False, True])
def test_precision_config_full_scene(lsdem, bench, polydisperse, learned):
    assert len(polydisperse["pos"]) == 100_000
    _replay(lsdem, bench, polydisperse, "polydisperse", learned)


@pytest.mark.parametrize("learned", [False, True])
def test_drum_config_slab(lsdem, bench, drum, learned):
    assert len(drum["pos"]) == 500_000
    big = 1.0
    _replay(lsdem, bench, drum, "drum", learned, region=(np.array([-big, -0.01, -big]), np.array([big, 0.01, big])))


@pytest.mark.parametrize("learned", [False, True])
def test_scale_config_column(lsdem, bench, scale, learned):
    assert len(scale["pos"]) == 2_000_000
    L = float(scale["max"][0])
    lo = np.array([0.3 * L, 0.3 * L, -1.0])
    hi = np.array([0.42 * L, 0.42 * L, 2.0 * float(scale["max"][2])])
    _replay(lsdem, bench, scale, "scale", learned, region=(lo, hi))
