"""Parity of the CUDA path (through the C ABI) with the oracle and with
golden fixtures made by the reference.

* octree walks: bit-exact (distance bits and triangle id) on every ray;
* table lookups: bit-exact;
* single events with identical uniforms: equal up to the transcendental
  functions' last-ulp differences (relative tolerance 1e-4 on every output,
  allowed to fail on at most 0.5 % of cases, where an ulp flips a branch);
* transport: SE/BSE yields within 3 sigma of the reference's at 10^6
  primaries, detected energy / polar angle / position distributions pass a
  two-sample KS test at p > 0.01 against the reference's.
"""
import numpy as np
import pytest

import nebula_b200 as nb
from conftest import load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _golden_geometry(name):
    o = load_golden("octree_%s.npz" % name)
    t = o["tri11"]
    tr = np.zeros(len(t), nb.TRI_DTYPE)
    tr["material_in"] = t[:, 0].astype(np.int32)
    tr["material_out"] = t[:, 1].astype(np.int32)
    tr["r0"], tr["e1"], tr["e2"] = t[:, 2:5], t[:, 5:8], t[:, 8:11]
    return nb.Geometry.from_linearized(o["octree_data"], tr, o["center"], o["halfsize"]), o


@pytest.mark.parametrize("name", ["slab", "grating"])
def test_ray_query_bit_exact_vs_reference_fixture(name):
    g, _ = _golden_geometry(name)
    r = load_golden("rays_%s.npz" % name)
    od, ot = g.ray_query(r["pos"], r["dir"], r["dist"], r["ignore_tri"], r["ignore_mat"])
    assert np.array_equal(ot, r["out_tri"])
    assert np.array_equal(od.view(np.uint32), r["out_dist"].view(np.uint32))


def test_ray_query_bit_exact_vs_oracle_many_rays(inputs):
    """200 k random walks on the grating built by this library's own builder."""
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    od_, tr = g.export()
    inf = g.info()
    t11 = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                          tr["r0"], tr["e1"], tr["e2"]], 1)
    og = O.Geometry(od_, t11, inf["center"], inf["halfsize"], inf["max_extent"])
    rng = np.random.default_rng(11)
    n = 200_000
    pos = np.stack([rng.uniform(-140, 140, n), rng.uniform(-490, 490, n), rng.uniform(-40, 49, n)], 1)
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    dist = rng.exponential(40.0, n).astype(np.float32)
    im = rng.choice(np.array([-123, 0, 1], np.int32), n)
    od, ot = g.ray_query(pos, d, dist, None, im)
    sub = rng.choice(n, 5000, replace=False)
    o_d, o_t = og.propagate(pos[sub].astype(np.float32), d[sub].astype(np.float32), dist[sub], None, im[sub])
    assert np.array_equal(ot[sub], o_t)
    assert np.array_equal(od[sub].view(np.uint32), o_d.view(np.uint32))


def test_ray_query_bit_exact_on_edges_vertices_and_ties(inputs):
    """Rays aimed at triangle edges and vertices (where u, v or u + v sits on
    its threshold), rays from cell-aligned points along diagonals (where two
    or three leaf exits tie) and rays with a zero or tiny direction
    component: the cases where a comparison cannot be decided from a fast
    quotient and the IEEE quotient must decide it.  Distance bits and
    triangle ids equal the oracle's on every ray."""
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    od_, tr = g.export()
    inf = g.info()
    t11 = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                          tr["r0"], tr["e1"], tr["e2"]], 1)
    og = O.Geometry(od_, t11, inf["center"], inf["halfsize"], inf["max_extent"])
    rng = np.random.default_rng(29)
    n = 6000
    ti = rng.integers(0, len(tr), n)
    r0, e1, e2 = (tr[k][ti].astype(np.float64) for k in ("r0", "e1", "e2"))
    a = rng.uniform(0, 1, (n, 1))
    kind = rng.integers(0, 4, n)[:, None]
    target = np.where(kind == 0, r0 + a * e1,                       # v = 0 edge
             np.where(kind == 1, r0 + a * e2,                       # u = 0 edge
             np.where(kind == 2, r0 + a * e1 + (1 - a) * e2,        # u + v = 1 edge
                      r0 + e1 * (rng.integers(0, 2, (n, 1))))))     # vertices
    off = rng.standard_normal((n, 3))
    off /= np.linalg.norm(off, axis=1, keepdims=True)
    pos = target + off * rng.uniform(0.5, 60.0, (n, 1))
    d = target - pos
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    # cell-aligned starts along diagonals, and zero / tiny direction components
    m = 3000
    gp = np.stack([rng.integers(-140, 140, m), rng.integers(-490, 490, m), rng.integers(-40, 49, m)], 1)
    gd = rng.choice(np.array([-1.0, 1.0]), (m, 3))
    gd[: m // 3, rng.integers(0, 3)] = 0.0
    gd[m // 3: 2 * m // 3, 2] = 1e-39
    gd /= np.linalg.norm(gd, axis=1, keepdims=True)
    pos = np.concatenate([pos, gp.astype(np.float64)]).astype(np.float32)
    d = np.concatenate([d, gd]).astype(np.float32)
    inside = np.all(np.abs(pos - inf["center"]) < 0.999 * np.asarray(inf["halfsize"]), axis=1)
    pos, d = pos[inside], d[inside]
    dist = rng.exponential(80.0, len(pos)).astype(np.float32)
    im = np.full(len(pos), -123, np.int32)
    od, ot = g.ray_query(pos, d, dist, None, im)
    o_d, o_t = og.propagate(pos, d, dist, None, im)
    assert inside[:n].sum() > n // 2 and (ot >= 0).sum() > n // 4     # the aimed rays do hit
    assert np.array_equal(ot, o_t)
    assert np.array_equal(od.view(np.uint32), o_d.view(np.uint32))


@pytest.mark.parametrize("which,rank", [("el_imfp", 1), ("el_icdf", 2), ("in_imfp", 1), ("in_omega", 2),
                                        ("in_q", 3), ("in_binding", 3)])
def test_table_lookup_bit_exact(inputs, which, rank):
    m = nb.Material.load(inputs["si.nmat"])
    om = O.Material(inputs["si.nmat"])
    rng = np.random.default_rng(3)
    n = 4000
    x = rng.uniform(-1.0, 10.5, n).astype(np.float32)     # log E incl. extrapolation
    y = rng.uniform(-0.1, 1.1, n).astype(np.float32)
    z = rng.uniform(-0.1, 1.1, n).astype(np.float32)
    if which == "in_binding":
        y = rng.uniform(-8, 0.5, n).astype(np.float32)
    t = getattr(om.view, which)
    for rd in ([False, True] if rank > 1 else [False]):
        got = m.table_lookup(which, x, y, z, rounddown=rd)
        fn = O.lib().orc_table_rounddown if rd else O.lib().orc_table_get
        exp = np.array([fn(t, rank, float(a), float(b), float(c)) for a, b, c in zip(x, y, z)], np.float32)
        # bit-exact, with every NaN equal to every NaN (rows below the Fermi
        # energy hold -inf, whose interpolation gives NaN on both sides)
        both_nan = np.isnan(got) & np.isnan(exp)
        assert np.array_equal(np.where(both_nan, 0, got.view(np.uint32)),
                              np.where(both_nan, 0, exp.view(np.uint32))), (which, rd)


def _event_cases(kind, n, rng, n_tri=None):
    E = np.exp(rng.uniform(np.log(13), np.log(9000), n))
    d = rng.standard_normal((n, 3)) * rng.uniform(0.5, 2, (n, 1))
    pos = np.stack([rng.uniform(-60, 60, n), rng.uniform(-60, 60, n), rng.uniform(-50, 30, n)], 1)
    st = np.concatenate([pos, d, E[:, None]], 1).astype(np.float32)
    mats = rng.integers(0, 2, n).astype(np.int32)
    tris = None
    if kind == 3:
        tris = rng.integers(0, n_tri, n).astype(np.int32)
        mats = rng.choice(np.array([0, 1, -123], np.int32), n)
    return st, mats, tris


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_single_events_match_oracle(inputs, kind):
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    ms = [nb.Material.load(inputs["si.nmat"]), nb.Material.load(inputs["pmma.nmat"])]
    oms = [O.Material(inputs["si.nmat"]), O.Material(inputs["pmma.nmat"])]
    od_, tr = g.export()
    inf = g.info()
    t11 = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                          tr["r0"], tr["e1"], tr["e2"]], 1)
    og = O.Geometry(od_, t11, inf["center"], inf["halfsize"], inf["max_extent"])
    rng = np.random.default_rng(100 + kind)
    n = 3000
    nu = 256
    st, mats, tris = _event_cases(kind, n, rng, len(tr))
    U = rng.random((n, nu)).astype(np.float32)
    U = np.clip(U, 1e-7, 1 - 1e-7).astype(np.float32)
    so, mo, status, se, hs, used = nb.debug_events(kind, ms, st, mats, U, geometry=g, tris=tris)
    bad = 0
    for i in range(n):
        h = O.lib().orc_rng_list(U[i].ctypes.data_as(O.f32p), nu)
        s2, m2, stat2, se2 = O.event(og, oms, kind, st[i], int(mats[i]), h, -1 if tris is None else int(tris[i]))
        used2 = O.lib().orc_rng_used(h)
        O.lib().orc_rng_free(h)
        ok = (m2 == mo[i] and stat2 == status[i] and (se2 is not None) == bool(hs[i]) and used2 == used[i]
              and np.allclose(so[i], s2, rtol=1e-4, atol=1e-4))
        if ok and se2 is not None:
            ok = np.allclose(se[i], se2, rtol=1e-4, atol=1e-4)
        bad += not ok
    assert bad <= 0.005 * n, "%d of %d events differ" % (bad, n)


def _ks(a, b):
    from scipy.stats import ks_2samp
    return ks_2samp(a, b).pvalue


def _yield_check(n, se, bse, se_sumsq, bse_sumsq, g):
    """Yields and their standard errors from per-group counts; compare."""
    def mean_var(total, sumsq, n_groups, n_pri):
        # per-group count c_k with n_pri / n_groups primaries each
        per = n_pri / n_groups
        m = total / n_groups
        var_group = max(sumsq / n_groups - m * m, 0.0)
        return total / n_pri, var_group / n_groups / (per * per)
    ys, vs = mean_var(se, se_sumsq, g["n_groups_gpu"], n)
    yb, vb = mean_var(bse, bse_sumsq, g["n_groups_gpu"], n)
    rs, rvs = mean_var(int(g["se"]), float(g["se_group_sumsq"]), int(g["n_groups"]), int(g["n_primaries"]))
    rb, rvb = mean_var(int(g["bse"]), float(g["bse_group_sumsq"]), int(g["n_groups"]), int(g["n_primaries"]))
    zs = (ys - rs) / np.sqrt(vs + rvs)
    zb = (yb - rb) / np.sqrt(vb + rvb)
    return (ys, rs, zs), (yb, rb, zb)


def _group_sumsq(rec, keys):
    k = rec["px"].astype(np.int64) * 100000 + rec["py"]
    se = rec["E"] < 50
    uk, inv = np.unique(keys, return_inverse=True)
    pos = np.searchsorted(uk, k)
    cs = np.bincount(pos[se], minlength=len(uk)).astype(np.float64)
    cb = np.bincount(pos[~se], minlength=len(uk)).astype(np.float64)
    return (cs ** 2).sum(), (cb ** 2).sum(), len(uk)


def _transport_parity(sim, pri, gold, keys):
    sim.push(pri)
    sim.run()
    rec = sim.flush_detected()
    c = sim.counters()
    n = len(pri)
    assert c["primaries_started"] == n
    assert c["queue_overflow"] == 0 and c["record_overflow"] == 0 and c["nan_state"] == 0
    se = int((rec["E"] < 50).sum())
    bse = int((rec["E"] >= 50).sum())
    assert se + bse == c["detected"]
    ss, sb, ng = _group_sumsq(rec, keys)
    g = dict(gold)
    g["n_groups_gpu"] = ng
    (ys, rs, zs), (yb, rb, zb) = _yield_check(n, se, bse, ss, sb, g)
    assert abs(zs) < 3, "SE yield %.5f vs reference %.5f (%.2f sigma)" % (ys, rs, zs)
    assert abs(zb) < 3, "BSE yield %.5f vs reference %.5f (%.2f sigma)" % (yb, rb, zb)
    d = rec["dir"].astype(np.float64)
    cos_t = d[:, 2] / np.linalg.norm(d, axis=1)
    for name, mine, ref in (("energy", rec["E"], gold["sub_E"]), ("cos_theta", cos_t, gold["sub_cos"]),
                            ("x", rec["pos"][:, 0], gold["sub_x"]), ("y", rec["pos"][:, 1], gold["sub_y"])):
        p = _ks(mine, ref)
        assert p > 0.01, "KS %s p=%.4g" % (name, p)
    return rec, c


def test_transport_slab_yields_and_distributions(inputs):
    """Slab, 10^6 primaries at 1 keV, one pixel per primary."""
    gold = load_golden("stats_slab.npz")
    g = nb.Geometry.from_tri_file(inputs["slab.tri"])
    m = nb.Material.load(inputs["si.nmat"])
    from nebula_b200.synth import primaries
    n = int(gold["n_primaries"])
    pri = primaries.point_beam(n)
    idx = np.arange(n)
    pri["px"] = idx % 1000
    pri["py"] = idx // 1000
    sim = nb.Simulation(g, [m], capacity=1 << 20, seed=1234, record_capacity=1 << 22)
    _transport_parity(sim, pri, gold, pri["px"].astype(np.int64) * 100000 + pri["py"])


def test_transport_grating_yields_and_distributions(inputs):
    """Line-space grating, 100 x 100 pixel subset x 100 primaries at 500 eV."""
    gold = load_golden("stats_grating.npz")
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    ms = [nb.Material.load(inputs["si.nmat"]), nb.Material.load(inputs["pmma.nmat"])]
    from nebula_b200.synth import workloads
    w = workloads.grating(pixels=gold["pixels"])
    sim = nb.Simulation(g, ms, capacity=1 << 20, seed=99, record_capacity=1 << 22, tally=(256, 256))
    rec, c = _transport_parity(sim, w.primaries, gold, w.primaries["px"].astype(np.int64) * 100000
                               + w.primaries["py"])
    se_img, bse_img, hist = sim.tallies()
    assert int(se_img.sum()) == int((rec["E"] < 50).sum())
    assert int(bse_img.sum()) == int((rec["E"] >= 50).sum())
    assert int(hist.sum()) == int((rec["E"] < 1000).sum())


def test_transport_events_per_primary_match_oracle(inputs):
    """Mean driver iterations per primary agree with the oracle's (the
    roofline's unit of work), slab, 1 keV."""
    from nebula_b200.synth import primaries
    g = nb.Geometry.from_tri_file(inputs["slab.tri"])
    m = nb.Material.load(inputs["si.nmat"])
    n = 20000
    pri = primaries.point_beam(n)
    sim = nb.Simulation(g, [m], capacity=1 << 18, seed=5)
    sim.push(pri)
    sim.run()
    c = sim.counters()
    od_, tr = g.export()
    inf = g.info()
    t11 = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                          tr["r0"], tr["e1"], tr["e2"]], 1)
    og = O.Geometry(od_, t11, inf["center"], inf["halfsize"], inf["max_extent"])
    _, _, ev = O.simulate(og, [O.Material(inputs["si.nmat"])], pri[:5000], 9, threads=4)
    gpu = c["flights"] / n
    cpu = ev / 5000
    assert abs(gpu - cpu) / cpu < 0.03, (gpu, cpu)


def test_transport_deterministic_and_capacity_independent(inputs):
    """Counter-based RNG: the same seed gives the same records whatever the
    pool capacity or launch shape (trajectories do not depend on slots)."""
    from nebula_b200.synth import primaries
    g = nb.Geometry.from_tri_file(inputs["slab.tri"])
    m = nb.Material.load(inputs["si.nmat"])
    pri = primaries.point_beam(3000)
    outs = []
    spilled = []
    counters = []
    # (pool capacity, threads per block, leaf cells a walk takes per
    # iteration before it continues in the next; 2^20: never cut)
    for cap, blk, cells in ((1 << 16, 256, 1), (1 << 12, 128, 1), (64, 64, 1), (1 << 16, 256, 1 << 20),
                            (64, 64, 1 << 20), (1 << 12, 128, 2), (64, 64, 3)):
        sim = nb.Simulation(g, [m], capacity=cap, seed=42, block_size=blk, walk_cells=cells)
        sim.push(pri)
        sim.run()
        r = sim.flush_detected()
        c = sim.counters()
        spilled.append(c["spilled"])
        counters.append({k: c[k] for k in ("flights", "boundary", "elastic", "inelastic", "spawned", "detected",
                                           "terminated", "primaries_started")})
        # the slab's octree is shallow: walks continue at budgets of 1 and 2 cells
        assert (c["walk_resumes"] == 0) if cells == 1 << 20 else (c["walk_resumes"] > 0 or cells > 2)
        outs.append(np.sort(r.view(np.dtype((np.void, 36))).ravel()).tobytes())
    assert all(o == outs[0] for o in outs[1:])
    assert all(c == counters[0] for c in counters[1:]), counters
    # the smallest pools must have parked secondaries in the overflow ring
    assert spilled[2] > 0 and spilled[4] > 0 and spilled[6] > 0


def test_small_capacity_forces_many_refills(inputs):
    """A pool far smaller than one cascade still finishes every primary."""
    from nebula_b200.synth import primaries
    g = nb.Geometry.from_tri_file(inputs["slab.tri"])
    m = nb.Material.load(inputs["si.nmat"])
    pri = primaries.point_beam(300, energy=1000.0)
    sim = nb.Simulation(g, [m], capacity=64, seed=1, iterations_per_graph=6)
    sim.push(pri)
    sim.run()
    c = sim.counters()
    assert c["primaries_started"] == 300
    assert c["primaries_started"] + c["spawned"] == c["detected"] + c["terminated"]
