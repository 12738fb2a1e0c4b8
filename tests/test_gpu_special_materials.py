"""Special material ids of the boundary step (material_manager.h:77-86,
boundary_intersect.h:73-97): DETECTOR, DETECTOR_LT50 / GE50 (detect below /
at or above 50 eV, otherwise pass), MIRROR, NOP (pass) and TERMINATOR.

* single crossings against the oracle with identical uniforms, for every id;
* transport: an LT50 plane under a plain detector splits the same detected
  population by energy (SE at the first plane, BSE at the second) with the
  yields of a single detector; a NOP plane inside the bulk changes nothing
  but the number of flights; a MIRROR box around the beam returns what it
  reflects.
"""
import numpy as np
import pytest

import nebula_b200 as nb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _geometry(tmp_path, name, extra):
    from nebula_b200.synth import geometry as G
    rows = []
    G.box(rows, (-500, -500, -1000), (500, 500, 0), 0, G.VACUUM)
    rows += extra
    p = str(tmp_path / (name + ".tri"))
    G.write_tri(p, np.asarray(rows, dtype=np.float64))
    return nb.Geometry.from_tri_file(p)


def _plane(mat_in, mat_out, z, h=500.0):
    return [[mat_in, mat_out, -h, -h, z, h, -h, z, h, h, z], [mat_in, mat_out, -h, -h, z, h, h, z, -h, h, z]]


def _run(g, m, pri, seed=3):
    sim = nb.Simulation(g, [m], capacity=1 << 16, seed=seed)
    sim.push(pri)
    sim.run()
    rec = sim.flush_detected()
    c = sim.counters()
    sim.close()
    return rec, c


def _yields(rec, n):
    se = (rec["E"] < 50).sum()
    bse = (rec["E"] >= 50).sum()
    return se / n, bse / n, np.sqrt(se) / n, np.sqrt(bse) / n


def test_special_ids_single_crossings_match_oracle(inputs, tmp_path):
    from nebula_b200.synth import geometry as G
    ids = [G.DETECTOR, G.DETECTOR_LT50, G.DETECTOR_GE50, G.MIRROR, G.NOP, G.TERMINATOR]
    extra = []
    for k, mid in enumerate(ids):
        extra += _plane(G.VACUUM, mid, 5.0 + 3.0 * k)
    g = _geometry(tmp_path, "special", extra)
    m = nb.Material.load(inputs["si.nmat"])
    od_, tr = g.export()
    inf = g.info()
    t11 = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                          tr["r0"], tr["e1"], tr["e2"]], 1)
    og = O.Geometry(od_, t11, inf["center"], inf["halfsize"], inf["max_extent"])
    special = np.flatnonzero(np.isin(tr["material_out"], ids))
    assert len(special) == 2 * len(ids)
    rng = np.random.default_rng(5)
    n = 2000
    tris = rng.choice(special, n).astype(np.int32)
    E = np.exp(rng.uniform(np.log(2), np.log(2000), n))
    d = rng.standard_normal((n, 3))
    st = np.concatenate([rng.uniform(-100, 100, (n, 3)), d, E[:, None]], 1).astype(np.float32)
    mats = np.full(n, G.VACUUM, np.int32)
    U = np.clip(rng.random((n, 8)), 1e-7, 1 - 1e-7).astype(np.float32)
    so, mo, status, se, hs, used = nb.debug_events(3, [m], st, mats, U, geometry=g, tris=tris)
    om = O.Material(inputs["si.nmat"])
    for i in range(n):
        h = O.lib().orc_rng_list(U[i].ctypes.data_as(O.f32p), 8)
        s2, m2, stat2, _ = O.event(og, [om], 3, st[i], int(mats[i]), h, int(tris[i]))
        O.lib().orc_rng_free(h)
        assert m2 == mo[i] and stat2 == status[i], (i, int(tr["material_out"][tris[i]]))
        assert np.allclose(so[i], s2, rtol=1e-5, atol=1e-5)
    # every id was exercised with each outcome it can have (electrons moving
    # along the planes' normal, +z, meet the special side; the others cross
    # from the special side into vacuum, an ordinary vacuum-vacuum crossing)
    outs = {int(tr["material_out"][t]): set() for t in special}
    for t, s, up in zip(tris, status, st[:, 5] > 0):
        if up:
            outs[int(tr["material_out"][t])].add(int(s))
    assert outs[G.DETECTOR] == {1} and outs[G.TERMINATOR] == {2}
    assert outs[G.DETECTOR_LT50] == {0, 1} and outs[G.DETECTOR_GE50] == {0, 1}
    assert outs[G.MIRROR] == {0} and outs[G.NOP] == {0}


def test_lt50_plane_splits_the_detected_population(inputs, tmp_path):
    from nebula_b200.synth import geometry as G, primaries
    m = nb.Material.load(inputs["si.nmat"])
    n = 40000
    pri = primaries.point_beam(n)
    g1 = _geometry(tmp_path, "one", _plane(G.VACUUM, G.DETECTOR, 10.0))
    g2 = _geometry(tmp_path, "two", _plane(G.VACUUM, G.DETECTOR_LT50, 5.0) + _plane(G.VACUUM, G.DETECTOR, 15.0))
    r1, _ = _run(g1, m, pri, seed=3)
    r2, _ = _run(g2, m, pri, seed=4)
    se2 = r2["E"] < 50
    assert np.all(np.abs(r2["pos"][se2, 2] - 5.0) < 1e-3)
    assert np.all(np.abs(r2["pos"][~se2, 2] - 15.0) < 1e-3)
    y1, y2 = _yields(r1, n), _yields(r2, n)
    assert abs(y1[0] - y2[0]) < 3 * np.hypot(y1[2], y2[2]) * 1.5
    assert abs(y1[1] - y2[1]) < 3 * np.hypot(y1[3], y2[3]) * 1.5


def test_nop_plane_in_the_bulk_changes_only_the_flight_count(inputs, tmp_path):
    from nebula_b200.synth import geometry as G, primaries
    m = nb.Material.load(inputs["si.nmat"])
    n = 40000
    pri = primaries.point_beam(n)
    g1 = _geometry(tmp_path, "plain", _plane(G.VACUUM, G.DETECTOR, 10.0))
    g2 = _geometry(tmp_path, "nop", _plane(G.VACUUM, G.DETECTOR, 10.0) + _plane(0, G.NOP, -3.0))
    r1, c1 = _run(g1, m, pri, seed=3)
    r2, c2 = _run(g2, m, pri, seed=4)
    y1, y2 = _yields(r1, n), _yields(r2, n)
    assert abs(y1[0] - y2[0]) < 3 * np.hypot(y1[2], y2[2]) * 1.5
    assert abs(y1[1] - y2[1]) < 3 * np.hypot(y1[3], y2[3]) * 1.5
    assert c2["boundary"] > c1["boundary"]
