"""Physics selection on the GPU (through the C ABI): the Kieft-Bosch
inelastic model and the option bools of every model, against the oracle and
against golden statistics made by the reference's own driver templates
(tests/golden/make_golden_physics.py).

* Kieft-Bosch table lookups: bit-exact;
* single events with identical uniforms and random option bools: equal up to
  the transcendental functions' last-ulp differences (relative tolerance 1e-4,
  at most 0.5 % of cases may differ, where an ulp flips a branch);
* transport for three non-default selections: SE/BSE yields within 3 sigma
  of the reference's at 10^6 primaries, KS p > 0.01 on the detected energy,
  polar angle and position distributions;
* batched runs honour the selection (per-job yields equal plain runs').
"""
import numpy as np
import pytest

import nebula_b200 as nb
from conftest import load_golden
from oracle import oracle as O
from test_gpu_parity import _event_cases, _transport_parity
from test_physics_options import PRESETS

pytestmark = pytest.mark.gpu


def _oracle_geometry(g):
    od_, tr = g.export()
    inf = g.info()
    t11 = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                          tr["r0"], tr["e1"], tr["e2"]], 1)
    return O.Geometry(od_, t11, inf["center"], inf["halfsize"], inf["max_extent"]), len(tr)


@pytest.mark.parametrize("which,rank", [("ki_imfp", 1), ("ki_w0", 2), ("ki_binding", 2)])
def test_kieft_table_lookup_bit_exact(inputs, which, rank):
    m = nb.Material.load(inputs["si_kieft.nmat"])
    om = O.Material(inputs["si_kieft.nmat"])
    rng = np.random.default_rng(4)
    n = 4000
    x = rng.uniform(-1.0, 10.5, n).astype(np.float32)
    y = rng.uniform(-0.1, 1.1, n).astype(np.float32)
    z = np.zeros(n, np.float32)
    t = getattr(om.view, which)
    for rd in ([False, True] if rank > 1 else [False]):
        got = m.table_lookup(which, x, y, z, rounddown=rd)
        fn = O.lib().orc_table_rounddown if rd else O.lib().orc_table_get
        exp = np.array([fn(t, rank, float(a), float(b), 0.0) for a, b in zip(x, y)], np.float32)
        both_nan = np.isnan(got) & np.isnan(exp)
        assert np.array_equal(np.where(both_nan, 0, got.view(np.uint32)),
                              np.where(both_nan, 0, exp.view(np.uint32))), (which, rd)


@pytest.mark.parametrize("model", ["penn", "kieft"])
@pytest.mark.parametrize("kind", [1, 2, 3])
def test_single_events_any_options_match_oracle(inputs, model, kind):
    suffix = "_kieft.nmat" if model == "kieft" else ".nmat"
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    ms = [nb.Material.load(inputs["si" + suffix]), nb.Material.load(inputs["pmma" + suffix])]
    oms = [O.Material(inputs["si" + suffix]), O.Material(inputs["pmma" + suffix])]
    og, n_tri = _oracle_geometry(g)
    rng = np.random.default_rng(200 + kind + (10 if model == "kieft" else 0))
    bad = total = 0
    for rep in range(8):
        opts = {k: int(rng.integers(0, 2)) for k in O.PHYSICS_BITS}
        opts["inelastic_model"] = 1 if model == "kieft" else 0
        bits = O.physics_bits(opts)
        n, nu = 400, 256
        st, mats, tris = _event_cases(kind, n, rng, n_tri)
        U = np.clip(rng.random((n, nu)), 1e-7, 1 - 1e-7).astype(np.float32)
        so, mo, status, se, hs, used = nb.debug_events(kind, ms, st, mats, U, geometry=g, tris=tris, physics=opts)
        for i in range(n):
            h = O.lib().orc_rng_list(U[i].ctypes.data_as(O.f32p), nu)
            s2, m2, stat2, se2 = O.event(og, oms, kind, st[i], int(mats[i]), h,
                                         -1 if tris is None else int(tris[i]), phys=bits)
            used2 = O.lib().orc_rng_used(h)
            O.lib().orc_rng_free(h)
            ok = (m2 == mo[i] and stat2 == status[i] and (se2 is not None) == bool(hs[i]) and used2 == used[i]
                  and np.allclose(so[i], s2, rtol=1e-4, atol=1e-4))
            if ok and se2 is not None:
                ok = np.allclose(se[i], se2, rtol=1e-4, atol=1e-4)
            bad += not ok
            total += 1
    assert bad <= 0.005 * total, "%d of %d events differ" % (bad, total)


@pytest.mark.parametrize("preset", ["kieft", "classical_boundary", "kieft_plain"])
def test_transport_yields_and_distributions_per_selection(inputs, preset):
    """Grating, 100 x 100 pixel subset x 100 primaries at 500 eV, against the
    reference driver instantiated with the same selection."""
    ph = PRESETS[preset]
    gold = load_golden("stats_physics_%s.npz" % preset)
    suffix = "_kieft.nmat" if ph.get("inelastic_model") == 1 else ".nmat"
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    ms = [nb.Material.load(inputs["si" + suffix]), nb.Material.load(inputs["pmma" + suffix])]
    from nebula_b200.synth import workloads
    w = workloads.grating(pixels=gold["pixels"])
    sim = nb.Simulation(g, ms, capacity=1 << 20, seed=77, record_capacity=1 << 22, physics=ph)
    rec, c = _transport_parity(sim, w.primaries, gold, w.primaries["px"].astype(np.int64) * 100000
                               + w.primaries["py"])
    # events per primary agree with the reference driver's (3 %)
    ev_ref = float(gold["events"]) / float(gold["n_primaries"])
    assert abs(c["flights"] / len(w.primaries) - ev_ref) / ev_ref < 0.03
    sim.close()


def test_batch_honours_physics_selection(inputs):
    from nebula_b200.synth import workloads
    ph = PRESETS["kieft"]
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    ms = [nb.Material.load(inputs["si_kieft.nmat"]), nb.Material.load(inputs["pmma_kieft.nmat"])]
    jobs = []
    for j, (px, n) in enumerate([((100, 120), 3000), ((140, 30), 500), ((60, 60), 1500)]):
        w = workloads.grating(pixels=[px], per_pixel=n)
        jobs.append((0, 500 + j, w.primaries))
    b = nb.Batch([g], ms, capacity=1 << 16, physics=ph)
    b.set_jobs(jobs)
    b.run()
    se_b, bse_b = b.job_yields()
    b.close()
    for j, (gi, seed, pri) in enumerate(jobs):
        s = nb.Simulation(g, ms, capacity=1 << 16, seed=seed, physics=ph)
        s.push(pri)
        s.run()
        rec = s.flush_detected()
        assert int((rec["E"] < 50).sum()) == int(se_b[j])
        assert int((rec["E"] >= 50).sum()) == int(bse_b[j])
        s.close()
