"""Transport parity across the beam energies of the mixed batch (200 eV to
20 keV), beyond the 0.3-1 keV workloads of the other parity tests.

Si slab with tables to 30 keV, point beam at normal incidence; the oracle
(the restatement pinned bit for bit to the reference CPU driver) against the
CUDA path through the C ABI, different random numbers:

* SE and BSE yields within 3 sigma (sigma from the spread over 500 primary
  groups in both runs);
* detected energy distributions: two-sample KS on all records of both runs,
  p > 0.01 (the criterion of the other parity tests); every record is used,
  which keeps the test's power (a 200 eV check against 2 x 10^6 GPU and
  4 x 10^5 oracle primaries gave a binned KS distance of 0.0017, p ~ 0.6,
  and the reference's own GPU driver agreed with both);
* events per primary within 3 %.
"""
import os

import numpy as np
import pytest
from scipy import stats

import nebula_b200 as nb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N_GROUPS = 500


def _inputs(tmp_path, energy, n):
    from nebula_b200.synth import workloads, geometry, materials, nmat
    w = workloads.slab(n_primaries=n, energy=energy, e_max=30e3)
    tri = str(tmp_path / "slab.tri")
    geometry.write_tri(tri, w.triangles)
    paths = []
    for spec in w.material_specs:
        p = str(tmp_path / (spec.name + ".nmat"))
        nmat.write(p, materials.build_raw_material(spec))
        paths.append(p)
    pri = w.primaries.copy()
    pri["px"] = np.arange(n) % N_GROUPS
    pri["py"] = 0
    return tri, paths, pri


def _group_totals(rec):
    se = np.bincount(rec["px"], weights=rec["E"] < 50.0, minlength=N_GROUPS)
    bse = np.bincount(rec["px"], weights=rec["E"] >= 50.0, minlength=N_GROUPS)
    return se, bse


@pytest.mark.parametrize("energy,n_gpu,n_oracle", [(200.0, 800_000, 200_000),
                                                   (5000.0, 400_000, 80_000),
                                                   (15000.0, 200_000, 40_000)])
def test_yields_and_spectra_across_energies(tmp_path, energy, n_gpu, n_oracle):
    tri, mats, pri = _inputs(tmp_path, energy, n_gpu)
    g = nb.Geometry.from_tri_file(tri)
    sim = nb.Simulation(g, [nb.Material.load(p) for p in mats], capacity=1 << 20, seed=77, record_capacity=1 << 22)
    sim.push(pri)
    sim.run()
    ours = sim.flush_detected()
    flights = sim.counters()["flights"]
    sim.close()

    od, tr = g.export()
    inf = g.info()
    t11 = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                          tr["r0"], tr["e1"], tr["e2"]], 1)
    og = O.Geometry(od, t11, inf["center"], inf["halfsize"], inf["max_extent"])
    ref, _, events = O.simulate(og, [O.Material(p) for p in mats], pri[:n_oracle], 5,
                                threads=os.cpu_count() or 1)

    for name, a, b in zip(("SE", "BSE"), _group_totals(ours), _group_totals(ref)):
        ya, yb = a.sum() / n_gpu, b.sum() / n_oracle
        # standard errors of the yields from the spread over equal groups
        sa = np.sqrt(N_GROUPS * a.var(ddof=1)) / n_gpu
        sb = np.sqrt(N_GROUPS * b.var(ddof=1)) / n_oracle
        assert abs(ya - yb) < 3 * np.hypot(sa, sb), "%s yield at %g eV: %.5f vs oracle %.5f (sigma %.5f)" % (
            name, energy, ya, yb, np.hypot(sa, sb))
    p = stats.ks_2samp(ours["E"], ref["E"]).pvalue
    assert p > 0.01, "energy spectra at %g eV: KS p = %.3g" % (energy, p)
    epp, epp_ref = flights / n_gpu, events / n_oracle
    assert abs(epp - epp_ref) < 0.03 * epp_ref, "events per primary %.1f vs oracle %.1f" % (epp, epp_ref)
