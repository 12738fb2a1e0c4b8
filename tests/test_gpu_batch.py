"""Batched persistent runs: per-job results equal those of each job run alone
in the plain wavefront with the same seed (the random streams are keyed by
job seed, primary index and ancestry only), for several launch shapes and
refill thresholds."""
import os

import numpy as np
import pytest

import nebula_b200 as nb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_batch(tmp_path_factory):
    from nebula_b200.synth import workloads, geometry, materials, nmat
    d = tmp_path_factory.mktemp("batch")
    geoms_tri, specs, jobs, desc = workloads.batch(seed=7, n_jobs=8, scale=0.004, e_max=30e3)
    # keep the test bounded: at most 3 keV
    jobs = [(gi, seed, pri[:400]) for gi, seed, pri in jobs]
    for _, _, pri in jobs:
        pri["E"] = np.minimum(pri["E"], 3000.0)
    geoms = []
    for i, t in enumerate(geoms_tri):
        p = os.path.join(str(d), "g%d.tri" % i)
        geometry.write_tri(p, t)
        geoms.append(nb.Geometry.from_tri_file(p))
    mats = []
    for sp in specs:
        p = os.path.join(str(d), sp.name + ".nmat")
        nmat.write(p, materials.build_raw_material(sp))
        mats.append(nb.Material.load(p))
    return geoms, mats, jobs


def _plain_yields(geoms, mats, jobs, physics=None):
    out = []
    for gi, seed, pri in jobs:
        g = geoms[gi]
        n_mat = 1 if gi == 0 else 2
        sim = nb.Simulation(g, mats[:n_mat], capacity=1 << 14, seed=seed, physics=physics)
        sim.push(pri)
        sim.run()
        rec = sim.flush_detected()
        out.append((int((rec["E"] < 50).sum()), int((rec["E"] >= 50).sum())))
        sim.close()
    return np.array(out)


@pytest.mark.parametrize("block,thr,cap,graph", [(256, 1.0, 1 << 16, True), (512, 0.3, 1 << 14, True),
                                                 (128, 0.5, 1 << 12, False)])
def test_batch_per_job_yields_equal_plain_runs(small_batch, block, thr, cap, graph):
    geoms, mats, jobs = small_batch
    ref = _plain_yields(geoms, mats, jobs)
    b = nb.Batch(geoms, mats, capacity=cap, refill_threshold=thr, block_size=block, use_graph=graph)
    b.set_jobs(jobs)
    for _ in range(2):      # a second run on the same batch object starts clean
        b.run()
        se, bse = b.job_yields()
        assert np.array_equal(se, ref[:, 0]), (se, ref[:, 0])
        assert np.array_equal(bse, ref[:, 1])
        c = b.counters()
        assert c["primaries_started"] == sum(len(p) for _, _, p in jobs)
        assert c["primaries_started"] + c["spawned"] == c["detected"] + c["terminated"]
        assert c["queue_overflow"] == 0
    b.close()


def test_batch_with_a_non_default_physics_selection(small_batch):
    """The batched kernel compiled for run-time physics bits: per-job yields
    equal plain runs with the same selection, and differ from the default
    selection's."""
    geoms, mats, jobs = small_batch
    physics = {"interface_refraction": 0, "quantum_transmission": 0, "interface_absorption": 1,
               "atomic_recoil_loss": 0}
    ref = _plain_yields(geoms, mats, jobs, physics)
    b = nb.Batch(geoms, mats, capacity=1 << 14, block_size=256, physics=physics)
    b.set_jobs(jobs)
    b.run()
    se, bse = b.job_yields()
    b.close()
    assert np.array_equal(se, ref[:, 0]) and np.array_equal(bse, ref[:, 1])
    assert not np.array_equal(ref, _plain_yields(geoms, mats, jobs))


def test_batch_rejects_bad_job_ranges(small_batch):
    geoms, mats, jobs = small_batch
    b = nb.Batch(geoms, mats, capacity=1 << 12)
    bad = [(len(geoms), 1, jobs[0][2])]
    with pytest.raises(nb.NblError):
        b.set_jobs(bad)
    b.close()


def _plain_records(geoms, mats, jobs):
    out = []
    for gi, seed, pri in jobs:
        sim = nb.Simulation(geoms[gi], mats[: (1 if gi == 0 else 2)], capacity=1 << 14, seed=seed)
        sim.push(pri)
        sim.run()
        out.append(sim.flush_detected())
        sim.close()
    return out


def _sorted(rec):
    return np.sort(rec.view(np.dtype((np.void, 36))).ravel()).tobytes()


def test_batch_records_equal_plain_runs(small_batch):
    """Every job's detected 36-byte records from the batched launch equal, as
    a set, the records of the job run alone in the plain wavefront."""
    geoms, mats, jobs = small_batch
    ref = _plain_records(geoms, mats, jobs)
    b = nb.Batch(geoms, mats, capacity=1 << 14, block_size=256, record_capacity=1 << 20)
    b.set_jobs(jobs)
    for _ in range(2):
        b.run()
        per_job = b.job_records()
        assert len(per_job) == len(jobs)
        for k, (got, want) in enumerate(zip(per_job, ref)):
            assert len(got) == len(want) > 0, k
            assert _sorted(got) == _sorted(want), k
        se, bse = b.job_yields()
        assert np.array_equal(se, [int((r["E"] < 50).sum()) for r in ref])
        assert b.counters()["records_pending"] == sum(len(r) for r in ref)
    b.close()


def test_batch_record_overflow_is_an_error(small_batch):
    geoms, mats, jobs = small_batch
    b = nb.Batch(geoms, mats, capacity=1 << 14, block_size=256, record_capacity=16)
    b.set_jobs(jobs)
    with pytest.raises(nb.NblError) as e:
        b.run()
    assert e.value.status == 6 and "record_capacity" in str(e.value)
    b.close()


def test_the_largest_material_table_gives_the_same_records(small_batch):
    """127 materials (the most a simulation takes; the jobs use the first two):
    the batched kernel stages every material's descriptor in shared memory
    (40.6 KB per block, above its default 48 KB limit together with its
    geometry and job tables), and the records equal those with two
    materials, batched and plain."""
    geoms, mats, jobs = small_batch
    many = list(mats) + [mats[1]] * (127 - len(mats))
    ref = _plain_records(geoms, mats, jobs)
    b = nb.Batch(geoms, many, capacity=1 << 14, block_size=512, record_capacity=1 << 20)
    b.set_jobs(jobs)
    b.run()
    for k, (got, want) in enumerate(zip(b.job_records(), ref)):
        assert _sorted(got) == _sorted(want), k
    b.close()
    gi, seed, pri = jobs[-1]
    sim = nb.Simulation(geoms[gi], many, capacity=1 << 14, seed=seed)
    sim.push(pri)
    sim.run()
    assert _sorted(sim.flush_detected()) == _sorted(ref[-1])
    sim.close()
