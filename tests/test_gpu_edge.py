"""Edge cases of the transport through the C ABI: empty runs, primaries
outside the domain, stepping a run piecewise, pushing primaries in parts,
and the documented error statuses (record buffer overflow, event budget,
NaN state) -- every failure is a status, never a silent result."""
import numpy as np
import pytest

import nebula_b200 as nb

pytestmark = pytest.mark.gpu


def _slab(inputs):
    return nb.Geometry.from_tri_file(inputs["slab.tri"]), nb.Material.load(inputs["si.nmat"])


def _sorted(rec):
    return np.sort(rec.view(np.dtype((np.void, 36))).ravel()).tobytes()


def test_empty_run(inputs):
    g, m = _slab(inputs)
    sim = nb.Simulation(g, [m], capacity=1024, seed=1, tally=(4, 4))
    sim.run()
    assert len(sim.flush_detected()) == 0
    c = sim.counters()
    assert c["flights"] == 0 and c["primaries_started"] == 0
    se, bse, hist = sim.tallies()
    assert se.sum() == 0 and bse.sum() == 0 and hist.sum() == 0
    sim.close()


def test_primaries_outside_the_domain_terminate(inputs):
    from nebula_b200.synth import primaries
    g, m = _slab(inputs)
    pri = primaries.point_beam(500)
    pri["pos"][:, 0] = 1.0e5                     # far outside the octree box
    sim = nb.Simulation(g, [m], capacity=1024, seed=1)
    sim.push(pri)
    sim.run()
    c = sim.counters()
    assert len(sim.flush_detected()) == 0
    assert c["primaries_started"] == 500 and c["terminated"] == 500 and c["flights"] == 500
    sim.close()


def test_stepping_and_split_push_equal_one_run(inputs):
    from nebula_b200.synth import primaries
    g, m = _slab(inputs)
    pri = primaries.point_beam(2000)
    a = nb.Simulation(g, [m], capacity=1 << 12, seed=9)
    a.push(pri)
    a.run()
    ra = a.flush_detected()
    b = nb.Simulation(g, [m], capacity=1 << 12, seed=9)
    b.push(pri[:700])
    b.push(pri[700:])
    steps = 0
    while b.do_iteration(24) > 0:
        steps += 1
        assert steps < 10000
    rb = b.flush_detected()
    assert steps > 1
    assert len(ra) > 0 and _sorted(ra) == _sorted(rb)
    a.close()
    b.close()


def test_record_buffer_overflow_is_an_error(inputs):
    from nebula_b200.synth import primaries
    g, m = _slab(inputs)
    sim = nb.Simulation(g, [m], capacity=1 << 14, seed=1, record_capacity=16)
    sim.push(primaries.point_beam(5000))
    with pytest.raises(nb.NblError) as e:
        sim.run()
    assert e.value.status == 6
    sim.close()


def test_event_budget_is_an_error(inputs):
    from nebula_b200.synth import primaries
    g, m = _slab(inputs)
    sim = nb.Simulation(g, [m], capacity=1024, seed=1, max_events=5)
    sim.push(primaries.point_beam(100))
    with pytest.raises(nb.NblError) as e:
        sim.run()
    assert e.value.status == 4
    sim.close()


def test_nan_state_is_an_error(inputs):
    from nebula_b200.synth import primaries
    g, m = _slab(inputs)
    pri = primaries.point_beam(10)
    pri["E"][3] = np.nan
    sim = nb.Simulation(g, [m], capacity=1024, seed=1)
    sim.push(pri)
    with pytest.raises(nb.NblError) as e:
        sim.run()
    assert e.value.status == 5
    sim.close()


def test_reset_gives_the_same_run_again(inputs):
    from nebula_b200.synth import primaries
    g, m = _slab(inputs)
    pri = primaries.point_beam(1500)
    sim = nb.Simulation(g, [m], capacity=1 << 12, seed=4, tally=(2, 2))
    outs = []
    for _ in range(2):
        sim.reset()
        sim.push(pri)
        sim.run()
        outs.append((_sorted(sim.flush_detected()), [t.tobytes() for t in sim.tallies()]))
    assert outs[0] == outs[1]
    sim.close()


def test_record_sink_streams_every_record(inputs):
    """Records written by the kernel straight into a host sink (page-locked,
    mapped) are exactly the records a plain drain returns, run after run; a
    sink too small for a run's records is an overflow error."""
    import torch
    from nebula_b200.synth import primaries
    g, m = _slab(inputs)
    pri = primaries.point_beam(4000)
    a = nb.Simulation(g, [m], capacity=1 << 12, seed=17, record_capacity=1 << 12)
    a.push(pri)
    a.run()
    ref = a.flush_detected()
    a.close()
    pinned = torch.empty(len(ref) * 36 + 36 * 1024, dtype=torch.uint8).pin_memory()
    sink = np.frombuffer(pinned.numpy(), dtype=nb.PRI_DTYPE)
    b = nb.Simulation(g, [m], capacity=1 << 12, seed=17, record_capacity=1 << 12)
    b.set_record_sink(sink)
    for _ in range(2):                       # reset restarts the sink
        b.reset()
        b.push(pri)
        b.run()
        got = b.sink_records().copy()
        assert len(got) == len(ref) and _sorted(got) == _sorted(ref)
        assert len(b.flush_detected()) == 0
    # pageable memory is page-locked by the library
    plain = np.zeros(len(ref) + 100, nb.PRI_DTYPE)
    b.set_record_sink(plain)
    b.reset()
    b.push(pri)
    b.run()
    assert _sorted(b.sink_records().copy()) == _sorted(ref)
    # too small
    small = np.zeros(len(ref) // 3, nb.PRI_DTYPE)
    b.set_record_sink(small)
    b.reset()
    b.push(pri)
    with pytest.raises(nb.NblError) as e:
        b.run()
    assert e.value.status == 6
    # removing the sink returns to the device buffer
    b.set_record_sink(None)
    b.reset()
    b.push(pri)
    b.run()
    assert _sorted(b.flush_detected()) == _sorted(ref)
    b.close()


def test_distinct_handles_run_concurrently_from_host_threads(inputs):
    """Calls on distinct simulation handles may come from different host
    threads at the same time (each handle has its own stream, buffers and
    graphs, captured in thread-local mode): four runs in four threads give
    exactly the records of the same four runs made one after another."""
    import threading
    from nebula_b200.synth import primaries
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    ms = [nb.Material.load(inputs["si.nmat"]), nb.Material.load(inputs["pmma.nmat"])]
    pri = primaries.raster_scan(16, 16, 40, 0.5, 500.0, 40.0, spot_sigma=1.0, seed=3)
    seeds = [101, 202, 303, 404]

    def one(seed):
        sim = nb.Simulation(g, ms, capacity=1 << 14, seed=seed)
        sim.push(pri)
        sim.run()
        rec = sim.flush_detected()
        sim.close()
        return _sorted(rec)

    alone = [one(s) for s in seeds]
    together = [None] * len(seeds)
    errors = []

    def worker(k):
        try:
            together[k] = one(seeds[k])
        except Exception as e:  # reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(len(seeds))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    assert together == alone


def test_resumed_and_sharded_scans_give_the_whole_scans_records(inputs):
    """A primary's random numbers are keyed by its index in the scan: a scan
    resumed at primary k (offset k) or split into shards (each with its first
    index) gives exactly the records of the whole scan run at once, on any
    capacity; without the offset a resumed part would reuse the first
    primaries' streams."""
    from nebula_b200.synth import primaries
    from nebula_b200 import replicas
    g = nb.Geometry.from_tri_file(inputs["grating.tri"])
    ms = [nb.Material.load(inputs["si.nmat"]), nb.Material.load(inputs["pmma.nmat"])]
    pri = primaries.raster_scan(24, 24, 50, 0.5, 500.0, 40.0, spot_sigma=1.0, seed=8)
    n = len(pri)
    whole = nb.Simulation(g, ms, capacity=1 << 15, seed=55)
    whole.push(pri)
    whole.run()
    ref = whole.flush_detected()
    whole.close()
    sim = nb.Simulation(g, ms, capacity=1 << 12, seed=55)
    # resumed at k
    k = 10_007
    resumed = []
    for first, chunk in ((0, pri[:k]), (k, pri[k:])):
        sim.reset()
        sim.set_primary_offset(first)
        sim.push(chunk)
        sim.run()
        resumed.append(sim.flush_detected())
    assert _sorted(np.concatenate(resumed)) == _sorted(ref)
    # three shards, as the replicas would take them
    parts = []
    for rank in range(3):
        lo, hi = replicas.shard(n, rank, 3)
        sim.reset()
        sim.set_primary_offset(lo)
        sim.push(pri[lo:hi])
        sim.run()
        parts.append(sim.flush_detected())
    assert _sorted(np.concatenate(parts)) == _sorted(ref)
    # the offset is refused while primaries are queued
    sim.reset()
    sim.set_primary_offset(0)
    sim.push(pri[:10])
    with pytest.raises(nb.NblError):
        sim.set_primary_offset(5)
    # without the offset the second part runs on the first primaries' streams
    sim.reset()
    sim.set_primary_offset(0)
    sim.push(pri[k:])
    sim.run()
    assert _sorted(sim.flush_detected()) != _sorted(resumed[1])
    sim.close()


def test_loaded_transport_kernel_is_sm100():
    # the runtime's own report of the loaded kernel image: built for sm_100
    import ctypes as C
    from nebula_b200 import _capi
    v = C.c_int32()
    _capi.check(_capi.lib().nbl_debug_kernel_arch(0, C.byref(v)))
    assert v.value == 100, v.value


def test_streamed_push_equals_a_plain_push(inputs):
    """Primaries pushed from page-locked memory without waiting for the copy
    (copied in chunks while the run goes, each admitted once its chunk has
    landed) give exactly the records of a plain push: alone, after a plain
    push of the first part, and into a record sink; pageable memory is
    refused."""
    import torch
    from nebula_b200.synth import primaries
    g, m = _slab(inputs)
    pri = primaries.point_beam(200_000, energy=500.0)
    pri["px"] = np.arange(len(pri)) % 64
    sim = nb.Simulation(g, [m], capacity=1 << 16, seed=9)
    sim.push(pri)
    sim.run()
    ref = sim.flush_detected()
    pinned = torch.from_numpy(pri.view(np.uint8).copy()).pin_memory()
    view = np.frombuffer(pinned.numpy(), dtype=nb.PRI_DTYPE)
    for split in (0, 70_000):
        sim.reset()
        if split:
            sim.push(pri[:split])
        sim.push_streamed(view[split:])
        sim.run()
        got = sim.flush_detected()
        assert len(got) == len(ref) and _sorted(got) == _sorted(ref)
        assert sim.counters()["primaries_started"] == len(pri)
    sink_mem = torch.empty((len(ref) + 1024) * 36, dtype=torch.uint8).pin_memory()
    sim.set_record_sink(np.frombuffer(sink_mem.numpy(), dtype=nb.PRI_DTYPE))
    sim.reset()
    sim.push_streamed(view)
    sim.run()
    assert _sorted(sim.sink_records().copy()) == _sorted(ref)
    with pytest.raises(nb.NblError) as e:
        sim.push_streamed(pri.copy())
    assert e.value.status == 1 and "page-locked" in str(e.value)
    # a plain array page-locked in place streams the same way
    plain = pri.copy()
    nb.page_lock(plain)
    with pytest.raises(nb.NblError) as e:
        nb.page_lock(plain)
    assert e.value.status == 1 and "already page-locked" in str(e.value)
    sim.set_record_sink(None)
    sim.reset()
    sim.push_streamed(plain)
    sim.run()
    assert _sorted(sim.flush_detected()) == _sorted(ref)
    nb.page_unlock(plain)
    sim.close()


def test_stepped_run_through_two_alternating_small_sinks(inputs):
    """A stepped run whose records far outgrow the sink: each step stops when
    the sink is full, the records that did not fit wait and go first into
    the next sink, and the sinks taken in turn hold exactly the records of a
    plain run.  nbl_sim_run with the same small sink still reports the
    overflow."""
    import torch
    from nebula_b200.synth import primaries
    g, m = _slab(inputs)
    pri = primaries.point_beam(60_000, energy=800.0)
    sim = nb.Simulation(g, [m], capacity=1 << 15, seed=21)
    sim.push(pri)
    sim.run()
    ref = sim.flush_detected()
    cap = len(ref) // 9
    mem = [torch.empty(cap * 36, dtype=torch.uint8).pin_memory() for _ in range(2)]
    sinks = [np.frombuffer(x.numpy(), dtype=nb.PRI_DTYPE) for x in mem]
    sim.reset()
    cur = 0
    sim.set_record_sink(sinks[cur])
    sim.push(pri)
    parts, full_stops = [], 0
    while True:
        running = sim.do_iteration(24)
        n = len(sim.sink_records())
        if n == cap:
            full_stops += 1
            parts.append(sim.sink_records().copy())
            cur ^= 1
            sim.set_record_sink(sinks[cur])
            continue
        if running == 0:
            parts.append(sim.sink_records().copy())
            break
    got = np.concatenate(parts)
    assert full_stops >= 8
    assert len(got) == len(ref) and _sorted(got) == _sorted(ref)
    sim.reset()
    sim.push(pri)
    with pytest.raises(nb.NblError) as e:
        sim.run()
    assert e.value.status == 6
    sim.close()
