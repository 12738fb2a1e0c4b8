"""Benchmark: primaries/s of the plain wavefront transport on one B200.

Workload (one step): the line-space grating scan -- 8 PMMA-like trapezoidal
lines (pitch 32 nm, top CD 16 nm, 86 deg sidewalls, 30 nm high, 4 144
triangles) on a Si-like substrate; 256 x 256 pixels at 0.5 nm x 100 primaries
per pixel = 6 553 600 primaries at 500 eV with a 1 nm Gaussian spot;
detector plane at z = 50 nm.  Synthetic geometry, materials and primaries of
those shapes (no external data).  A step is the whole scan: every primary
and its full secondary cascade.

value: primaries/s with the primary records already in HBM when the timed
       region starts (a device-to-device push, then the run).
e2e:   the same through the public API from pinned host records: host->device
       copy of the primaries (streamed in chunks while the run starts), the
       run (every detected 36-byte record copied into a pinned host buffer
       while the run goes), and the device->host copy of the tallies, all
       inside the timed region.

The same line also carries: the mixed 64-job batch, batched kernel against
the plain kernel job after job (``batched``); the seed-replay adjoint against
the forward run on the 64 x 64 x 10^4 grating scan, with finite differences
(``adjoint``); the full 512 x 512 x 200 rough-lines scan on its 1.2 M-triangle
mesh (``rough_lines``); the reference CPU driver on a bounded sample
(``cpu_baseline``); the transport kernel's roofline (``roofline``) and the
SM clocks sampled during the timed region (``clocks``).

Multi-GPU (torchrun): replicas, one scan per rank with its own seed (weak
scaling); time = max over ranks.  The single-GPU measurements (batched,
adjoint, rough lines, CPU baseline) are on the one-GPU line only.  --impl reference times the reference's own
multithreaded CPU driver (oracle/_ref/nebula_cpu_mt built from its sources)
on a bounded sample of the same scan with all host threads; its line also
carries the reference's own GPU driver (oracle/_ref/nebula_gpu, gpu_main.cu
built for sm_100a) timed on 8 copies of the full scan on one GPU, and the same
driver run job after job on the mixed 64-job batch (oracle/_ref/ref_gpu_jobs).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "primaries/s on 1 B200, plain vs batched; adjoint:forward time at yield err ≤3σ"
BYTES_PER_EVENT = 96   # 48-byte electron state read + written per event
# DRAM bytes (read + write) per event of the transport kernel, measured on a
# bounded case of this workload: the same grating scan at a pool of 2^20
# (4.8 GB on the device), one whole graph of 6 launches in the middle of the
# scan (launches 240-245, two ncu captures of 3 launches, warm L2:
# --cache-control none), dram__bytes_read.sum + dram__bytes_write.sum over
# those launches / the free flights of that graph (--trace-graphs).  It
# exceeds the 96 algorithmic bytes because a flight whose walk continues in
# the next iteration reads and writes its state again, plus 32 bytes of walk
# state each way.
DRAM_BYTES_PER_EVENT = 141.2


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, t0=None, t1=None):
        """Median SM clock, its maximum and the throttle reasons seen in the
        samples taken between t0 and t1 (time.time(); default: all)."""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, ln in self.lines:
            if (t0 is not None and ts < t0) or (t1 is not None and ts > t1):
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_inputs(workdir, seed):
    from nebula_b200.synth import workloads, geometry, materials, nmat
    w = workloads.grating(seed=seed)
    tri = os.path.join(workdir, "grating.tri")
    geometry.write_tri(tri, w.triangles)
    mats = []
    for spec in w.material_specs:
        p = os.path.join(workdir, spec.name + ".nmat")
        nmat.write(p, materials.build_raw_material(spec))
        mats.append(p)
    return w, tri, mats


# ---------------------------------------------------------------------------- CPU
def run_reference_cpu(tri, mats, pri_records, workdir):
    """The reference's own multithreaded CPU driver on the given primaries.
    Returns (primaries/s from its 'Simulation' timer, seconds, wall seconds)."""
    from nebula_b200.synth import primaries
    from oracle import oracle as O
    pri_path = os.path.join(workdir, "sample.pri")
    primaries.write_pri(pri_path, pri_records)
    t0 = time.time()
    r = subprocess.run([O.REF_CPU_MT, tri, pri_path] + mats, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                       text=True)
    wall = time.time() - t0
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    m = re.search(r"Simulation:\s*([0-9.]+)", r.stderr)
    sim_s = float(m.group(1)) if m else wall
    return len(pri_records) / sim_s, sim_s, wall


def cpu_sample(w, cores, per_core):
    """A bounded, contiguous block of pixels of the scan (rows from the top)."""
    n_pix = max(1, int(cores * per_core) // 100)
    return w.primaries[: n_pix * 100], n_pix


def cpu_baseline(w, tri, mats, workdir):
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    # ~10k primaries/s per core: ~15 s of work, so the reference's whole-second
    # "Simulation" timer is within a few percent
    sample, n_pix = cpu_sample(w, cores, 150000)
    if os.path.exists(O.REF_CPU_MT):
        rate, sim_s, wall = run_reference_cpu(tri, mats, sample, workdir)
        return {"value": rate, "unit": "primaries/s", "cores": cores, "kind": "reference",
                "sample": "%d pixels x 100 primaries (%d) of the scan, reference nebula_cpu_mt, %d threads, "
                          "its Simulation timer %.2f s" % (n_pix, len(sample), cores, sim_s)}
    # the oracle port when the reference build is absent
    import nebula_b200 as nb  # noqa: F401
    om = [O.Material(p) for p in mats]
    g = nb.Geometry.from_tri_file(tri)
    od, tr = g.export()
    inf = g.info()
    t11 = np.concatenate([np.stack([tr["material_in"], tr["material_out"]], 1).astype(np.float32),
                          tr["r0"], tr["e1"], tr["e2"]], 1)
    og = O.Geometry(od, t11, inf["center"], inf["halfsize"], inf["max_extent"])
    t0 = time.time()
    O.simulate(og, om, sample, 1, threads=cores)
    dt = time.time() - t0
    return {"value": len(sample) / dt, "unit": "primaries/s", "cores": cores, "kind": "port",
            "sample": "%d primaries of the scan, oracle restatement, %d threads" % (len(sample), cores)}


def _cuda_visible():
    # gpu_main.cu never returns without a GPU (it waits for its per-GPU
    # worker threads), so it is only started where one is visible
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def run_reference_gpu(tri, mats, pri_records, workdir, repeat, device=0):
    """The reference's own GPU driver (oracle/_ref/nebula_gpu: gpu_main.cu
    unmodified, built for sm_100a) on `repeat` copies of the given primaries,
    on one GPU, its records to /dev/null.  Its "Simulation" timer polls once a
    second, so the rate is also taken from the slope of its per-second
    progress line (primaries taken from its work pool)."""
    from oracle import oracle as O
    pri_path = os.path.join(workdir, "ref_gpu.pri")
    raw = np.ascontiguousarray(pri_records).tobytes()
    with open(pri_path, "wb") as f:
        for _ in range(repeat):
            f.write(raw)
    n = repeat * len(pri_records)
    # one GPU: the device-th of the ones this process may see
    visible = [x for x in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if x.strip()]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=visible[device] if device < len(visible) else str(device))
    try:
        with open(os.devnull, "wb") as sink, ClockSampler(device) as clk:
            r = subprocess.run([O.REF_GPU, tri, pri_path] + mats, stdout=sink, stderr=subprocess.PIPE, text=True,
                               env=env, timeout=300)
    finally:
        os.remove(pri_path)
    if r.returncode != 0 or "Simulation successful" not in r.stderr:
        raise RuntimeError(r.stderr[-500:])
    m = re.search(r"Simulation:\s*([0-9.]+)", r.stderr)
    sim_s = float(m.group(1))
    prog = [float(x) for x in re.findall(r"Progress ([0-9.]+)%", r.stderr)]
    slope = None
    if len(prog) >= 3:
        # ticks 1 .. k-1 are one second apart while the pool drains
        slope = (prog[-2] - prog[0]) / (len(prog) - 2) / 100.0 * n
    return {"value": slope if slope else n / sim_s, "unit": "primaries/s",
            "kind": "reference GPU driver (gpu_main.cu unmodified, sm_100a, default capacity 10^6)",
            "sample": "%d x the 256x256x100 scan (%d primaries), one GPU" % (repeat, n),
            "simulation_timer_s": sim_s, "rate_from_timer": n / sim_s, "rate_from_progress": slope,
            "clocks": clk.summary()}


def run_reference_gpu_jobs(workdir, device=0):
    """The reference's plain GPU driver job after job on the mixed 64-job
    batch (oracle/_ref/ref_gpu_jobs: the reference's gpu_driver calls
    sequenced as gpu_main.cu's worker does -- prescan, then frames -- with
    per-phase timers instead of its once-a-second poll).  Its run time is the
    sum of the jobs' prescan and frame phases; driver construction (pool
    allocation, 10^6 cuRAND states) is reported apart, as pool creation is
    not timed for the plain kernel either."""
    from oracle import oracle as O
    from nebula_b200.synth import workloads, geometry, materials, nmat, primaries
    gt, specs, jobs, _ = workloads.batch()
    tris = []
    for i, t in enumerate(gt):
        p = os.path.join(workdir, "batch_g%d.tri" % i)
        geometry.write_tri(p, t)
        tris.append(p)
    mats = []
    for sp in specs:
        p = os.path.join(workdir, "batch_%s.nmat" % sp.name)
        nmat.write(p, materials.build_raw_material(sp))
        mats.append(p)
    lines = []
    for k, (gi, seed, pri) in enumerate(jobs):
        p = os.path.join(workdir, "batch_j%d.pri" % k)
        primaries.write_pri(p, pri)
        lines.append("%s %s %d" % (tris[gi], p, seed))
    jobs_txt = os.path.join(workdir, "batch_jobs.txt")
    with open(jobs_txt, "w") as f:
        f.write("\n".join(lines) + "\n")
    visible = [x for x in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if x.strip()]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=visible[device] if device < len(visible) else str(device))
    with ClockSampler(device) as clk:
        r = subprocess.run([O.REF_GPU_JOBS, jobs_txt] + mats, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                           text=True, env=env, timeout=600)
    if r.returncode != 0:
        raise RuntimeError((r.stdout + r.stderr)[-500:])
    per_job = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    n = sum(j["primaries"] for j in per_job)
    run_s = sum(j["prescan_s"] + j["frames_s"] for j in per_job)
    return {"value": n / run_s, "unit": "primaries/s",
            "kind": "reference GPU driver (drivers/gpu/gpu_driver.inl) job after job, gpu_main.cu's worker steps",
            "workload": "mixed batch: %d jobs, %d primaries" % (len(per_job), n),
            "seconds": run_s, "construct_seconds": sum(j["construct_s"] for j in per_job),
            "prescan_seconds": sum(j["prescan_s"] for j in per_job),
            "se": sum(j["se"] for j in per_job), "bse": sum(j["bse"] for j in per_job),
            "clocks": clk.summary()}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    if not os.path.exists(O.REF_CPU_MT):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build oracle/_ref/nebula_cpu_mt missing"}))
        return
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        w, tri, mats = make_inputs(d, seed=7)
        sample, n_pix = cpu_sample(w, cores, 100000)
        for _ in range(args.warmup):
            run_reference_cpu(tri, mats, sample[: max(100, len(sample) // 10)], d)
        rates, secs = [], []
        for _ in range(args.steps):
            r, s, _ = run_reference_cpu(tri, mats, sample, d)
            rates.append(r)
            secs.append(s)
        ref_gpu = None
        if not args.no_reference_gpu and os.path.exists(O.REF_GPU) and _cuda_visible():
            try:
                ref_gpu = run_reference_gpu(tri, mats, w.primaries, d, repeat=8,
                                            device=int(os.environ.get("LOCAL_RANK", "0")))
            except Exception as e:  # reported, not fatal
                ref_gpu = {"value": None, "error": str(e)[:300]}
        ref_gpu_batch = None
        if not args.no_reference_gpu and os.path.exists(O.REF_GPU_JOBS) and _cuda_visible():
            try:
                ref_gpu_batch = run_reference_gpu_jobs(d, device=int(os.environ.get("LOCAL_RANK", "0")))
            except Exception as e:  # reported, not fatal
                ref_gpu_batch = {"value": None, "error": str(e)[:300]}
    value = len(sample) * len(secs) / sum(secs)
    desc = "%d pixels x 100 primaries (%d) of the scan per step, reference nebula_cpu_mt, %d threads" % (
        n_pix, len(sample), cores)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "primaries/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * float(np.mean(secs)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "grating-256x256x100-500eV (bounded CPU sample)", "sample": desc},
        "cpu_baseline": {"value": value, "unit": "primaries/s", "cores": cores, "kind": "reference", "sample": desc},
        "e2e": {"value": value, "unit": "primaries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if ref_gpu is not None:
        line["reference_gpu"] = ref_gpu
    if ref_gpu_batch is not None:
        line["reference_gpu_mixed_batch"] = ref_gpu_batch
    print(json.dumps(line))


# ---------------------------------------------------------------------------- batch
def batched_vs_plain(args, dev, workdir):
    """The mixed 64-job batch: one persistent batched launch against the
    plain wavefront run job after job (one pool reused per geometry, with the
    plain bench's capacity; pool creation not timed), same seeds, so per-job
    records must be identical.  Both arms deliver the same outputs -- every
    job's detected 36-byte records on the host -- and are timed two ways:

    device: the transport kernels alone (CUDA events around the batched
            launch; around every graph of the plain runs, summed);
    e2e:    wall time from the host primaries to the host records (batched:
            upload of the batch's primaries and job table, the launch, the
            records' read-back; plain: per job the push, the run and the
            drain of its records).

    Batch parameters come from the autotuner's stored choice when present."""
    import torch
    import nebula_b200 as nb
    from nebula_b200 import autotune
    from nebula_b200.tune_mixed_batch import load_mixed_batch, OUT as TUNED
    geoms, mats, jobs, desc = load_mixed_batch(workdir)
    n_pri = sum(len(p) for _, _, p in jobs)
    if os.path.exists(TUNED):
        best = autotune.load(TUNED)
        params = dict(capacity=int(best["capacity"]), block=int(best["block"]), threshold=float(best["threshold"]),
                      walk_cells=int(best.get("walk_cells", 1)),
                      source="autotuner (nebula_b200/tuned/mixed_batch.json)")
    else:
        params = dict(capacity=1 << 22, block=512, threshold=0.5, walk_cells=1, source="default")
    b = nb.Batch(geoms, mats, capacity=params["capacity"], block_size=params["block"],
                 refill_threshold=params["threshold"], device=dev, record_capacity=1 << 24,
                 walk_cells=params["walk_cells"])

    # the batch's primaries laid end to end, as the caller holds them (the
    # plain arm holds one array per job)
    all_pri = np.ascontiguousarray(np.concatenate([p for _, _, p in jobs]), nb.PRI_DTYPE)

    def batch_pass():
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        b.set_jobs(jobs, primaries=all_pri)
        b.run()
        rec, job = b.records()                  # every job's records and their job ids, on the host
        return (rec, job), time.perf_counter() - t0, b.kernel_ms()

    batch_pass()                                # warm-up
    b_wall, b_dev = [], []
    for _ in range(args.steps):
        _, w, m = batch_pass()
        b_wall.append(w)
        b_dev.append(m)
    c = b.counters()
    recs_b = b.job_records()
    b.close()

    def plain_pass():
        recs, ms_dev, wall, flights = [], 0.0, 0.0, 0
        cur = None
        for gi, seed, pri in jobs:
            if cur is None or cur[0] != gi:
                if cur is not None:
                    cur[1].close()
                cur = (gi, nb.Simulation(geoms[gi], mats[: (1 if gi == 0 else 2)], capacity=args.capacity,
                                         seed=seed, record_capacity=1 << 24, device=dev))
            s = cur[1]
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            s.reset()
            s.set_seed(seed)
            s.push(pri)
            s.run()
            rec = s.flush_detected()
            wall += time.perf_counter() - t0
            ms_dev += s.kernel_ms()
            flights += s.counters()["flights"]
            recs.append(rec)
        cur[1].close()
        return recs, wall, ms_dev, flights

    plain_pass()                                # warm-up
    p_wall, p_dev = [], []
    for _ in range(args.steps):
        recs_p, w, m, p_flights = plain_pass()
        p_wall.append(w)
        p_dev.append(m)
    srt = lambda r: np.sort(r.view(np.dtype((np.void, 36))).ravel()).tobytes()
    identical = all(len(x) == len(y) and srt(x) == srt(y) for x, y in zip(recs_b, recs_p))
    bd, pd = float(np.mean(b_dev)) / 1e3, float(np.mean(p_dev)) / 1e3
    bw, pw = float(np.mean(b_wall)), float(np.mean(p_wall))
    return {"workload": "mixed batch: %d jobs, %d primaries (slab / gratings pitch 20-64 nm, 200 eV-20 keV, "
                        "1e3-1e6 primaries per job)" % (len(jobs), n_pri),
            "value": n_pri / bd, "unit": "primaries/s", "seconds": bd,
            "plain_value": n_pri / pd, "plain_seconds": pd,
            "ratio_batched_over_plain": pd / bd,
            "e2e": {"value": n_pri / bw, "seconds": bw, "plain_value": n_pri / pw, "plain_seconds": pw,
                    "ratio_batched_over_plain": pw / bw,
                    "what": "host primaries to host records, both arms (uploads, launches, record read-back)"},
            "flights_per_s": c["flights"] / bd, "plain_flights_per_s": p_flights / pd,
            "timing": "value / plain_value: transport kernels only (CUDA events), both arms",
            "flights": c["flights"], "iterations": c["iterations"], "spilled": c["spilled"],
            "records": int(sum(len(r) for r in recs_b)), "per_job_records_identical": bool(identical),
            "se_total": int(sum(int((r["E"] < 50).sum()) for r in recs_b)),
            "bse_total": int(sum(int((r["E"] >= 50).sum()) for r in recs_b)),
            "params": params, "launches_per_run": 1}


# ---------------------------------------------------------------------------- adjoint
ADJ_NAMES = ["s_inel_si", "s_el_si", "W_si", "s_inel_pmma", "s_el_pmma", "W_pmma"]


def adjoint_vs_forward(args, dev, workdir, nx=64, per_pixel=10_000, fd=True, seeds=16):
    """Grating scan of 64 x 64 pixels x 1e4 primaries at 500 eV: the forward
    run against the seed-replay adjoint run (per-pixel gradients of the SE
    yield for the 6 material parameters: score functions for the
    mean-free-path scales, a replay shifted by +-0.05 eV per primary for the
    work functions), wall time of each including the host push and the
    drain.

    With ``fd``, the gradients against central finite differences with
    common random numbers (the same seed in the + and - runs), averaged over
    independent seeds (mean and standard error over seeds, the seeds'
    adjoint - difference pairs giving the error of the comparison):
    all six parameters with the steps 1 % of a scale / 0.05 eV of a work
    function on the first two seeds; the Si inelastic scale, a gradient of
    ~0.003 that is a near cancellation of the trench's and the lines'
    parts, also with a 5 % step on all ``seeds`` seeds, which is what brings
    its difference's standard error near 1.5 %."""
    import torch
    import nebula_b200 as nb
    from nebula_b200.synth import workloads, geometry, materials, nmat
    from nebula_b200.torch_adjoint import ScanProblem
    w = workloads.grating(nx=nx, ny=nx, per_pixel=per_pixel)
    tri = os.path.join(workdir, "adj.tri")
    geometry.write_tri(tri, w.triangles)
    ms = []
    for sp in w.material_specs:
        pth = os.path.join(workdir, "adj_" + sp.name + ".nmat")
        nmat.write(pth, materials.build_raw_material(sp))
        ms.append(nb.Material.load(pth))
    g = nb.Geometry.from_tri_file(tri)
    prob = ScanProblem(g, ms, w.primaries, (nx, nx), seed=11, capacity=1 << 22, device=dev)
    th0 = prob.theta0().numpy()
    prob.forward(th0)
    prob.jacobian(th0)                                    # warm-up
    tf, ta, kf, ka = [], [], [], []
    for _ in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        y = prob.forward(th0)
        tf.append(time.perf_counter() - t0)
        kf.append(prob.forward_sim.kernel_ms())
        t0 = time.perf_counter()
        prob.jacobian(th0)
        ta.append(time.perf_counter() - t0)
        ka.append(prob.adjoint_sim.kernel_ms())
    W = prob.per_pixel
    N = W.sum()
    n_pix = W.size
    ypix = y * W
    out = {"workload": "grating-%dx%dx%d-500eV (%d primaries), 6 parameters" % (nx, nx, per_pixel, int(N)),
           "forward_seconds": float(np.mean(tf)), "adjoint_seconds": float(np.mean(ta)),
           "ratio_adjoint_over_forward": float(np.mean(ta) / np.mean(tf)),
           "ratio_transport_kernels": float(np.mean(ka) / np.mean(kf)),
           "work_function_step_eV": prob.w_step,
           "se_yield": float(ypix.sum() / N), "se_yield_sigma": float(ypix.std(ddof=1) * np.sqrt(n_pix) / N)}
    if fd:
        # per seed: the adjoint gradients and the differences asked for
        samples = {}                       # (param, step) -> list of (adjoint, difference)
        for si in range(seeds):
            prob.set_seed(11 + si)
            J = prob.jacobian(th0)         # runs the forward pass at th0 first
            adj = (J * W[..., None]).sum((0, 1)) / N
            plan = [(k, 0.05 if k % 3 == 2 else 0.01) for k in range(6)] if si < 2 else []
            plan.append((0, 0.05))
            for k, step in plan:
                delta = step if k % 3 == 2 else step * float(th0[k])
                tp, tm = th0.copy(), th0.copy()
                tp[k] += delta
                tm[k] -= delta
                fdv = float(((prob.forward(tp) - prob.forward(tm)) * W).sum() / N / (2 * delta))
                samples.setdefault((k, step), []).append((float(adj[k]), fdv))
        rows = {}
        for (k, step), v in sorted(samples.items()):
            a = np.array(v)
            n = len(a)
            se = lambda x: float(x.std(ddof=1) / np.sqrt(n)) if n > 1 else None
            d = a[:, 0] - a[:, 1]
            fd_mean = float(a[:, 1].mean())
            key = ADJ_NAMES[k] + ("" if (k % 3 == 2 or step == 0.01) else "_step5pct")
            rows[key] = {"seeds": n, "fd_step": ("%g eV" % step) if k % 3 == 2 else ("%g %%" % (100 * step)),
                         "adjoint": float(a[:, 0].mean()), "adjoint_se": se(a[:, 0]),
                         "crn_fd": fd_mean, "crn_fd_se": se(a[:, 1]),
                         "diff_pct": float(100 * d.mean() / abs(fd_mean)),
                         "diff_se_pct": (100 * se(d) / abs(fd_mean)) if n > 1 else None}
        out["dYse_dtheta"] = rows
        out["fd_seeds"] = "seeds 11..%d (per-seed common random numbers)" % (10 + seeds)
    prob.close()
    return out


# ---------------------------------------------------------------------------- rough lines
def device_raster_scan(nx, ny, per_pixel, pixel_size, energy, z0, spot_sigma, seed, dev):
    """A raster scan built directly in device memory as 36-byte records
    (pixel-major, ``per_pixel`` primaries per pixel centre with a Gaussian
    spot, normal incidence): the same layout as the host generator's, random
    spot offsets from torch's device generator."""
    import torch
    n = nx * ny * per_pixel
    gen = torch.Generator(device=f"cuda:{dev}")
    gen.manual_seed(seed)
    words = torch.zeros((n, 9), dtype=torch.float32, device=f"cuda:{dev}")
    k = torch.arange(n, device=f"cuda:{dev}", dtype=torch.int64) // per_pixel
    px, py = k % nx, k // nx
    off = torch.randn((n, 2), generator=gen, device=f"cuda:{dev}", dtype=torch.float32) * spot_sigma
    words[:, 0] = (px.to(torch.float32) - (nx - 1) / 2.0) * pixel_size + off[:, 0]
    words[:, 1] = (py.to(torch.float32) - (ny - 1) / 2.0) * pixel_size + off[:, 1]
    words[:, 2] = z0
    words[:, 5] = -1.0
    words[:, 6] = energy
    iw = words.view(torch.int32)
    iw[:, 7] = px.to(torch.int32)
    iw[:, 8] = py.to(torch.int32)
    del off, k, px, py
    return words


def rough_lines(args, dev, workdir):
    """Large-mesh plain method: the 16-line grating with line-edge roughness
    (1.2 M triangles, octree depth <= 12, <= 16 triangles per leaf), the full
    512 x 512 pixel scan x 200 primaries at 300 eV (52.4 M primaries, built in
    device memory).  Reports the host octree build time (all host threads)
    and primaries/s over the run's wall time, every detected record delivered
    to page-locked host memory (the record sink, copied there graph by graph
    while the run goes) and the per-pixel tallies on the device."""
    import torch
    import nebula_b200 as nb
    from nebula_b200.synth import geometry, materials, nmat
    t0 = time.perf_counter()
    tri_rows = geometry.rough_grating()
    t_gen = time.perf_counter() - t0
    tris = nb.triangles_from_vertices(tri_rows)
    t0 = time.perf_counter()
    g = nb.Geometry.from_triangles(tris, max_depth=12, split_count=16)
    t_build = time.perf_counter() - t0
    ms = []
    for sp in (materials.silicon(), materials.pmma()):
        pth = os.path.join(workdir, "rough_" + sp.name + ".nmat")
        nmat.write(pth, materials.build_raw_material(sp))
        ms.append(nb.Material.load(pth))
    words = device_raster_scan(512, 512, 200, 0.5, 300.0, 40.0, 1.0, 11, dev)
    n = words.shape[0]
    sim = nb.Simulation(g, ms, capacity=args.capacity, seed=31, record_capacity=1 << 24, tally=(512, 512), device=dev,
                        walk_cells=args.walk_cells)
    # ~1.05 detected electrons per primary: room for 1.25 per primary
    sink_cap = n * 5 // 4
    sink_host = torch.empty(sink_cap * 36, dtype=torch.uint8).pin_memory()
    sim.set_record_sink(np.frombuffer(sink_host.numpy(), dtype=nb.PRI_DTYPE))
    pri_dev = words
    sim.reset()
    sim.push_device(pri_dev.data_ptr(), n)
    sim.run()                                          # warm-up
    ms_list, flights = [], 0
    steps = max(1, min(args.steps, 2))
    for _ in range(steps):
        sim.reset()
        sim.push_device(pri_dev.data_ptr(), n)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        sim.run()
        torch.cuda.synchronize(dev)
        ms_list.append((time.perf_counter() - t0) * 1e3)
        flights = sim.counters()["flights"]
    n_rec = len(sim.sink_records())
    se, bse, _ = sim.tallies()
    info = g.info()
    sim.close()
    g.close()
    t = float(np.mean(ms_list)) / 1e3
    return {"workload": "rough lines: 16 lines, %d triangles, 512 x 512 pixels x 200 primaries at 300 eV (%d primaries)"
                        % (len(tris), n),
            "value": n / t, "unit": "primaries/s", "seconds": t, "events_per_primary": flights / n,
            "se_yield": float(se.sum()) / n, "bse_yield": float(bse.sum()) / n,
            "records": n_rec, "records_to": "page-locked host memory, copied graph by graph during the run",
            "octree_words": int(info["n_octree"]), "octree_build_seconds": t_build,
            "octree_build_threads": os.cpu_count(), "mesh_generation_seconds": t_gen}


# ---------------------------------------------------------------------------- profiling cases
def run_case(args):
    """A bounded run of one workload for profilers and timing sweeps
    (``--case``): ``--repeat`` runs after one warm-up run, one JSON line with
    the transport kernel time, primaries/s and events per primary.

    grating: a ``--pixels`` x ``--pixels`` block at the centre of the 256 x 256
             grating raster, ``--per-pixel`` primaries at ``--energy`` (500 eV);
    rough:   the same block at the centre of the rough lines' 512 x 512 raster
             (1.2 M triangles, octree depth <= 12; 300 eV unless given);
    slab:    ``pixels^2 x per_pixel`` primaries on the 1 um Si slab;
    batch:   the 64-job mixed batch with every job's primaries scaled by
             ``--batch-scale``, in the batched persistent kernel;
    driver:  the drop-in executable (nebula_b200/nebula_b200_gpu) on
             ``--repeat`` copies of the whole grating scan, its records to a
             file, as the reference executable is timed (its "Simulation"
             phase; ``--capacity`` passed on).
    Small enough for an ncu capture of a few launches on one GPU (driver
    aside)."""
    import nebula_b200 as nb
    from nebula_b200.synth import workloads, geometry, materials, nmat
    if args.case == "driver":
        from nebula_b200 import build
        with tempfile.TemporaryDirectory() as d:
            w, tri, mats = make_inputs(d, seed=7)
            pri_path = os.path.join(d, "scan.pri")
            raw = np.ascontiguousarray(w.primaries).tobytes()
            with open(pri_path, "wb") as f:
                for _ in range(args.repeat):
                    f.write(raw)
            out = os.path.join(d, "detected.bin")
            t0 = time.perf_counter()
            with open(out, "wb") as sink:
                r = subprocess.run([build.DRIVER, "--capacity", str(args.capacity), tri, pri_path] + mats,
                                   stdout=sink, stderr=subprocess.PIPE, text=True, timeout=600)
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                raise RuntimeError(r.stderr[-1000:])
            phases = dict((k.strip(), float(v)) for k, v in
                          re.findall(r"([A-Za-z][A-Za-z ]+):\s*([0-9.]+)", r.stderr.split("Timing (seconds):")[-1]))
            n = args.repeat * len(w.primaries)
            print(json.dumps({"case": "drop-in executable, %d x the 256x256x100 grating scan" % args.repeat,
                              "primaries": n, "record_bytes": os.path.getsize(out), "phases_s": phases,
                              "wall_s": wall, "primaries_per_s": n / phases["Simulation"]}))
        return
    if args.case == "batch":
        from nebula_b200.tune_mixed_batch import load_mixed_batch
        with tempfile.TemporaryDirectory() as d:
            geoms, mats, jobs, _ = load_mixed_batch(d, scale=args.batch_scale)
            b = nb.Batch(geoms, mats, capacity=args.capacity, block_size=args.block or 512, refill_threshold=0.5,
                         walk_cells=args.walk_cells)
            b.set_jobs(jobs)
            runs = []
            for r in range(args.repeat + 1):
                b.run()
                if r > 0:
                    runs.append(b.kernel_ms())
            c = b.counters()
            b.close()
        n = sum(len(p) for _, _, p in jobs)
        kms = float(np.mean(runs))
        print(json.dumps({"case": "mixed batch x %g (%d jobs)" % (args.batch_scale, len(jobs)), "primaries": n,
                          "kernel_ms": kms, "primaries_per_s": n / (kms / 1e3),
                          "events_per_primary": c["flights"] / n, "iterations": c["iterations"]}))
        return
    energy = args.energy if args.energy else (300.0 if args.case == "rough" else 500.0)
    with tempfile.TemporaryDirectory() as d:
        if args.case == "grating":
            px = np.arange(128 - args.pixels // 2, 128 - args.pixels // 2 + args.pixels)
            pixels = np.stack(np.meshgrid(px, px, indexing="xy"), -1).reshape(-1, 2)
            w = workloads.grating(pixels=pixels, per_pixel=args.per_pixel, energy=energy)
        elif args.case == "rough":
            px = np.arange(256 - args.pixels // 2, 256 - args.pixels // 2 + args.pixels)
            pixels = np.stack(np.meshgrid(px, px, indexing="xy"), -1).reshape(-1, 2)
            w = workloads.rough(pixels=pixels, per_pixel=args.per_pixel, energy=energy, pixel_streams=False)
        else:
            w = workloads.slab(n_primaries=args.pixels * args.pixels * args.per_pixel, energy=energy)
        ms = []
        for sp in w.material_specs:
            p = os.path.join(d, sp.name + ".nmat")
            nmat.write(p, materials.build_raw_material(sp))
            ms.append(nb.Material.load(p))
        if args.case == "rough":
            g = nb.Geometry.from_triangles(nb.triangles_from_vertices(w.triangles), max_depth=12, split_count=16)
        else:
            tri = os.path.join(d, "g.tri")
            geometry.write_tri(tri, w.triangles)
            g = nb.Geometry.from_tri_file(tri)
        sim = nb.Simulation(g, ms, capacity=args.capacity, seed=3, record_capacity=1 << 24, block_size=args.block,
                            iterations_per_graph=args.graph_iters,
                            walk_cells=args.walk_cells)
        runs = []
        trace = []
        for r in range(args.repeat + 1):
            sim.reset()
            sim.push(w.primaries)
            t0 = time.perf_counter()
            if r == 0 and args.trace_graphs:
                # the first run graph by graph (--graph-iters iterations
                # each), with the free flights each graph made: the launch
                # index of an ncu capture maps to its graph, and so to its
                # flights per launch
                while True:
                    left = sim.do_iteration(args.graph_iters)
                    trace.append(sim.counters()["flights"])
                    if left == 0:
                        break
            else:
                sim.run()
            wall = time.perf_counter() - t0
            c = sim.counters()
            sim.flush_detected()
            if r > 0 or args.repeat == 0:
                runs.append((sim.kernel_ms(), wall, c["flights"], c["iterations"]))
        sim.close()
    n = len(w.primaries)
    kms = float(np.mean([r[0] for r in runs]))
    print(json.dumps({"case": "%s %dx%dx%d at %g eV" % (args.case, args.pixels, args.pixels, args.per_pixel, energy),
                      "primaries": n, "capacity": args.capacity,
                      "walk_cells": args.walk_cells, "kernel_ms": kms,
                      "primaries_per_s": n / (kms / 1e3), "events_per_primary": runs[-1][2] / n,
                      "iterations": runs[-1][3], "wall_s": float(np.mean([r[1] for r in runs])),
                      "flights_per_graph": list(np.diff([0] + trace).tolist()) if trace else None}))


# ---------------------------------------------------------------------------- GPU
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--capacity", type=int, default=1 << 23)
    ap.add_argument("--record-capacity", type=int, default=1 << 24)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the mixed-batch (batched vs plain) measurement")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint vs forward measurement")
    ap.add_argument("--no-rough", action="store_true", help="skip the large-mesh (rough lines) measurement")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip timing the reference's own GPU driver beside its CPU driver")
    ap.add_argument("--case", choices=["grating", "rough", "slab", "batch", "driver"],
                    help="run one bounded profiling case instead of the benchmark (see run_case)")
    ap.add_argument("--pixels", type=int, default=64, help="--case: pixels per side of the scanned block")
    ap.add_argument("--per-pixel", type=int, default=100, help="--case: primaries per pixel")
    ap.add_argument("--energy", type=float, default=0.0, help="--case: beam energy in eV (0: the case's own)")
    ap.add_argument("--repeat", type=int, default=1, help="--case: timed runs after one warm-up run")
    ap.add_argument("--batch-scale", type=float, default=0.02, help="--case batch: fraction of every job's primaries")
    ap.add_argument("--block", type=int, default=0, help="--case: threads per block of the kernel (0: default)")
    ap.add_argument("--graph-iters", type=int, default=24,
                    help="--case: wavefront iterations per CUDA graph (a multiple of 6)")
    ap.add_argument("--trace-graphs", action="store_true",
                    help="--case: run the first run graph by graph and report the flights of each graph")
    ap.add_argument("--walk-cells", type=int, default=0,
                    help="leaf cells a flight's walk takes per iteration before continuing in the next (0: the "
                         "library default, 1)")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.case:
        return run_case(args)

    import torch
    import nebula_b200 as nb

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = local

    with tempfile.TemporaryDirectory() as d:
        w, tri, mats = make_inputs(d, seed=7)
        g = nb.Geometry.from_tri_file(tri)
        ms = [nb.Material.load(p) for p in mats]
        n_pri = len(w.primaries)
        stream = torch.cuda.Stream(device=dev)
        from nebula_b200 import replicas
        sim = nb.Simulation(g, ms, capacity=args.capacity, seed=replicas.replica_seed(1000, rank), device=dev,
                            tally=w.n_pixels,
                            stream=stream.cuda_stream, record_capacity=args.record_capacity,
                            walk_cells=args.walk_cells)
        pri_dev = torch.from_numpy(w.primaries.view(np.uint8)).to(f"cuda:{dev}")
        pri_host = torch.from_numpy(w.primaries.view(np.uint8).copy()).pin_memory()
        rec_host = torch.empty(args.record_capacity * 36, dtype=torch.uint8).pin_memory()
        rec_view = np.frombuffer(rec_host.numpy(), dtype=nb.PRI_DTYPE)

        def step_device():
            sim.reset()
            sim.push_device(pri_dev.data_ptr(), n_pri)
            sim.run()

        pri_host_view = np.frombuffer(pri_host.numpy(), dtype=nb.PRI_DTYPE)

        def step_e2e():
            # the primaries stream in from the pinned host buffer while the
            # run starts (each admitted once its chunk has landed); the
            # detected records are copied into the pinned host sink while
            # the run goes
            sim.reset()
            sim.push_streamed(pri_host_view)
            sim.run()
            rec = sim.sink_records()
            tal = sim.tallies()
            return rec, tal

        # clocks are sampled from the warm-up on (nvidia-smi takes a moment to
        # start); the line reports the samples inside the timed region, or
        # those of warm-up and timed region together when it is too short
        clk = ClockSampler(dev).__enter__()
        t_warm = time.time()
        for _ in range(args.warmup):
            step_device()
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()

        # timed: device-resident inputs
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        kernel_ms = 0.0
        flights = 0
        resumes = 0
        iters = 0
        detected = 0
        try:
            torch.cuda.synchronize(dev)
            t_timed = time.time()
            ev0.record(stream)
            for _ in range(args.steps):
                step_device()
                c = sim.counters()
                kernel_ms += sim.kernel_ms()
                flights += c["flights"]
                resumes += c["walk_resumes"]
                iters += c["iterations"]
                detected += c["detected"]
            ev1.record(stream)
            torch.cuda.synchronize(dev)
            t_end = time.time()
        finally:
            clk.__exit__(None, None, None)
        clocks = clk.summary(t_timed, t_end)
        clocks["window"] = "timed region"
        if clocks["samples"] < 3:
            clocks = clk.summary(t_warm, t_end)
            clocks["window"] = "warm-up and timed region"
        ms = ev0.elapsed_time(ev1)
        if dist:
            ms = replicas.max_over_ranks(ms, dist, device=f"cuda:{dev}")

        # timed: end to end from pinned host records
        h2d = n_pri * 36
        d2h = 0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sim.set_record_sink(rec_view)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.steps):
            rec, tal = step_e2e()
            d2h = len(rec) * 36 + sum(x.nbytes for x in tal if x is not None)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        e2e_ms = e0.elapsed_time(e1)
        if dist:
            e2e_ms = replicas.max_over_ranks(e2e_ms, dist, device=f"cuda:{dev}")

        value = n_pri * args.steps * world / (ms / 1000.0)
        e2e_value = n_pri * args.steps * world / (e2e_ms / 1000.0)
        peak, peak_kind = measured_peaks()
        achieved = flights * BYTES_PER_EVENT / (kernel_ms / 1000.0) / 1e9
        out = {
            "metric": METRIC, "value": value, "unit": "primaries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "grating-256x256x100-500eV", "method": "plain wavefront",
                       "primaries_per_step": n_pri, "triangles": int(len(w.triangles)),
                       "capacity": args.capacity, "parallelism": "replicas x%d" % world,
                       "l2": "inputs larger than L2 (primaries 236 MB, queues > 1 GB)"},
            "events_per_primary": flights / (n_pri * args.steps),
            "walk_resumes_per_event": resumes / max(flights, 1),
            "detected_per_primary": detected / (n_pri * args.steps),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": DRAM_BYTES_PER_EVENT * flights / max(iters, 1),
                         "traffic_unit": "bytes per launch: %.1f B per event (ncu, one graph of the same scan at a "
                                         "2^20 pool) x this run's events per launch" % DRAM_BYTES_PER_EVENT,
                         "note": "%d B algorithmic per event x %d events / transport-kernel time %.1f ms; "
                                 "peak %s" % (BYTES_PER_EVENT, flights, kernel_ms, peak_kind)},
            "e2e": {"value": e2e_value, "unit": "primaries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": iters,
            "clocks": clocks,
        }
        sim.close()
        # the single-GPU measurements ride on the one-GPU line only (every
        # rank skips them alike, so the ranks' collective steps stay equal)
        if not args.no_batch and world == 1:
            out["batched"] = batched_vs_plain(args, dev, d)
        if not args.no_adjoint and world == 1:
            out["adjoint"] = adjoint_vs_forward(args, dev, d)
        if not args.no_rough and world == 1:
            out["rough_lines"] = rough_lines(args, dev, d)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            try:
                out["cpu_baseline"] = cpu_baseline(w, tri, mats, d)
            except Exception as e:  # reported, not fatal
                out["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        if rank == 0:
            print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
