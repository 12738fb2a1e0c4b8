"""Seed-replay adjoint: without a work-function step the replay reproduces
the forward run exactly; the gradients of the total SE yield agree with
central finite differences taken with common random numbers (same seed, so
the runs share every random number): score-function estimates for the
mean-free-path scales, the shifted-replay difference for the work functions.

Tolerance of the gradient check: 5 % of the finite difference, on scans
chosen so that 3 standard errors of the difference (estimated from the
per-pixel spread, a pixel being an independent block of primaries) are at
most 5 % of it.
"""
import numpy as np
import pytest
import torch

import nebula_b200 as nb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem(tmp_path_factory):
    from nebula_b200.synth import workloads, geometry, materials, nmat
    from nebula_b200.torch_adjoint import ScanProblem
    d = tmp_path_factory.mktemp("adj")
    w = workloads.grating(nx=16, ny=16, per_pixel=2000)
    tri = str(d / "g.tri")
    geometry.write_tri(tri, w.triangles)
    ms = []
    for sp in w.material_specs:
        p = str(d / (sp.name + ".nmat"))
        nmat.write(p, materials.build_raw_material(sp))
        ms.append(nb.Material.load(p))
    g = nb.Geometry.from_tri_file(tri)
    prob = ScanProblem(g, ms, w.primaries, (16, 16), seed=11, capacity=1 << 20)
    prob.geometry, prob.materials = g, ms
    yield prob
    prob.close()


def test_adjoint_with_a_walk_cell_budget(problem):
    """Walks cut at a cell budget and continued in later iterations give the
    same adjoint tallies: the replay's records equal the unbounded run's and
    the gradient sums agree to rounding (double atomics add in another
    order)."""
    out = []
    for cells in (1 << 20, 2):
        fwd = nb.Simulation(problem.geometry, problem.materials, capacity=1 << 18, seed=5, tally=(16, 16),
                            walk_cells=cells)
        adj = nb.Simulation(problem.geometry, problem.materials, capacity=1 << 18, seed=5, tally=(16, 16),
                            adjoint=True, adjoint_w_step=0.05, walk_cells=cells)
        for s in (fwd, adj):
            s.push(problem.primaries[:60000])
            s.run()
        key = np.sort(adj.flush_detected().view(np.dtype((np.void, 36))).ravel()).tobytes()
        gs, gb = adj.gradients(fwd)
        out.append((key, gs, gb, adj.counters()["walk_resumes"]))
        fwd.close()
        adj.close()
    assert out[0][0] == out[1][0]
    assert out[0][3] == 0 and out[1][3] > 0
    for k in (1, 2):
        assert np.allclose(out[0][k], out[1][k], rtol=1e-9, atol=1e-9)


def test_adjoint_replay_reproduces_forward(problem):
    from nebula_b200.torch_adjoint import ScanProblem
    p0 = ScanProblem(problem.geometry, problem.materials, problem.primaries, (16, 16), seed=11,
                     capacity=1 << 20, w_step=0.0)
    th = p0.theta0().numpy()
    y = p0.forward(th)
    J = p0.jacobian(th)
    se_f, bse_f, _ = p0.forward_sim.tallies()
    se_a, bse_a, _ = p0.adjoint_sim.tallies()
    assert np.array_equal(se_f, se_a) and np.array_equal(bse_f, bse_a)
    assert y.sum() > 0 and np.all(np.isfinite(J))
    p0.close()


@pytest.mark.parametrize("physics", [{"interface_refraction": 0, "quantum_transmission": 0,
                                      "interface_absorption": 1, "acoustic_phonon_loss": 0}])
def test_adjoint_with_a_non_default_physics_selection(problem, physics):
    """The adjoint kernel compiled for run-time physics bits (any selection
    but the reference default): the replay without a work-function step
    still reproduces the forward run, the score-function gradient of a
    mean-free-path scale still matches its finite difference, and the
    selection changes the yields."""
    from nebula_b200.torch_adjoint import ScanProblem
    p0 = ScanProblem(problem.geometry, problem.materials, problem.primaries, (16, 16), seed=11,
                     capacity=1 << 20, w_step=0.0, physics=physics)
    th = p0.theta0().numpy()
    y = p0.forward(th)
    J = p0.jacobian(th)
    se_f, bse_f, _ = p0.forward_sim.tallies()
    se_a, bse_a, _ = p0.adjoint_sim.tallies()
    assert np.array_equal(se_f, se_a) and np.array_equal(bse_f, bse_a)
    y_default = problem.forward(problem.theta0().numpy())
    assert abs(y.sum() - y_default.sum()) > 0
    W = p0.per_pixel
    N = W.sum()
    k = 4                                       # elastic scale of PMMA: a well-resolved gradient
    delta = 0.01 * float(th[k])
    tp, tm = th.copy(), th.copy()
    tp[k] += delta
    tm[k] -= delta
    fd_pix = (p0.forward(tp) - p0.forward(tm)) * W / (2 * delta)
    adj_pix = J[..., k] * W
    d = (adj_pix - fd_pix).ravel()
    sigma = d.std(ddof=1) * np.sqrt(d.size) / N
    fd, adj = fd_pix.sum() / N, adj_pix.sum() / N
    assert abs(adj - fd) <= 0.05 * abs(fd) + 3 * sigma, (adj, fd, sigma)
    p0.close()


def _resolving_problem(tmp_path_factory, which):
    """A scan on which the parameters of one material carry a gradient that
    a common-random-number difference resolves well within 5 %:
    ``si``: 8.4 x 10^6 primaries at 500 eV on the 1 um Si slab (32 x 32
    pixel groups of one point beam: independent blocks of primaries);
    ``pmma``: 6.1 x 10^6 primaries at 500 eV on the grating's line-top
    pixels (x beyond +-8 nm of the trench centre, 32 of the 64 columns).
    On the whole grating field the Si inelastic gradient is a near
    cancellation of its trench and line-top parts (~0.003), which no scan
    of test size resolves to 5 %."""
    from nebula_b200.synth import workloads, geometry, materials, nmat
    from nebula_b200.torch_adjoint import ScanProblem
    d = tmp_path_factory.mktemp("adj_" + which)
    if which == "si":
        w = workloads.slab(n_primaries=8 << 20, energy=500.0)
        w.primaries["px"] = np.arange(len(w.primaries)) % 32
        w.primaries["py"] = np.arange(len(w.primaries)) // 32 % 32
        tally, n_mat = (32, 32), 1
    else:
        nx = 64
        cols = list(range(0, 16)) + list(range(48, 64))
        w = workloads.grating(nx=nx, ny=nx, per_pixel=3000,
                              pixels=np.array([(x, y) for y in range(nx) for x in cols]))
        tally, n_mat = (nx, nx), 2
    tri = str(d / "g.tri")
    geometry.write_tri(tri, w.triangles)
    ms = []
    for sp in w.material_specs[:n_mat]:
        p = str(d / (sp.name + ".nmat"))
        nmat.write(p, materials.build_raw_material(sp))
        ms.append(nb.Material.load(p))
    g = nb.Geometry.from_tri_file(tri)
    return ScanProblem(g, ms, w.primaries, tally, seed=17, capacity=1 << 21), g, ms


@pytest.mark.parametrize("which,ks", [("si", (0, 1, 2)), ("pmma", (3, 4, 5))])
def test_gradients_match_crn_fd(tmp_path_factory, which, ks):
    """Adjoint gradient of the total SE yield against the central difference
    with common random numbers (5 % of a mean-free-path scale, 0.05 eV of a
    work function), each on a scan where the difference is resolved: the
    test asserts that it is (3 standard errors of adjoint - difference at
    most 5 % of the difference) and then that the two agree within 5 %,
    with no statistical allowance on top -- a 6 % bias in the adjoint
    cannot pass.  The runs are deterministic (counter-based random
    numbers), so the outcome is too."""
    prob, g, ms = _resolving_problem(tmp_path_factory, which)
    th0 = prob.theta0().numpy()
    w = prob.per_pixel
    N = w.sum()
    J = prob.jacobian(th0)
    for k in ks:
        adj_pix = (J[..., k] * w)[w > 0]     # per-pixel contributions to N * dY/dtheta_k
        adj = adj_pix.sum() / N
        delta = 0.05 if k % 3 == 2 else 0.05 * th0[k]
        tp, tm = th0.copy(), th0.copy()
        tp[k] += delta
        tm[k] -= delta
        fd_pix = ((prob.forward(tp) - prob.forward(tm)) * w / (2 * delta))[w > 0]
        fd = fd_pix.sum() / N
        diff = adj_pix - fd_pix
        se = diff.std(ddof=1) * np.sqrt(diff.size) / N
        assert 3 * se <= 0.05 * abs(fd), ("not resolved", k, adj, fd, se)
        assert abs(adj - fd) <= 0.05 * abs(fd), (k, adj, fd, se)
    prob.close()
    g.close()


def test_torch_autograd_matches_jacobian(problem):
    from nebula_b200.torch_adjoint import se_yield
    th = problem.theta0().clone().requires_grad_(True)
    y = se_yield(th, problem)
    wts = torch.from_numpy(problem.per_pixel)
    (y * wts).sum().backward()
    problem.forward(th.detach().numpy())
    J = problem.jacobian(th.detach().numpy())
    expect = (J * problem.per_pixel[..., None]).sum((0, 1))
    assert np.allclose(th.grad.numpy(), expect, rtol=1e-9, atol=1e-9)


def test_gradients_match_reference_driver_fd(tmp_path):
    """The adjoint's total SE-yield gradients against central finite
    differences of the REFERENCE's own CPU driver (tests/golden/
    make_golden_adjoint.py: same scan, 16 x 16 pixels x 4000 primaries, its
    mt19937 reseeded per primary so the +- runs share random numbers).  The
    reference differences carry their own statistical error; the bound is
    5 % of the difference plus 3 combined standard errors."""
    from conftest import load_golden
    from nebula_b200.synth import workloads, geometry, materials, nmat
    from nebula_b200.torch_adjoint import ScanProblem
    ref = load_golden("adjoint_ref_fd.npz")
    nx, per = int(ref["nx"]), int(ref["per_pixel_n"])
    w = workloads.grating(nx=nx, ny=nx, per_pixel=per)
    tri = str(tmp_path / "g.tri")
    geometry.write_tri(tri, w.triangles)
    ms = []
    for sp in w.material_specs:
        pth = str(tmp_path / (sp.name + ".nmat"))
        nmat.write(pth, materials.build_raw_material(sp))
        ms.append(nb.Material.load(pth))
    g = nb.Geometry.from_tri_file(tri)
    prob = ScanProblem(g, ms, w.primaries, (nx, nx), seed=21, capacity=1 << 20)
    th0 = prob.theta0().numpy()
    J = prob.jacobian(th0)
    W = prob.per_pixel
    assert np.array_equal(W, ref["per_pixel"])
    N = W.sum()
    counts, deltas = ref["counts_se"], ref["deltas"]
    for k in range(6):
        adj_pix = J[..., k] * W
        adj = adj_pix.sum() / N
        se_adj = adj_pix.std(ddof=1) * np.sqrt(adj_pix.size) / N
        fd_pix = (counts[k, 1] - counts[k, 0]) / (2 * deltas[k])
        fd = fd_pix.sum() / N
        se_fd = fd_pix.std(ddof=1) * np.sqrt(fd_pix.size) / N
        assert abs(adj - fd) <= 0.05 * abs(fd) + 3 * np.hypot(se_adj, se_fd), (str(ref["params"][k]), adj, fd, se_fd)
    prob.close()


def test_adjoint_replay_with_energy_deposits(problem):
    """Adjoint and energy deposits together (their own kernel
    instantiation): with no work-function step the replay writes exactly the
    forward run's deposit records and detected records."""
    sims = []
    for adj in (False, True):
        s = nb.Simulation(problem.geometry, problem.materials, capacity=1 << 16, seed=21, tally=(16, 16),
                          adjoint=adj, adjoint_w_step=0.0, deposit_capacity=1 << 22)
        s.push(problem.primaries[:20000])
        s.run()
        sims.append(s)
    key = lambda a, n: np.sort(a.view(np.dtype((np.void, n))).ravel()).tobytes()
    dep = [s.drain_deposits() for s in sims]
    det = [s.flush_detected() for s in sims]
    assert len(dep[0]) > 20000
    assert key(dep[0], 28) == key(dep[1], 28)
    assert key(det[0], 36) == key(det[1], 36)
    for s in sims:
        s.close()
