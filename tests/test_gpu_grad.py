"""The CUDA adjoint (jf_grad_*) against the float64 autograd reference.

The reference (oracle/torch_mpm.py) is itself checked against FP64 finite
differences in test_grad_reference.py.  The CUDA path runs in FP32.  Measured
on a 32^2 tank over 40 substeps: parameter gradients within 1.4e-6 relative,
position gradients with a median error of 3e-9 and a maximum of 1.2e-2 of
their max-norm; over 200 substeps 8.7e-4 relative for the parameters.  The
loss itself (a 5e-6 displacement, ~170 FP32 ulps of a 0.4 position) differs
from FP64 by 3e-3 from position rounding alone.  Re-running the adjoint
accumulates its scatter with float atomics, so two runs agree to ~1e-7, not
bitwise; the forward (fixed-point P2G) is bitwise reproducible.
"""
import numpy as np
import pytest

import grad_cases

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

STEPS = 40
T0 = 0.02


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jellyfih_b200 import build
    build.build()


def _cuda_grads(pos, mat, fib, prm, K, path="plain"):
    from jellyfih_b200 import Engine, InstanceSpec
    e = Engine([InstanceSpec(len(mat), 32, 32, 1.0)], path=path)
    e.load(0, pos, mat, fib)
    e.set_params(**{k: [v] for k, v in prm.items()})
    e.time = T0
    loss = e.grad_forward(STEPS, K)
    final = e.read(0)
    g = e.grad_backward()
    gx = e.grad_positions(0)
    after = e.read(0)
    e.close()
    return loss[0], {k: v[0] for k, v in g.items()}, gx, final, after


def _torch_grads(pos, mat, fib, prm):
    from oracle import torch_mpm as T
    x0 = torch.tensor(pos.astype(np.float64), requires_grad=True)
    p = {k: torch.tensor(v, dtype=torch.float64, requires_grad=True) for k, v in prm.items()}
    loss, _ = T.displacement(x0, torch.zeros_like(x0), torch.tensor(mat).long(),
                             torch.tensor(fib.astype(np.float64)), p, STEPS, 32, 32, 1.0, t0=T0)
    loss.backward()
    return loss.item(), {k: p[k].grad.item() for k in ("actuation", "contraction", "freq")}, x0.grad.numpy()


def test_adjoint_matches_float64_autograd():
    pos, mat, fib, prm = grad_cases.small_tank()
    loss, g, gx, final, after = _cuda_grads(pos, mat, fib, prm, K=15)
    rloss, rg, rgx = _torch_grads(pos, mat, fib, prm)
    assert abs(loss - rloss) <= 1e-2 * abs(rloss), (loss, rloss)
    for k in ("actuation", "contraction", "freq"):
        assert abs(g[k] - rg[k]) <= 2e-5 * abs(rg[k]), (k, g[k], rg[k])
    live = mat >= 0
    scale = np.abs(rgx[live]).max()
    err = np.abs(gx[live] - rgx[live])
    assert err.max() <= 5e-2 * scale, (err.max(), scale)
    assert np.median(err) <= 1e-6 * scale
    # the engine is left at the rollout's final state
    for key in ("x", "v", "C", "F"):
        assert np.array_equal(after[key], final[key]), key


def test_checkpoint_interval_does_not_change_gradients():
    """The forward is deterministic, so recomputed segments reproduce it exactly."""
    pos, mat, fib, prm = grad_cases.small_tank(seed=4)
    a = _cuda_grads(pos, mat, fib, prm, K=STEPS)
    b = _cuda_grads(pos, mat, fib, prm, K=7)
    assert a[0] == b[0]
    for k in ("actuation", "contraction", "freq"):
        assert abs(a[1][k] - b[1][k]) <= 1e-5 * abs(a[1][k]), k
    assert np.abs(a[2] - b[2]).max() <= 1e-5 * np.abs(a[2]).max()


def test_batched_engine_gradients_equal_plain():
    pos, mat, fib, prm = grad_cases.small_tank(seed=5)
    a = _cuda_grads(pos, mat, fib, prm, K=10, path="plain")
    b = _cuda_grads(pos, mat, fib, prm, K=10, path="batched")
    assert a[0] == b[0]
    for k in ("actuation", "contraction", "freq"):
        assert abs(a[1][k] - b[1][k]) <= 1e-5 * abs(a[1][k]), k
    assert np.abs(a[2] - b[2]).max() <= 1e-5 * np.abs(a[2]).max()


def test_autograd_function_and_refinement():
    from jellyfih_b200 import Engine, InstanceSpec, tank
    from jellyfih_b200.autograd import refine_timing_genes, rollout_displacement
    pos, mat, fib, prm = grad_cases.small_tank(seed=6)
    e = Engine([InstanceSpec(len(mat), 32, 32, 1.0)] * 2, path="plain")
    act = torch.tensor([prm["actuation"], 700.0], dtype=torch.float64, requires_grad=True)
    con = torch.tensor([prm["contraction"], 0.4], dtype=torch.float64, requires_grad=True)
    frq = torch.tensor([prm["freq"], 0.9], dtype=torch.float64, requires_grad=True)
    x = torch.tensor(np.stack([pos, pos]), requires_grad=True)
    d = rollout_displacement(e, act, con, frq, x, [mat, mat], [fib, fib], STEPS, 15, T0)
    (2.0 * d[0] - d[1]).backward()
    # the same gradients straight from the engine, weighted like the loss above
    e.set_params(actuation=act.detach().numpy(), contraction=con.detach().numpy(), freq=frq.detach().numpy())
    for m in range(2):
        e.load(m, pos, mat, fib)
    e.time = T0
    e.grad_forward(STEPS, 15)
    g = e.grad_backward()
    for name, t in (("actuation", act), ("contraction", con), ("freq", frq)):
        np.testing.assert_allclose(t.grad.numpy(), [2 * g[name][0], -g[name][1]], rtol=1e-5)
    gx0 = e.grad_positions(0)
    # two runs of the adjoint: its scatter sums with float atomics, whose order
    # noise the stiff water amplifies for a few particles (the median agrees to
    # ~1e-7 of the max-norm, single elements to ~1e-2)
    diff = np.abs(x.grad[0].numpy() - 2 * gx0)
    scale = np.abs(2 * gx0).max()
    assert np.median(diff) <= 1e-6 * scale and diff.max() <= 2e-2 * scale, (np.median(diff), diff.max(), scale)
    genomes = [np.r_[tank.AURELIA_GENOME, 0.3, 1.0]] * 2
    refined, hist = refine_timing_genes(e, genomes, [pos, pos], [mat, mat], [fib, fib], STEPS,
                                        iterations=2, checkpoint_every=20)
    assert len(hist) == 2 and np.all(np.isfinite(hist))
    assert np.all(refined[:, 9] != 0.3) and np.all(refined[:, 10] != 1.0)
    e.close()


@pytest.mark.parametrize("fp64", (False, True))
def test_adjoint_matches_gpu_central_differences(fp64):
    """The CUDA adjoint against central differences of the CUDA forward
    itself, in both builds.  In FP32 the loss (a ~5e-6 displacement) is
    resolved only to ~2e-9, so the differences need large steps (actuation
    +-10, timing genes +-0.01) and then agree to 2-7 % (measured).  In the
    FP64 build two forward runs differ by ~1e-13 in the loss (the order of
    its FP64 atomic sums), which puts a floor of ~1e-4 relative under
    differences at steps of 1e-4; with steps of 5 (1 %) on the actuation,
    whose gradient here is only ~2e-9, and 1e-3 on the timing genes the
    adjoint must agree with its own forward's differences to 1e-3."""
    from jellyfih_b200 import Engine, InstanceSpec
    pos, mat, fib, prm = grad_cases.small_tank()

    def run(p, grads=False):
        e = Engine([InstanceSpec(len(mat), 32, 32, 1.0)], path="plain", grad_fp64=fp64)
        e.load(0, pos, mat, fib)
        e.set_params(**{k: [v] for k, v in p.items()})
        e.time = T0
        loss = e.grad_forward(STEPS, 10)[0]
        g = e.grad_backward() if grads else None
        e.close()
        return loss, g

    _, g = run(prm, True)
    steps = (("actuation", 5.0), ("contraction", 1e-3), ("freq", 1e-3)) if fp64 else \
        (("actuation", 10.0), ("contraction", 1e-2), ("freq", 1e-2))
    tol = 1e-3 if fp64 else 0.1
    for name, h in steps:
        fd = (run(dict(prm, **{name: prm[name] + h}))[0] - run(dict(prm, **{name: prm[name] - h}))[0]) / (2 * h)
        assert abs(g[name][0] - fd) <= tol * abs(fd), (name, g[name][0], fd)


def _oracle_disp_at(pos, mat, fib, prm, t0, steps, nx=32):
    from oracle import oracle as O
    s = O.new_state(pos.astype(np.float64), mat, fib, "f64", nx, nx)
    inst = O.Instance(nx=nx, ny=nx, domain_h=1.0, **prm)
    c0 = O.stats_any([s["x"]], [s["material"]])[0, 0]
    O.run(inst, s, np.float64(t0), steps)
    return O.stats_any([s["x"]], [s["material"]])[0, 0] - c0


def test_waveform_drop_inside_the_rollout_matches_fp64_differences():
    """The waveform drops from 1 to 0 at phase == contraction
    (mpm_sim.py:176-180).  With the drop in the middle of a 200-substep
    rollout (t0 = 0.5 s, freq 1, contraction 0.502: the drop at t = 0.502 s,
    substep 100), FP64 central differences of the C oracle at h = 1e-3 on the
    contraction fraction and the frequency multiplier (the drop moves by 25
    substeps either way) are dominated by the drop: the discrete adjoint alone
    (and the float64 autograd restatement, which has no drop term) is four
    orders of magnitude smaller.  The CUDA gradient, with the drop's boundary
    term, must match the differences within 5 %, and within 2 % their
    Richardson extrapolation from h = 1e-3 and 5e-4 (the h -> 0 limit)."""
    from jellyfih_b200 import Engine, InstanceSpec
    pos, mat, fib, prm = grad_cases.small_tank(seed=7)
    prm = dict(prm, contraction=0.502, freq=1.0)
    t0, steps = 0.5, 200
    e = Engine([InstanceSpec(len(mat), 32, 32, 1.0)], path="plain")
    e.load(0, pos, mat, fib)
    e.set_params(**{k: [v] for k, v in prm.items()})
    e.time = t0
    e.grad_forward(steps, 50)
    g = e.grad_backward()
    assert not e.error_flags().any()
    e.close()

    def fd(name, h):
        hi = _oracle_disp_at(pos, mat, fib, dict(prm, **{name: prm[name] + h}), t0, steps)
        lo = _oracle_disp_at(pos, mat, fib, dict(prm, **{name: prm[name] - h}), t0, steps)
        return (hi - lo) / (2 * h)

    for name in ("contraction", "freq"):
        f1, f2 = fd(name, 1e-3), fd(name, 5e-4)
        limit = f2 + (f2 - f1) / 3.0
        got = g[name][0]
        print(f"\n{name}: CUDA {got:.5e}, FP64 differences h=1e-3 {f1:.5e}, h=5e-4 {f2:.5e}, "
              f"extrapolated {limit:.5e}")
        assert abs(got - f1) <= 0.05 * abs(f1), (name, got, f1)
        assert abs(got - limit) <= 0.02 * abs(limit), (name, got, limit)
    fa = fd("actuation", 1e-2)
    assert abs(g["actuation"][0] - fa) <= 1e-2 * abs(fa), (g["actuation"][0], fa)


def test_gradient_path_reports_nonfinite_states():
    """A particle with a NaN velocity: the deterministic forward's G2P flags its
    instance, grad_forward / grad_backward report JF_ERR_NONFINITE (the Python
    wrapper records it), the other instance stays clean."""
    from jellyfih_b200 import Engine, InstanceSpec
    from jellyfih_b200 import _lib as L
    pos, mat, fib, prm = grad_cases.small_tank(seed=8)
    e = Engine([InstanceSpec(len(mat), 32, 32, 1.0)] * 2, path="plain")
    for m in range(2):
        e.load(m, pos, mat, fib)
    v = np.zeros((len(mat), 2), np.float32)
    v[np.flatnonzero(mat == 0)[0]] = np.nan
    e.write(1, v=v)
    e.time = 0.0
    e.grad_forward(10, 5)
    flags = e.error_flags()
    assert flags[0] == 0 and flags[1] != 0
    assert "non-finite" in e.nonfinite_message
    e.clear_error_flags()
    e.nonfinite_message = ""
    for m in range(2):
        e.load(m, pos, mat, fib)
    e.write(1, v=v)
    loss = np.zeros(2)
    rc = e._lib.jf_grad_forward(e._h, 10, 5, loss.ctypes.data)
    assert rc == L.JF_ERR_NONFINITE
    assert np.isfinite(loss[0])
    e.close()


def test_grad_step_graph_matches_forward_and_backward():
    """jf_grad_step (forward + backward as one CUDA graph, replayed on later
    calls) against jf_grad_forward + jf_grad_backward and against the same
    step with graphs off: the deterministic forward gives the same loss bit
    for bit; the adjoint's float-atomic order moves gradients by ~1e-7."""
    from jellyfih_b200 import Engine, InstanceSpec
    pos, mat, fib, prm = grad_cases.small_tank(seed=9)
    out = {}
    for name, graphs in (("graph", True), ("direct", False)):
        e = Engine([InstanceSpec(len(mat), 32, 32, 1.0)] * 2, path="plain", graphs=graphs)
        e.set_params(**{k: [v, v] for k, v in prm.items()})
        runs = []
        for _ in range(3):  # capture, then two replays
            for m in range(2):
                e.load(m, pos, mat, fib)
            e.time = T0
            loss, g = e.grad_step(STEPS, 15)
            runs.append((loss, g, e.grad_positions(0), e.time))
        if graphs:
            for m in range(2):
                e.load(m, pos, mat, fib)
            e.time = T0
            loss2 = e.grad_forward(STEPS, 15)
            g2 = e.grad_backward()
            runs.append((loss2, g2, e.grad_positions(0), e.time))
        assert not e.error_flags().any()
        e.close()
        out[name] = runs
    ref = out["direct"][0]
    for loss, g, gx, t in out["graph"] + out["direct"][1:]:
        assert np.array_equal(loss, ref[0])
        assert t == ref[3]
        for k in ("actuation", "contraction", "freq"):
            np.testing.assert_allclose(g[k], ref[1][k], rtol=1e-5)
        diff = np.abs(gx - ref[2])
        assert np.median(diff) <= 1e-6 * np.abs(ref[2]).max()


def test_adjoint_queries_follow_the_latest_rollout():
    """jf_grad_backward needs a completed forward and jf_grad_positions the
    backward of the latest rollout: before them, and after a new forward,
    they return JF_ERR_INVALID instead of a stale adjoint."""
    from jellyfih_b200 import Engine, InstanceSpec
    from jellyfih_b200 import _lib as L
    pos, mat, fib, prm = grad_cases.small_tank(seed=6)
    e = Engine([InstanceSpec(len(mat), 32, 32, 1.0)], path="plain")
    e.load(0, pos, mat, fib)
    e.set_params(actuation=[prm["actuation"]], contraction=[prm["contraction"]], freq=[prm["freq"]])
    with pytest.raises(L.JfError, match="completed jf_grad_forward"):
        e.grad_backward()
    e.time = T0
    e.grad_forward(10, 5)
    with pytest.raises(L.JfError, match="latest rollout"):
        e.grad_positions(0)
    e.grad_backward()
    gx = e.grad_positions(0)
    assert gx.shape == (len(mat), 2) and np.all(np.isfinite(gx))
    e.load(0, pos, mat, fib)
    e.time = T0
    e.grad_forward(10, 5)
    with pytest.raises(L.JfError, match="latest rollout"):
        e.grad_positions(0)
    e.load(0, pos, mat, fib)
    e.time = T0
    e.grad_step(10, 5)
    # the same rollout again: equal up to the adjoint's float-atomic order
    assert np.median(np.abs(e.grad_positions(0) - gx)) <= 1e-6 * np.abs(gx).max()
    e.close()
