"""The CUDA adjoint (jf_grad_*) against the float64 autograd reference.

The reference (oracle/torch_mpm.py) is itself checked against FP64 finite
differences in test_grad_reference.py.  The CUDA path runs in FP32, so its
gradients carry FP32 rounding of a stiff system; the tolerances below are
stated against that.
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
    assert abs(loss - rloss) <= 2e-3 * abs(rloss), (loss, rloss)
    for k in ("actuation", "contraction", "freq"):
        assert abs(g[k] - rg[k]) <= 2e-2 * abs(rg[k]), (k, g[k], rg[k])
    live = mat >= 0
    scale = np.abs(rgx[live]).max()
    err = np.abs(gx[live] - rgx[live])
    assert err.max() <= 5e-2 * scale, (err.max(), scale)
    assert np.median(err) <= 1e-3 * scale
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
        assert a[1][k] == b[1][k], k
    assert np.array_equal(a[2], b[2])


def test_batched_engine_gradients_equal_plain():
    pos, mat, fib, prm = grad_cases.small_tank(seed=5)
    a = _cuda_grads(pos, mat, fib, prm, K=10, path="plain")
    b = _cuda_grads(pos, mat, fib, prm, K=10, path="batched")
    assert a[0] == b[0]
    for k in ("actuation", "contraction", "freq"):
        assert a[1][k] == b[1][k], k
    assert np.array_equal(a[2], b[2])
