"""The torch.autograd front end of the differentiable rollout
(jellyfih_b200/autograd.py), on the CPU with a stand-in engine.

RolloutDisplacement hands the engine's parameter and position gradients back
to torch scaled by the upstream gradient, in the inputs' shapes, and refuses a
backward once the engine has run another rollout (the engine keeps only the
latest rollout's checkpoints, so that backward would differentiate the wrong
rollout).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from jellyfih_b200.autograd import rollout_displacement  # noqa: E402


class StandInEngine:
    """The Engine calls RolloutDisplacement makes, with fixed gradients."""

    def __init__(self, M=2, n=3):
        self.M, self.n = M, n
        self.rollouts = 0
        self.loaded = {}
        self.params = {}
        self.time = None

    def set_params(self, **kw):
        self.params.update(kw)

    def load(self, m, pos, mat, fib):
        self.loaded[m] = np.array(pos)

    def grad_forward(self, steps, checkpoint_every):
        self.rollouts += 1
        return np.arange(1.0, self.M + 1.0)

    def grad_backward(self):
        return {"actuation": np.full(self.M, 2.0), "contraction": np.full(self.M, 3.0),
                "freq": np.full(self.M, 5.0)}

    def grad_positions(self, m):
        return np.full((self.n, 2), float(m + 1), np.float32)


def _inputs(M=2, n=3):
    act = torch.full((M,), 500.0, dtype=torch.float64, requires_grad=True)
    con = torch.full((M,), 0.3, dtype=torch.float64, requires_grad=True)
    frq = torch.full((M,), 1.0, dtype=torch.float64, requires_grad=True)
    pos = torch.rand(M, n, 2, requires_grad=True)
    mats = [np.zeros(n, np.int32)] * M
    fibs = [np.zeros((n, 2), np.float32)] * M
    return act, con, frq, pos, mats, fibs


def test_gradients_are_scaled_by_the_upstream_gradient():
    e = StandInEngine()
    act, con, frq, pos, mats, fibs = _inputs()
    loss = rollout_displacement(e, act, con, frq, pos, mats, fibs, steps=10, checkpoint_every=5)
    assert loss.tolist() == [1.0, 2.0]
    assert np.allclose(e.loaded[1], pos[1].detach().numpy())
    w = torch.tensor([0.5, -2.0], dtype=torch.float64)
    (loss * w).sum().backward()
    assert act.grad.tolist() == [1.0, -4.0]
    assert con.grad.tolist() == [1.5, -6.0]
    assert frq.grad.tolist() == [2.5, -10.0]
    assert pos.grad.shape == pos.shape and pos.grad.dtype == torch.float32
    assert torch.all(pos.grad[0] == 0.5) and torch.all(pos.grad[1] == -4.0)


def test_backward_after_another_rollout_is_refused():
    e = StandInEngine()
    act, con, frq, pos, mats, fibs = _inputs()
    first = rollout_displacement(e, act, con, frq, pos, mats, fibs, steps=10)
    e.grad_forward(10, 100)  # another rollout on the same engine
    with pytest.raises(RuntimeError, match="another differentiable rollout"):
        first.sum().backward()
    second = rollout_displacement(e, act, con, frq, pos, mats, fibs, steps=10)
    second.sum().backward()
    assert act.grad.tolist() == [2.0, 2.0]
