"""The reference gradient (float64 PyTorch autograd restatement, standing in for
Taichi autodiff) against central finite differences of the FP64 C oracle."""
import numpy as np
import torch

import grad_cases

STEPS = 40
T0 = 0.02


def _oracle_disp(O, pos, mat, fib, prm, nx):
    s = O.new_state(pos.astype(np.float64), mat, fib, "f64", nx, nx)
    inst = O.Instance(nx=nx, ny=nx, domain_h=1.0, **prm)
    c0 = O.stats_any([s["x"]], [s["material"]])[0, 0]
    O.run(inst, s, np.float64(T0), STEPS)
    return O.stats_any([s["x"]], [s["material"]])[0, 0] - c0


def test_autograd_matches_fp64_finite_differences(oracle):
    from oracle import torch_mpm as T
    pos, mat, fib, prm = grad_cases.small_tank()
    nx = 32
    x0 = torch.tensor(pos.astype(np.float64), requires_grad=True)
    p = {k: torch.tensor(v, dtype=torch.float64, requires_grad=True) for k, v in prm.items()}
    loss, _ = T.displacement(x0, torch.zeros_like(x0), torch.tensor(mat).long(),
                             torch.tensor(fib.astype(np.float64)), p, STEPS, nx, nx, 1.0, t0=T0)
    loss.backward()
    # the restatement's value agrees with the C oracle
    ref = _oracle_disp(oracle, pos, mat, fib, prm, nx)
    assert abs(loss.item() - ref) <= 1e-9 * abs(ref) + 1e-15
    for name, h in (("actuation", 1e-2), ("contraction", 1e-4), ("freq", 1e-4)):
        hi = dict(prm, **{name: prm[name] + h})
        lo = dict(prm, **{name: prm[name] - h})
        fd = (_oracle_disp(oracle, pos, mat, fib, hi, nx) - _oracle_disp(oracle, pos, mat, fib, lo, nx)) / (2 * h)
        ag = p[name].grad.item()
        assert abs(ag - fd) <= 1e-4 * abs(fd) + 1e-12, (name, ag, fd)
    rng = np.random.default_rng(0)
    live = np.flatnonzero(mat >= 0)
    pick = np.concatenate([rng.choice(np.flatnonzero(mat == 2), 4, replace=False),
                           rng.choice(live, 8, replace=False)])
    h = 1e-5 / nx
    g = x0.grad.numpy()
    scale = np.abs(g[live]).max()
    for k in pick:
        for a in (0, 1):
            up, dn = pos.astype(np.float64).copy(), pos.astype(np.float64).copy()
            up[k, a] += h
            dn[k, a] -= h
            fd = (_oracle_disp(oracle, up, mat, fib, prm, nx) - _oracle_disp(oracle, dn, mat, fib, prm, nx)) / (2 * h)
            assert abs(g[k, a] - fd) <= 1e-4 * scale, (k, a, g[k, a], fd)
