"""The FP64 build of the differentiable rollout (JF_FLAG_GRAD_FP64) against
the oracle's FP64 build.

The same kernels built for double, every constant the reference's Python
double, P2G summed with double atomics.  On the 32^2 tank of the other
gradient tests: the loss (summed from the FP64 final state) equals the FP64
oracle's displacement to 1e-6 (3e-8 measured), the forward's final positions equal the
oracle's (up to summation order) once both are rounded to FP32, and the
gradients with
respect to the three waveform parameters and to particle positions agree with
FP64 central differences of the oracle.
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


def _oracle64(pos, mat, fib, prm, nx=32):
    from oracle import oracle as O
    s = O.new_state(pos.astype(np.float64), mat, fib, "f64", nx, nx)
    inst = O.Instance(nx=nx, ny=nx, domain_h=1.0, **prm)
    c0 = O.stats_any([s["x"]], [s["material"]])[0, 0]
    O.run(inst, s, np.float64(T0), STEPS)
    return O.stats_any([s["x"]], [s["material"]])[0, 0] - c0, s


def test_fp64_rollout_gradients_match_fp64_differences():
    from jellyfih_b200 import Engine, InstanceSpec
    pos, mat, fib, prm = grad_cases.small_tank()
    e = Engine([InstanceSpec(len(mat), 32, 32, 1.0)], path="plain", grad_fp64=True)
    e.load(0, pos, mat, fib)
    e.set_params(**{k: [v] for k, v in prm.items()})
    e.time = T0
    loss, g = e.grad_step(STEPS, 15)
    gx = e.grad_positions(0)
    final = e.read(0)
    assert not e.error_flags().any()
    e.close()
    ref, s = _oracle64(pos, mat, fib, prm)
    live = mat >= 0
    # the loss is summed from the FP64 final state, not from its FP32 rounding
    # (which resolves the ~5e-6 displacement to ~1e-4): 3e-8 measured, the
    # P2G sums' order amplified by the stiff water over 40 substeps
    assert abs(loss[0] - ref) <= 1e-6 * abs(ref), (loss[0], ref)
    # the final state, rounded to FP32, is the FP64 oracle's
    assert np.abs(final["x"][live].astype(np.float64) - s["x"][live]).max() <= 2 * np.spacing(np.float32(1.0))
    for name, h in (("actuation", 1e-2), ("contraction", 1e-4), ("freq", 1e-4)):
        fd = (_oracle64(pos, mat, fib, dict(prm, **{name: prm[name] + h}))[0] -
              _oracle64(pos, mat, fib, dict(prm, **{name: prm[name] - h}))[0]) / (2 * h)
        assert abs(g[name][0] - fd) <= 1e-5 * abs(fd), (name, g[name][0], fd)
    rng = np.random.default_rng(0)
    pick = np.concatenate([rng.choice(np.flatnonzero(mat == 2), 4, replace=False),
                           rng.choice(np.flatnonzero(live), 8, replace=False)])
    h = 1e-5 / 32
    scale = np.abs(gx[live]).max()
    for k in pick:
        for a in (0, 1):
            up, dn = pos.astype(np.float64).copy(), pos.astype(np.float64).copy()
            up[k, a] += h
            dn[k, a] -= h
            fd = (_oracle64(up, mat, fib, prm)[0] - _oracle64(dn, mat, fib, prm)[0]) / (2 * h)
            # differences of a ~1e-13 loss change resolve ~1e-4 of the max-norm
            assert abs(gx[k, a] - fd) <= 1e-4 * scale, (k, a, gx[k, a], fd)
