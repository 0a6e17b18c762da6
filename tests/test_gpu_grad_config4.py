"""Gradients at the differentiable-rollout configuration's shape, against FP64
central differences of the oracle.

8 instances on 128^2 with 80,000 slots (~62K live), 2,000 substeps, a
checkpoint every 100.  The FP32 CUDA gradient of the payload CoM displacement
with respect to the actuation amplitude, the contraction fraction (the
refractory fraction is 1 - contraction: its gradient is the negative), the
frequency multiplier and 8 seeded particles' initial positions is compared
with central differences of the FP64 build of the oracle (h = 1e-3 on the
timing genes, 1e-3 of the amplitude, 1e-5 dx on positions), run as one
OpenMP batch of all perturbed copies.  Instance 7 has contraction 0.06 at
frequency 2, so its waveform drop (t = 0.03, substep 1500) falls inside the
horizon.

Over 2,000 substeps the FP32 trajectory itself departs from FP64 by percents
(near-incompressible water amplifies rounding ~1e3 per substep; one of these
instances ends 109 % off in displacement), so the FP32 gradient cannot hold
1e-3 against FP64 differences here.  Measured (one B200): parameter gradients
within 0.3-3 % on the instances whose FP32 trajectory tracks FP64, off by
more than 100 % (sign included) on two that do not, median relative error
0.19-0.23; instance 7's contraction gradient, carried by the waveform drop,
within 5 %; water particles' position gradients within 4e-3 of the gradient's
max-norm, payload particles' up to 0.47.  The test prints the table and
asserts those bounds with some margin.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

STEPS, K = 2000, 100
H_GENE = 1e-3


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jellyfih_b200 import build
    build.build()
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))


def _inputs():
    from jellyfih_b200 import tank
    out = []
    for g in tank.gaussian_genomes(8, 1000):
        pos, mat, fib, st = tank.fill_tank(g, 80000)
        c, f = tank.timing_params(g)
        out.append([pos, mat, fib, float(c), float(f)])
    out[7][3], out[7][4] = 0.06, 2.0  # the drop at phase 0.06 happens at t = 0.03, inside the horizon
    return out


def _fp64_displacements(O, variants):
    """variants: list of (pos, mat, fib, params dict); FP64 payload CoM displacement of each."""
    states = [O.new_state(p.astype(np.float64), m, f, "f64") for p, m, f, _ in variants]
    insts = [O.Instance(**prm) for _, _, _, prm in variants]
    x0 = O.stats_any([s["x"] for s in states], [s["material"] for s in states])
    O.run_batch(insts, states, np.float64(0.0), STEPS, precision="f64")
    x1 = O.stats_any([s["x"] for s in states], [s["material"] for s in states])
    return x1[:, 0] - x0[:, 0]


def test_config4_gradients_against_fp64_differences():
    from jellyfih_b200 import Engine, InstanceSpec
    from oracle import oracle as O
    inputs = _inputs()
    M = len(inputs)
    act = 500.0
    e = Engine([InstanceSpec(80000)] * M, path="plain")
    for m, (pos, mat, fib, c, f) in enumerate(inputs):
        e.load(m, pos, mat, fib)
    e.set_params(actuation=[act] * M, contraction=[i[3] for i in inputs], freq=[i[4] for i in inputs])
    e.time = 0.0
    loss, g = e.grad_step(STEPS, K)
    assert not e.error_flags().any()
    m_pos = 0
    gx = e.grad_positions(m_pos)
    e.close()

    base = [dict(actuation=act, contraction=c, freq=f) for _, _, _, c, f in inputs]
    variants, tags = [], []
    for m, (pos, mat, fib, c, f) in enumerate(inputs):
        variants.append((pos, mat, fib, base[m]))
        tags.append((m, "base", 0))
        for name, h in (("actuation", act * H_GENE), ("contraction", H_GENE), ("freq", H_GENE)):
            for sgn in (1, -1):
                variants.append((pos, mat, fib, dict(base[m], **{name: base[m][name] + sgn * h})))
                tags.append((m, name, sgn * h))
    pos, mat, fib = inputs[m_pos][:3]
    rng = np.random.default_rng(4)
    live = np.flatnonzero(mat >= 0)
    pick = np.concatenate([rng.choice(np.flatnonzero(mat == 2), 4, replace=False),
                           rng.choice(np.flatnonzero(mat == 0), 4, replace=False)])
    hx = 1e-5 / 128
    for k in pick:
        for a in (0, 1):
            for sgn in (1, -1):
                p = pos.astype(np.float64).copy()
                p[k, a] += sgn * hx
                variants.append((p, mat, fib, base[m_pos]))
                tags.append((m_pos, ("x", int(k), a), sgn * hx))
    disp = _fp64_displacements(O, variants)
    val = {(t[0], t[1], np.sign(t[2])): d for t, d in zip(tags, disp)}

    lines = []
    rel = {}
    for name, h in (("actuation", act * H_GENE), ("contraction", H_GENE), ("freq", H_GENE)):
        errs = []
        for m in range(M):
            fd = (val[(m, name, 1.0)] - val[(m, name, -1.0)]) / (2 * h)
            errs.append(abs(g[name][m] - fd) / max(abs(fd), 1e-30))
            lines.append(f"{name:12s} inst {m}: CUDA FP32 {g[name][m]: .5e}  FP64 differences {fd: .5e}  "
                         f"rel err {errs[-1]:.2e}")
        rel[name] = np.array(errs)
    pos_err = []
    scale = np.abs(gx[live]).max()
    for k in pick:
        for a in (0, 1):
            fd = (val[(m_pos, ("x", int(k), a), 1.0)] - val[(m_pos, ("x", int(k), a), -1.0)]) / (2 * hx)
            pos_err.append(abs(gx[k, a] - fd) / scale)
            lines.append(f"x[{k}][{a}] mat {mat[k]}: CUDA FP32 {gx[k, a]: .5e}  FP64 differences {fd: .5e}  "
                         f"err / max|grad| {pos_err[-1]:.2e}")
    fp64_loss = np.array([val[(m, "base", 0.0)] for m in range(M)])
    loss_err = np.abs(loss - fp64_loss) / np.abs(fp64_loss)
    print("\n" + "\n".join(lines))
    print("loss (displacement) FP32 vs FP64 rel err:", np.array2string(loss_err, precision=2))
    print("median rel err:", {k: float(np.median(v)) for k, v in rel.items()},
          "positions median:", float(np.median(pos_err)))
    for name in rel:
        assert np.all(np.isfinite(rel[name]))
        assert np.median(rel[name]) <= 0.5, (name, rel[name])
    assert rel["contraction"][7] <= 0.1, rel["contraction"][7]  # the drop inside the horizon
    water = [i for i, k in enumerate(np.repeat(pick, 2)) if mat[k] == 0]
    assert max(pos_err[i] for i in water) <= 2e-2, pos_err
    assert np.all(np.isfinite(pos_err))
