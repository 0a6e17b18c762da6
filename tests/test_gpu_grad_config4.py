"""Gradients at the differentiable-rollout configuration's shape, against FP64
central differences of the oracle, for the FP32 kernels and their FP64 build.

8 instances on 128^2 with 80,000 slots (~62K live), 2,000 substeps, a
checkpoint every 100.  The CUDA gradient of the payload CoM displacement with
respect to the actuation amplitude, the contraction fraction (the refractory
fraction is 1 - contraction: its gradient is the negative), the frequency
multiplier and 64 seeded particles' initial positions is compared with central
differences of the FP64 build of the oracle, run as one OpenMP batch of all
perturbed copies: the genes at the configuration's step (1e-3, and 1e-3 of
the amplitude) and at 1e-5 (1e-5 of the amplitude), positions at 1e-5 dx.
Instance 7 has contraction 0.06 at frequency 2, so its waveform drop
(t = 0.03, substep 1500) falls inside the horizon.

What was measured (one B200):
* The FP64 build of the kernels is the derivative of the discrete rollout:
  against the 1e-5 differences its gene gradients agree within 2e-7 to 3e-5
  relative (medians 1.1e-5 actuation, 1.5e-5 contraction, 8e-6 frequency),
  its position gradients within 1.9e-5 of the gradient's max-norm (median
  6.5e-7), its loss
  within 2e-7 to 4e-5 of the FP64 oracle's (3e-4 for instance 7).  Two
  exceptions are the differences' own: the contraction of instances 3 and 4
  is not linear even at 1e-5 (the 1e-3 and 1e-5 differences of instance 3
  are -9.2e-3 and -6.8e-3 against the gradient's -5.0e-3), and instance 7's
  drop makes differences at 1e-5 quantized.
* Differences at the configuration's 1e-3 step are not in the linear regime
  for half of these instances: over 2,000 substeps the loss, a function of a
  gene, is rough at that scale (the same FP64 differences at 1e-5 agree with
  the FP64 gradient to 1e-7 where the 1e-3 ones differ in sign), so 1e-3
  differences are compared on the instances where they agree with the 1e-5
  ones.
* The FP32 kernels: their trajectory itself departs from FP64 by percents
  over 2,000 substeps (near-incompressible water amplifies rounding ~1e3 per
  substep; one instance ends 109 % off in displacement), so their gradients
  agree with FP64 differences within 0.3-3 % on the instances whose FP32
  trajectory tracks FP64 and are off by more than 100 % on others; position
  gradients of water particles within 1.9e-2 of the max-norm (median 3e-5),
  of jelly and muscle within 6.4e-3, of payload up to 0.29.
* The waveform drop (instance 7): the 1e-3 differences spread the drop over
  +-25 substeps; the CUDA gradient of the contraction, carried by the drop's
  boundary term, is within 10 % of them in both precisions.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

STEPS, K = 2000, 100
H_GENE = 1e-3
H_FINE = 1e-5


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
    m_pos = 0
    gpu = {}
    for prec in ("fp32", "fp64"):
        e = Engine([InstanceSpec(80000)] * M, path="plain", grad_fp64=(prec == "fp64"))
        for m, (pos, mat, fib, c, f) in enumerate(inputs):
            e.load(m, pos, mat, fib)
        e.set_params(actuation=[act] * M, contraction=[i[3] for i in inputs], freq=[i[4] for i in inputs])
        e.time = 0.0
        loss_p, g_p = e.grad_step(STEPS, K)
        assert not e.error_flags().any()
        gpu[prec] = (loss_p, g_p, e.grad_positions(m_pos))
        e.close()

    base = [dict(actuation=act, contraction=c, freq=f) for _, _, _, c, f in inputs]
    steps_of = {"actuation": (act * H_GENE, act * H_FINE), "contraction": (H_GENE, H_FINE),
                "freq": (H_GENE, H_FINE)}
    variants, tags = [], []
    for m, (pos, mat, fib, c, f) in enumerate(inputs):
        variants.append((pos, mat, fib, base[m]))
        tags.append((m, "base", 0, 0))
        for name, hs in steps_of.items():
            for which, h in enumerate(hs):
                for sgn in (1, -1):
                    variants.append((pos, mat, fib, dict(base[m], **{name: base[m][name] + sgn * h})))
                    tags.append((m, name, which, sgn))
    pos, mat, fib = inputs[m_pos][:3]
    rng = np.random.default_rng(4)
    live = np.flatnonzero(mat >= 0)
    # 64 seeded particles: 8 of each robot material (jelly, payload, muscle), the rest water
    robot = [rng.choice(np.flatnonzero(mat == k), 8, replace=False) for k in (1, 2, 3)]
    pick = np.concatenate(robot + [rng.choice(np.flatnonzero(mat == 0), 64 - 24, replace=False)])
    hx = 1e-5 / 128
    for k in pick:
        for a in (0, 1):
            for sgn in (1, -1):
                p = pos.astype(np.float64).copy()
                p[k, a] += sgn * hx
                variants.append((p, mat, fib, base[m_pos]))
                tags.append((m_pos, ("x", int(k), a), 0, sgn))
    disp = _fp64_displacements(O, variants)
    val = {t: d for t, d in zip(tags, disp)}

    def fd(m, name, which):
        h = steps_of[name][which]
        return (val[(m, name, which, 1)] - val[(m, name, which, -1)]) / (2 * h)

    lines = []
    err = {}  # (precision, name, which) -> per-instance relative errors
    for prec in ("fp32", "fp64"):
        g = gpu[prec][1]
        for name in steps_of:
            for which in (0, 1):
                errs = []
                for m in range(M):
                    d = fd(m, name, which)
                    errs.append(abs(g[name][m] - d) / max(abs(d), 1e-30))
                    lines.append(f"{prec} {name:12s} inst {m} h={steps_of[name][which]:.0e}: CUDA {g[name][m]: .6e}"
                                 f"  FP64 differences {d: .6e}  rel err {errs[-1]:.2e}")
                err[(prec, name, which)] = np.array(errs)
    pos_err = {}
    for prec in ("fp32", "fp64"):
        gx = gpu[prec][2]
        scale = np.abs(gx[live]).max()
        pe = []
        for k in pick:
            for a in (0, 1):
                d = (val[(m_pos, ("x", int(k), a), 0, 1)] - val[(m_pos, ("x", int(k), a), 0, -1)]) / (2 * hx)
                pe.append(abs(gx[k, a] - d) / scale)
                lines.append(f"{prec} x[{k}][{a}] mat {mat[k]}: CUDA {gx[k, a]: .6e}  FP64 differences {d: .6e}  "
                             f"err / max|grad| {pe[-1]:.2e}")
        pos_err[prec] = np.array(pe)
    fp64_loss = np.array([val[(m, "base", 0, 0)] for m in range(M)])
    print("\n" + "\n".join(lines))
    for prec in ("fp32", "fp64"):
        print(f"{prec} loss vs FP64 oracle rel err:", np.array2string(np.abs(gpu[prec][0] - fp64_loss) /
                                                                       np.abs(fp64_loss), precision=2))
        print(f"{prec} median rel err:", {f"{n} h={steps_of[n][w]:.0e}": float(np.median(err[(prec, n, w)]))
                                          for n in steps_of for w in (0, 1)},
              "positions max:", float(pos_err[prec].max()))

    # FP64 build: the derivative of the discrete rollout (fine differences).
    # Instance 7 is left out: the drop quantizes differences this small.  Even
    # at 1e-5 a rollout can sit off the linear regime (the contraction of
    # instances 3 and 4), so the bar is the median and 5 of the 7 instances.
    no_drop = np.arange(7)
    for name in steps_of:
        e64 = err[("fp64", name, 1)][no_drop]
        assert np.median(e64) <= 1e-4, (name, e64)
        assert np.count_nonzero(e64 <= 1e-3) >= 5, (name, e64)
    assert pos_err["fp64"].max() <= 1e-4, pos_err["fp64"]
    # the configuration's step: where it is in the linear regime (agrees with the fine one)
    for name in steps_of:
        lin = [m for m in no_drop if abs(fd(m, name, 0) - fd(m, name, 1)) <= 1e-2 * abs(fd(m, name, 1))]
        assert all(err[("fp64", name, 0)][m] <= 2e-2 for m in lin), (name, lin, err[("fp64", name, 0)])
    # the drop inside the horizon
    assert err[("fp64", "contraction", 0)][7] <= 0.1 and err[("fp32", "contraction", 0)][7] <= 0.1
    # FP32: the bounds it was measured within
    for name in steps_of:
        assert np.all(np.isfinite(err[("fp32", name, 1)]))
        assert np.median(err[("fp32", name, 0)]) <= 0.5, (name, err[("fp32", name, 0)])
    water = [i for i, k in enumerate(np.repeat(pick, 2)) if mat[k] == 0]
    assert np.median(pos_err["fp32"][water]) <= 1e-3, pos_err["fp32"]
    assert pos_err["fp32"][water].max() <= 5e-2, pos_err["fp32"]
