"""The CPU oracle against fixtures recorded from the reference's own mpm_sim.py.

The fixtures were produced by executing mpm_sim.py:153-340 (substep) and
:740-834 (stats, run_batch_headless) under the Taichi stand-in; the FP32 oracle
follows the same operation order, so the comparison is bit-exact.
"""
import numpy as np
import pytest

import golden_io as G

FIELDS = ("x", "v", "C", "F", "Jp", "glow")


def _oracle_state(O, d, m):
    s = O.new_state(G.load_positions(d, m), d[f"in{m}_material"], d[f"in{m}_fiber"], "f32",
                    int(d["n_grid"]), int(d["n_grid_y"]))
    for k in ("x", "v", "C", "F", "Jp", "glow"):
        s[k][...] = d[f"in{m}_{k}"]
    return s


def _inst(O, d, m):
    return O.Instance(nx=int(d["n_grid"]), ny=int(d["n_grid_y"]), domain_h=float(d["domain_height"]),
                      dt=float(d["dt"]), axisym=G.axisym(d), **G.instance_params(d, m))


@pytest.mark.parametrize("case", G.STEP_CASES)
def test_substep_bit_exact(oracle, case):
    d = G.load(case)
    for m in range(G.n_instances(d)):
        s = _oracle_state(oracle, d, m)
        inst = _inst(oracle, d, m)
        t = np.float32(d["t0"])
        done = 0
        for cp in d["checkpoints"]:
            t = oracle.run(inst, s, t, int(cp) - done)
            done = int(cp)
            assert t == d[f"time_{cp}"]
            for k in FIELDS:
                ref = d[f"s{cp}_{m}_{k}"]
                assert np.array_equal(s[k].view(np.uint32), ref.view(np.uint32)), (case, m, cp, k)
            gv, gm = G.dense_grid(d, cp, m)
            assert int(d[f"s{cp}_{m}_grid_v_nonzero_outside"]) == 0
            assert np.array_equal(s["grid_m"], gm), (case, m, cp, "grid_m")
            assert np.array_equal(s["grid_v"], gv), (case, m, cp, "grid_v")


# The reference sums CoM coordinates with FP32 atomics (mpm_sim.py:751-753);
# the oracle (like the GPU engine) sums in FP64.  The FP32 running sum of n
# values carries a relative error up to about n * 2**-24 (n <= ~2000 here).
STATS_RTOL = 2000 * 2.0 ** -24


def test_headless_and_stats(oracle):
    d = G.load("headless_3inst")
    M = G.n_instances(d)
    states = [_oracle_state(oracle, d, m) for m in range(M)]
    xs = [s["x"] for s in states]
    mats = [s["material"] for s in states]
    np.testing.assert_allclose(oracle.payload_stats(xs, mats), d["payload_stats_before"], rtol=STATS_RTOL)
    before = oracle.stats_any(xs, mats)
    np.testing.assert_allclose(before, d["stats_any_before"], rtol=STATS_RTOL)
    steps = int(d["checkpoints"][-1])
    for m in range(M):
        t = oracle.run(_inst(oracle, d, m), states[m], np.float32(0.0), steps)
    assert t == d["time_after"]
    for m in range(M):
        assert np.array_equal(states[m]["x"], d[f"s{steps}_{m}_x"])
    after = oracle.stats_any(xs, mats)
    rows = oracle.headless_rows(before, after)
    np.testing.assert_allclose(rows, d["headless"], rtol=STATS_RTOL, atol=0)
    assert rows[2, 4] == 0.0 and rows[0, 4] == 1.0 and rows[1, 2] > 0  # floor-invalid, body fallback
    np.testing.assert_allclose(oracle.payload_stats(xs, mats), d["payload_stats_after"], rtol=STATS_RTOL)


def test_fp64_build_close_to_fp32(oracle):
    """The FP64 build of the same algorithm stays close to FP32 over 5 steps."""
    d = G.load("perturbed_1inst")
    s32 = _oracle_state(oracle, d, 0)
    s64 = oracle.cast_state(s32, "f64")
    inst = _inst(oracle, d, 0)
    oracle.run(inst, s32, np.float32(d["t0"]), 5)
    oracle.run(inst, s64, np.float64(d["t0"]), 5)
    live = s32["material"] >= 0
    for k in ("x", "v", "F"):
        a, b = s32[k][live], s64[k][live]
        scale = np.abs(b).max()
        assert np.abs(a - b).max() <= 1e-4 * scale, k


def test_svd_invariants(oracle):
    rng = np.random.default_rng(7)
    for _ in range(200):
        A = rng.normal(size=(2, 2))
        U, sig, V = oracle.svd2(A.astype(np.float64))
        np.testing.assert_allclose(U @ np.diag(sig) @ V.T, A, atol=1e-12)
        np.testing.assert_allclose(U @ U.T, np.eye(2), atol=1e-12)
        np.testing.assert_allclose(V @ V.T, np.eye(2), atol=1e-12)
        assert sig[0] >= sig[1]
        # R = U V^T is the polar rotation (det +1), as in the reference's stress
        assert np.linalg.det(U @ V.T) == pytest.approx(1.0)


def test_waveform(oracle):
    inst = oracle.Instance(contraction=0.2, freq=1.0)
    assert oracle.activation(inst, np.float32(0.1)) == pytest.approx(0.5, abs=1e-6)
    assert oracle.activation(inst, np.float32(0.25)) == 0.0
    # the arch drops from ~1 to 0 at phase == contraction (mpm_sim.py:179-180)
    assert oracle.activation(inst, np.float32(0.1999)) > 0.99
    inst2 = oracle.Instance(contraction=0.3, freq=2.0)
    assert oracle.activation(inst2, np.float32(0.55)) == pytest.approx(
        oracle.activation(inst2, np.float32(0.05)), abs=1e-5)


def _rel_err(a, b):
    scale = np.abs(b).max()
    return np.abs(a.astype(np.float64) - b).max() / max(scale, 1e-30)


@pytest.mark.parametrize("case", ["perturbed_1inst", "walls_2inst", "tall_1inst"])
def test_fixed_point_p2g_matches_the_reference_per_substep(oracle, case):
    """The order-free P2G option (2^-44 fixed-point sums, the GPU deterministic
    forward's accumulation) changes one substep by rounding only: within 1e-5
    of each field's max-norm of the fixtures recorded from the reference."""
    d = G.load(case)
    cp = int(d["checkpoints"][0])
    for m in range(G.n_instances(d)):
        s = _oracle_state(oracle, d, m)
        inst = _inst(oracle, d, m)
        inst.fixed_p2g = True
        oracle.run(inst, s, np.float32(d["t0"]), cp)
        live = s["material"] >= 0
        for k in ("v", "C", "F"):
            assert _rel_err(s[k][live], d[f"s{cp}_{m}_{k}"][live]) <= 1e-5, (case, m, k)
        assert np.abs(s["x"][live].astype(np.float64) - d[f"s{cp}_{m}_x"][live]).max() <= 4e-7


def test_fixed_point_p2g_is_order_free(oracle):
    """With fixed-point sums the substep does not depend on the particles'
    order: a permuted copy of the state gives bit-identical fields after 20
    substeps (with FP32 sums it does not)."""
    d = G.load("walls_2inst")
    s = _oracle_state(oracle, d, 0)
    n = len(s["material"])
    perm = np.random.default_rng(11).permutation(n)
    sp = {k: (np.ascontiguousarray(a[perm]) if k not in ("grid_v", "grid_m") else a.copy()) for k, a in s.items()}
    inst = _inst(oracle, d, 0)
    inst.fixed_p2g = True
    oracle.run(inst, s, np.float32(d["t0"]), 20)
    oracle.run(inst, sp, np.float32(d["t0"]), 20)
    for k in ("x", "v", "C", "F", "Jp"):
        assert np.array_equal(s[k][perm].view(np.uint32), sp[k].view(np.uint32)), k
    # the same permutation with FP32 sums changes the fields
    s2 = _oracle_state(oracle, d, 0)
    sp2 = {k: (np.ascontiguousarray(a[perm]) if k not in ("grid_v", "grid_m") else a.copy()) for k, a in s2.items()}
    inst.fixed_p2g = False
    oracle.run(inst, s2, np.float32(d["t0"]), 20)
    oracle.run(inst, sp2, np.float32(d["t0"]), 20)
    assert not np.array_equal(s2["v"][perm], sp2["v"])
