"""Loading of the golden fixtures produced by tests/golden/make_golden.py."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
STEP_CASES = ("perturbed_1inst", "walls_2inst", "tall_1inst", "axisym_1inst", "axisym_tall_2inst")


def load(case):
    return dict(np.load(os.path.join(GOLDEN, f"{case}.npz")))


def axisym(d):
    """True for fixtures recorded with JELLY_AXISYM=1."""
    return bool(int(d.get("axisym", 0)))


def load_positions(d, m):
    """Positions given to load_particles (they set r_ref); ``in{m}_x`` holds the
    positions the substeps start from, written after the load."""
    return d.get(f"in{m}_x_load", d[f"in{m}_x"])


def n_instances(d):
    return len(d["param_actuation"])


def instance_params(d, m):
    return dict(actuation=float(d["param_actuation"][m]), contraction=float(d["param_contraction"][m]),
                freq=float(d["param_freq"][m]), payload_density=float(d["param_payload_density"][m]))


def dense_grid(d, cp, m):
    nx, ny = int(d["n_grid"]), int(d["n_grid_y"])
    gm = np.zeros(nx * ny, np.float32)
    gv = np.zeros((nx * ny, 2), np.float32)
    idx = d[f"s{cp}_{m}_grid_idx"]
    gm[idx] = d[f"s{cp}_{m}_grid_m"]
    gv[idx] = d[f"s{cp}_{m}_grid_v"]
    return gv.reshape(nx, ny, 2), gm.reshape(nx, ny)
