"""Host restatement of the CMA-ES fitness (evolve.py:90-124), authoritative
for callers; Engine.fitness computes the same scores on the GPU in FP64."""
from __future__ import annotations

import numpy as np

PENALTY_INVALID = 100.0   # evolve.py:65
MUSCLE_FLOOR = 200        # evolve.py:66
MUSCLE_REFERENCE = 500    # evolve.py:67


def compute_fitness(sim_results, muscle_counts, genomes=None, domain_height=1.0, mode="efficiency"):
    """Scores to minimise, one per instance, from run_batch_headless rows."""
    raw = []
    for i in range(len(sim_results)):
        init_y = sim_results[i, 0]
        final_y = sim_results[i, 2]
        valid = sim_results[i, 4]
        if valid == 0 or muscle_counts[i] < MUSCLE_FLOOR:
            raw.append(None)
            continue
        displacement = min(final_y, domain_height - 0.07) - init_y
        if mode == "displacement":
            raw.append(-displacement)
        else:
            if genomes is not None and len(genomes[i]) > 9:
                active_frac = float(np.clip(genomes[i][9], 0.05, 0.60))
            else:
                active_frac = 0.20
            muscle_cost = (muscle_counts[i] * active_frac / MUSCLE_REFERENCE) ** 0.5
            raw.append(-displacement / muscle_cost)
    valid_scores = [s for s in raw if s is not None]
    penalty = (max(valid_scores) + 1.0) if valid_scores else PENALTY_INVALID
    return [penalty if s is None else s for s in raw]
