"""Train the packaged learned near-field preconditioner on the GPU.

    python -m multiplescatteringcalculations_b200.data.make_nearfield_weights [out.npz]

Training slabs: 16 Gaussian-random-field slabs of 64 x 64 x 16 cells (correlation length
U[2, 6] cells, relative std U[0.1, 0.3], ka U[0.3, 1], incidence U[0, 40] degrees, P or SV;
seeds 3000..3015), validation on 4 more (seeds 4000..4003), degree 4, the library's
forward/backward kernels and Adam (``train_nearfield``). The result is written to
``nearfield_grf.npz`` next to this script (or the path given), which
``compute_slab_scattering_gpu(..., preconditioner="learned")`` loads.
"""

from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np


def grf_problem(seed: int, M: int = 64, N_z: int = 16):
    from multiplescatteringcalculations_b200 import (BatchProblem, ReferenceMedium, SlabGeometry,
                                                     gaussian_random_field_material)

    ref = ReferenceMedium(3000.0, 1732.0, 2500.0)
    r = np.random.default_rng(seed)
    ell, std, ka = r.uniform(2, 6), r.uniform(0.1, 0.3), r.uniform(0.3, 1.0)
    g = SlabGeometry(M, N_z, 1.0)
    mat = gaussian_random_field_material(g, ref, correlation_length=ell, std=std, seed=seed)
    th = r.uniform(0, np.deg2rad(40))
    wave = "P" if r.random() < 0.5 else "S"
    return BatchProblem(g, mat, ka * ref.beta, np.array([np.cos(th), np.sin(th), 0.0]), wave)


def main(out: str | None = None) -> int:
    from multiplescatteringcalculations_b200.learned import train_nearfield

    path = Path(out) if out else Path(__file__).resolve().parent / "nearfield_grf.npz"
    t = time.perf_counter()
    net = train_nearfield([grf_problem(3000 + i) for i in range(16)], [grf_problem(4000 + i) for i in range(4)],
                          max_iter=6000)
    net.adam = None
    net.save(path)
    print(json.dumps({"path": str(path), "seconds": time.perf_counter() - t, "degree": net.degree,
                      "adam_steps": len(net.history[0]["losses"]), "validation": net.history[1],
                      "selected": net.history[-1]}))
    return 0


if __name__ == "__main__":
    sys.exit(main(*sys.argv[1:]))
