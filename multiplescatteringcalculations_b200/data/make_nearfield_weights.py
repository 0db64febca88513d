"""Train the packaged learned near-field preconditioner on the GPU.

    python -m multiplescatteringcalculations_b200.data.make_nearfield_weights [out.npz] [--pairs N]

Default: 16 Gaussian-random-field training slabs of 64 x 64 x 16 cells (correlation length
U[2, 6] cells, relative std U[0.1, 0.3], ka U[0.3, 1], incidence U[0, 40] degrees, P or SV;
seeds 3000..3015), validation on 4 more (seeds 4000..4003), degree 4, the library's
forward/backward kernels and Adam (``train_nearfield``).

``--pairs N``: the streamed form (``train_nearfield_stream``) over N solver residuals from
fresh slabs of the same distribution (seeds 10000, 10001, ...; the residuals after 2, 4, 8,
16, 32 and 64 FP64 GMRES matvecs of each), learning rate 3e-5, with model selection on
validation slabs that converge under the untrained polynomial in 60-2500 matvecs (the
first 6 such seeds from 4000 on).

The result is written to ``nearfield_grf.npz`` next to this script (or the path given),
which ``compute_slab_scattering_gpu(..., preconditioner="learned")`` loads. The packaged file
was made with ``--pairs 20000``: validation operator applications fell from 2910 (the
untrained polynomial) to 2884 after 2004 residuals and then rose steadily to 12568 after
20 000 (the one-step objective drifts away from what a solve needs), so model selection kept
the checkpoint at 2004 residuals.
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


def converging_validation(count: int = 6, start: int = 4000, lo: int = 60, hi: int = 2500, scan: int = 64):
    """The first ``count`` slabs from seed ``start`` whose FGMRES solve with the untrained
    degree-4 polynomial takes between ``lo`` and ``hi`` operator applications."""
    from multiplescatteringcalculations_b200.learned import NearFieldPreconditioner, fgmres_matvecs

    out = []
    net = NearFieldPreconditioner(4)
    for s in range(start, start + scan):
        p = grf_problem(s)
        m = fgmres_matvecs([p], net, max_iter=hi + 1)[0]
        if lo <= m <= hi:
            out.append(p)
            if len(out) == count:
                break
    return out


def main_stream(path: Path, n_pairs: int) -> int:
    from multiplescatteringcalculations_b200.learned import train_nearfield_stream

    t = time.perf_counter()
    val = converging_validation()
    gen = (grf_problem(10000 + i) for i in range(10 ** 6))
    net = train_nearfield_stream(gen, val, n_pairs=n_pairs, verbose=True)
    net.adam = None
    net.save(path)
    print(json.dumps({"path": str(path), "seconds": time.perf_counter() - t, "degree": net.degree,
                      "pairs": net.history[0]["pairs"], "validation": net.history[1]["validation"],
                      "selected_at_pairs": net.history[2]["selected_at_pairs"]}))
    return 0


def main(out: str | None = None, *rest: str) -> int:
    from multiplescatteringcalculations_b200.learned import train_nearfield

    if out == "--pairs":
        out, rest = None, ("--pairs",) + rest
    path = Path(out) if out else Path(__file__).resolve().parent / "nearfield_grf.npz"
    if rest and rest[0] == "--pairs":
        return main_stream(path, int(rest[1]))
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
