"""B200-native slab Foldy-Lax multiple-scattering solver.

Drop-in for the GPU slab path of tmnestor/MultipleScatteringCalculations
(``cubic_scattering.slab_scattering_gpu.compute_slab_scattering_gpu`` and its
config entry ``run_from_config``), computing in hand-written sm_100a CUDA kernels
behind the C-ABI library ``libmsc_b200.so``.
"""

from .slab import (  # noqa: F401
    BatchProblem,
    BatchSolution,
    MaterialContrast,
    ReferenceMedium,
    SlabGeometry,
    SlabMaterial,
    SlabPlan,
    SlabResult,
    SlabSweepResult,
    clear_plan_cache,
    compute_slab_scattering_batch,
    compute_slab_rpp_sweep,
    compute_slab_scattering_gpu,
    compute_slab_tmatrices,
    gaussian_random_field_material,
    random_slab_material,
    slab_reflected_field,
    slab_rpp_periodic,
    t0_compress,
    t0_expand,
    uniform_random_material,
    uniform_slab_material,
)

from .learned import (  # noqa: F401,E402
    NearFieldPreconditioner,
    fgmres_matvecs,
    solver_residuals,
    train_nearfield,
    train_nearfield_stream,
)
from .sphere import SphereDecompositionResult, compute_sphere_foldy_lax_fft_gpu, sphere_grid  # noqa: F401,E402

__version__ = "0.1.0"
