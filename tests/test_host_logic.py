"""Host-side logic without a GPU: config parsing and validation (the reference's
schema and messages), material generators (bit-exact RNG use), argument checks."""

from pathlib import Path

import numpy as np
import pytest
import yaml
from numpy.testing import assert_array_equal

from multiplescatteringcalculations_b200 import (
    MaterialContrast,
    ReferenceMedium,
    SlabGeometry,
    SlabMaterial,
    gaussian_random_field_material,
    random_slab_material,
    t0_compress,
    t0_expand,
    uniform_random_material,
    uniform_slab_material,
)
from multiplescatteringcalculations_b200.solver_config import build_material, load_config

HERE = Path(__file__).resolve().parent
REF = ReferenceMedium(5000.0, 3000.0, 2500.0)


def test_load_config_reference_schema():
    cfg = load_config(HERE / "configs" / "slab_small.yml")
    assert cfg.problem.type == "slab"
    assert cfg.solver.gmres_tol == 1e-10 and cfg.solver.restart == 30 and cfg.solver.precision == "mixed"
    g = cfg.problem.to_slab_geometry()
    assert (g.M, g.N_z, g.a) == (6, 3, 1.0)
    mat = build_material(cfg)
    ref = random_slab_material(g, REF, MaterialContrast(2e9, 1e9, 100.0), 0.3, 42)
    assert_array_equal(mat.Dlambda, ref.Dlambda)


@pytest.mark.parametrize("patch,match", [
    (lambda d: d.pop("problem"), "missing required 'problem'"),
    (lambda d: d["problem"]["incident"].update(wave_type="X"), "Invalid wave_type"),
    (lambda d: d["problem"]["reference"].update(beta=-1.0), "must be positive"),
    (lambda d: d["solver"].update(initial_guess="guess"), "Invalid initial_guess"),
    (lambda d: d["problem"]["frequency"].pop("omega"), "problem.frequency.omega"),
    (lambda d: d["problem"]["geometry"].pop("N_z"), "problem.geometry.N_z"),
    (lambda d: d["solver"].update(precision="half"), "Invalid precision"),
    (lambda d: d["device"].update(backend="tpu"), "Invalid backend"),
    (lambda d: d["problem"]["slab"].update(material_type="grf"), "correlation_length"),
    (lambda d: d["solver"].update(preconditioner="magic"), "Invalid preconditioner"),
    (lambda d: d["problem"].update(type="sphere"), "requires a 'sphere' section"),
])
def test_validation_messages(tmp_path, patch, match):
    d = yaml.safe_load((HERE / "configs" / "slab_small.yml").read_text())
    patch(d)
    p = tmp_path / "c.yml"
    p.write_text(yaml.safe_dump(d))
    with pytest.raises(ValueError, match=match):
        load_config(p)


def test_missing_config_file(tmp_path):
    with pytest.raises(FileNotFoundError, match="example_slab.yml"):
        load_config(tmp_path / "nope.yml")


def test_random_material_matches_reference_draws(golden):
    """random_slab_material consumes default_rng exactly as the reference does."""
    z = golden("solve_small.npz")
    ref = ReferenceMedium(*[float(v) for v in z["medium"]])
    for name, M, Nz in (("ap_P", 4, 2), ("va_P", 3, 2), ("ap_S", 3, 3)):
        mat = random_slab_material(SlabGeometry(M, Nz, 1.0), ref, MaterialContrast(2e9, 1e9, 100.0), 0.5, seed=5)
        assert_array_equal(mat.Dlambda, z[f"{name}_dlam"])
        assert_array_equal(mat.Drho, z[f"{name}_drho"])


def test_iid_material_matches_headline_fixture(golden):
    z = golden("slab_16x16x4.npz")
    ref = ReferenceMedium(*[float(v) for v in z["medium"]])
    mat = uniform_random_material(SlabGeometry(16, 4, 1.0), ref, 0.10, seed=0)
    assert_array_equal(mat.Dlambda, z["dlam"])
    assert_array_equal(mat.Dmu, z["dmu"])
    assert_array_equal(mat.Drho, z["drho"])


def test_grf_statistics_and_seed():
    g = SlabGeometry(48, 12, 1.0)
    a = gaussian_random_field_material(g, REF, correlation_length=3.0, std=0.15, seed=7)
    b = gaussian_random_field_material(g, REF, correlation_length=3.0, std=0.15, seed=7)
    c = gaussian_random_field_material(g, REF, correlation_length=3.0, std=0.15, seed=8)
    assert_array_equal(a.Dlambda, b.Dlambda)
    assert not np.array_equal(a.Dlambda, c.Dlambda)
    f = a.Dlambda / REF.lam
    assert abs(f.mean()) < 0.02 and 0.13 < f.std() < 0.16
    # neighbouring cells are correlated (exp(-1/9) ~ 0.89 for l = 3), far cells are not
    lag1 = np.corrcoef(f[:, :-1, :].ravel(), f[:, 1:, :].ravel())[0, 1]
    lag12 = np.corrcoef(f[:, :-12, :].ravel(), f[:, 12:, :].ravel())[0, 1]
    assert lag1 > 0.8 and abs(lag12) < 0.1
    strong = gaussian_random_field_material(g, REF, correlation_length=2.0, std=0.8, seed=1)
    assert np.abs(strong.Drho / REF.rho).max() <= 0.9 + 1e-15


def test_t0_expand_compress_roundtrip():
    rng = np.random.default_rng(0)
    t4 = rng.standard_normal((4, 2, 3, 3)) + 1j * rng.standard_normal((4, 2, 3, 3))
    T = t0_expand(t4)
    assert T.shape == (2, 3, 3, 9, 9)
    np.testing.assert_allclose(t0_compress(T), t4, rtol=1e-14, atol=1e-14)
    assert T[0, 0, 0, 3, 4] == t4[1, 0, 0, 0] and T[0, 0, 0, 3, 3] == t4[1, 0, 0, 0] + t4[2, 0, 0, 0]


def test_dataclass_validation():
    with pytest.raises(ValueError, match="M must be"):
        SlabGeometry(0, 1, 1.0)
    with pytest.raises(ValueError, match="a must be"):
        SlabGeometry(2, 1, 0.0)
    with pytest.raises(ValueError, match="shapes must match"):
        SlabMaterial(np.zeros((1, 2, 2)), np.zeros((1, 2, 3)), np.zeros((1, 2, 2)), REF)
    with pytest.raises(ValueError, match="3D"):
        SlabMaterial(np.zeros((2, 2)), np.zeros((2, 2)), np.zeros((2, 2)), REF)
    mat = uniform_slab_material(SlabGeometry(2, 3, 1.0), REF, MaterialContrast(1.0, 2.0, 3.0))
    assert mat.Dmu.shape == (3, 2, 2) and np.all(mat.Dmu == 2.0)


def test_result_arrays_are_recycled_only_when_unreferenced():
    from multiplescatteringcalculations_b200 import slab as S

    a = S._host_array((3, 7))[0]
    ida = id(a)
    b = S._host_array((3, 7))[0]
    assert a is not b
    del a
    c = S._host_array((3, 7))[0]
    assert id(c) == ida  # dropped by the caller: filled again
    v = c[1:]
    del c
    d = S._host_array((3, 7))[0]
    assert d is not v.base  # a view keeps it alive


def test_nearfield_network_parameters_roundtrip(tmp_path):
    """The learned network's parameters survive save/load; its complex64 layers default to
    the tensor cores ("bf16_tc"), and a saved weight form is kept as saved."""
    from multiplescatteringcalculations_b200 import NearFieldPreconditioner

    net = NearFieldPreconditioner(3)
    assert net.weights == "bf16_tc"
    assert_array_equal(net.coef, np.ones(4))
    assert net.w.shape == (3, 27, 9, 9) and not net.w.any()
    rng = np.random.default_rng(0)
    net.coef = rng.standard_normal(4) + 1j * rng.standard_normal(4)
    net.w = rng.standard_normal((3, 27, 9, 9)) + 1j * rng.standard_normal((3, 27, 9, 9))
    net.weights = "bf16"
    net.save(tmp_path / "net.npz")
    back = NearFieldPreconditioner.load(tmp_path / "net.npz")
    assert back.degree == 3 and back.weights == "bf16" and back.adam is None
    assert_array_equal(back.coef, net.coef)
    assert_array_equal(back.w, net.w)
    with pytest.raises(ValueError):
        NearFieldPreconditioner(7)
    with pytest.raises(ValueError):
        NearFieldPreconditioner(2, coef=np.ones(5))


def test_packaged_network_runs_on_tensor_cores():
    """The packaged network (data/nearfield_grf.npz, trained in the BF16 form) is installed
    with its layers on the tensor cores."""
    from multiplescatteringcalculations_b200.slab import _packaged_network

    net = _packaged_network()
    assert net.weights == "bf16_tc"
    assert net.degree == 4 and net.w.shape == (4, 27, 9, 9)


def test_sphere_incident_columns_batched_equal_per_column():
    """The 9 incident patterns of the sphere built at once equal the per-column form
    (resonance_tmatrix.py:526-586 restated), bit for bit (CPU tensors)."""
    import torch

    from multiplescatteringcalculations_b200 import sphere as S

    n = 6
    mask, _, centres, a_sub = S.sphere_grid(0.5, n)
    c1 = (-n / 2 + 0.5 + np.arange(n)) * (2 * a_sub)
    pos = torch.stack(torch.meshgrid(*(torch.tensor(c1),) * 3, indexing="ij"), -1)
    phase = torch.exp(1j * 5.0 * (pos @ torch.tensor([0.3, 0.4, np.sqrt(0.75)])))
    xm = torch.tensor(centres.mean(axis=0))
    mt = torch.from_numpy(mask)
    a = torch.stack([S._incident_column(c, pos, mt, phase, xm) for c in range(9)])
    assert torch.equal(a, S._incident_columns(pos, mt, phase, xm))
