"""The result container against the reference's own post-processing.

``tests/golden/result_groups.npz`` holds the reference's
``get_solution_group`` / ``get_lnA`` / ``get_solution_scale`` outputs on
recorded light-network states, including a state with non-positive bins inside
and at both ends of every species block (``make_golden.py --groups``).
"""

import os

import numpy as np
import pytest

from prince_b200.data import EnergyGrid, SpeciesManager
from prince_b200.results import UHECRPropagationResult, common_energy_grid, grid_triple

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "result_groups.npz")
NAMES = ["plain", "two_src", "mixed", "multi0", "multi1", "multi2", "multi3"]
RTOL = 1e-13


@pytest.fixture(scope="module")
def golden():
    z = dict(np.load(GOLDEN))
    grid = EnergyGrid(*tuple(z["cr_grid"]))
    sm = SpeciesManager([int(p) for p in z["species"]], grid.d)
    return z, grid, sm


def _close(a, b):
    np.testing.assert_allclose(a, b, rtol=RTOL, atol=0)


@pytest.mark.parametrize("name", NAMES)
def test_group_spectra_match_reference(golden, name):
    z, grid, sm = golden
    res = UHECRPropagationResult(z[f"{name}_state"], grid.grid, sm, grid)
    g, f = res.get_solution_group("CR", epow=3)
    np.testing.assert_array_equal(g, z["common_grid"])
    _close(f, z[f"{name}_CR_e3"])
    _close(res.get_solution_group("CR", epow=0)[1], z[f"{name}_CR_e0"])
    _close(res.get_solution_group([1000020030, 1000020040, 1000010030], epow=2)[1], z[f"{name}_heavy_e2"])
    _close(res.get_solution_group("all", epow=3, egrid=z["custom_grid"])[1], z[f"{name}_custom_e3"])
    _close(res.get_solution_scale(1000020040, epow=1)[1], z[f"{name}_He4_scale_e1"])


@pytest.mark.parametrize("name", NAMES)
def test_lnA_matches_reference(golden, name):
    z, grid, sm = golden
    res = UHECRPropagationResult(z[f"{name}_state"], grid.grid, sm, grid)
    _, mean, var = res.get_lnA("CR")
    for mine, ref in ((mean, z[f"{name}_lnA_mean"]), (var, z[f"{name}_lnA_var"])):
        fin = np.isfinite(ref)
        np.testing.assert_array_equal(np.isfinite(mine), fin)
        np.testing.assert_allclose(mine[fin], ref[fin], rtol=1e-11, atol=1e-12)


def test_batched_columns_equal_single_columns(golden):
    z, grid, sm = golden
    X = np.stack([z[f"{n}_state"] for n in NAMES], axis=1)
    res = UHECRPropagationResult(X, grid.grid, sm, grid)
    _, F = res.get_solution_group("CR", epow=3)
    assert F.shape == (z["common_grid"].size, len(NAMES))
    for k, n in enumerate(NAMES):
        np.testing.assert_array_equal(F[:, k], UHECRPropagationResult(X[:, k], grid.grid, sm, grid)
                                      .get_solution_group("CR", epow=3)[1])
        _close(F[:, k], z[f"{n}_CR_e3"])


def test_grid_triple_from_centres_matches_the_grid():
    for tr in ((6, 14, 8), (5, 14, 96 / 9), (-3, 14, 128 / 17)):
        g = EnergyGrid(*tr)
        lo, hi, bpd = grid_triple(g.grid)
        np.testing.assert_allclose((lo, hi, bpd), tr, rtol=1e-9)
        np.testing.assert_array_equal(common_energy_grid(g, 56), common_energy_grid(g.grid, 56))


def test_container_protocol(golden):
    z, grid, sm = golden
    a = UHECRPropagationResult(z["plain_state"], grid.grid, sm, grid)
    b = UHECRPropagationResult(z["two_src_state"], grid.grid, sm, grid)
    np.testing.assert_array_equal((a + b).state, z["plain_state"] + z["two_src_state"])
    np.testing.assert_array_equal((a * 2.5).state, 2.5 * z["plain_state"])
    with pytest.raises(TypeError):
        a * np.ones(3)
    other = UHECRPropagationResult(z["plain_state"], grid.grid * 2, sm, grid)
    with pytest.raises(ValueError):
        a + other
    c = UHECRPropagationResult.from_dict(a.to_dict())
    np.testing.assert_array_equal(c.state, a.state)
    assert c.known_species == a.known_species
    e, n = a.get_solution(2212)
    np.testing.assert_array_equal(n, z["plain_state"][sm.pdgid2sref[2212].sl])
    from scipy.integrate import trapezoid
    A = sm.pdgid2sref[1000020040].A
    expect = trapezoid(A * grid.grid * a.get_solution(1000020040)[1], grid.grid)
    assert a.get_energy_density(1000020040) == pytest.approx(expect, rel=1e-14)


def test_torch_projection_is_differentiable(golden):
    import torch

    z, grid, sm = golden
    X = torch.tensor(np.stack([z["plain_state"], z["mixed_state"]], axis=1), requires_grad=True)
    res = UHECRPropagationResult(X, grid.grid, sm, grid)
    _, F = res.get_solution_group("CR", epow=3)
    _close(F.detach().numpy()[:, 1], z["mixed_CR_e3"])
    F.sum().backward()
    g = X.grad.numpy()
    assert np.all(np.isfinite(g))
    # a bin that is not positive never enters the interpolation
    assert np.all(g[z["mixed_state"] <= 0, 1] == 0)


def test_projection_derivative_stays_finite_across_dynamic_range(golden):
    """Spectra spanning ~600 decades (subnormal tails, values next to zeros):
    the log-log projection and its derivative stay finite."""
    import torch

    z, grid, sm = golden
    x = np.array(z["mixed_state"])
    d = grid.d
    for i in range(len(sm.species_refs)):
        blk = x[i * d:(i + 1) * d]
        blk[-6:] = np.abs(blk[-6:]) * np.array([1e-150, 1e-300, 5e-320, 1e-310, 0.0, 1e-200])
    X = torch.tensor(np.stack([x, z["plain_state"]], axis=1), requires_grad=True)
    _, F = UHECRPropagationResult(X, grid.grid, sm, grid).get_solution_group("CR", epow=3)
    (torch.log(F[F > 0]) ** 2).sum().backward()
    assert torch.isfinite(X.grad).all()
