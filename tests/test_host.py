"""Host-side logic that needs no GPU: C-ABI symbols, schedule, column ordering."""

import re
import os

import numpy as np
import pytest

from oracle import etd2_oracle as O
from prince_b200 import schedule as S
from prince_b200.cosmology import H, dldz
from prince_b200.constants import PRINCE_UNITS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    text = open(os.path.join(ROOT, "include", "prince_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(pb_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_header_symbol():
    from prince_b200 import build, _lib

    build.build()
    lib = _lib.load()
    syms = _header_symbols()
    assert syms, "no declarations parsed from the header"
    for name in syms:
        assert hasattr(lib, name), name
    assert set(syms) == set(_lib.exported_symbols())
    assert lib.pb_abi_version() == 2


def test_header_constants_match_the_binding():
    """Every PB_* constant of the header has the same value in the ctypes binding."""
    from prince_b200 import _lib
    text = open(os.path.join(ROOT, "include", "prince_b200.h")).read()
    consts = dict(re.findall(r"^#define\s+(PB_[A-Z_0-9]+)\s+(\d+)u?\b", text, flags=re.M))
    assert "PB_OPT_TMA_STAGING" in consts and "PB_INFO_LAST_TMA" in consts
    for name, value in consts.items():
        if name.startswith("PB_NOALLOC"):
            continue
        assert hasattr(_lib, name), name
        assert getattr(_lib, name) == int(value), name


def test_context_without_gpu_raises_cleanly():
    from prince_b200 import _lib

    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(RuntimeError):
        _lib.Context(0)


@pytest.mark.parametrize("zi,zf,dz,thr", [(1.0, 0.0, 1e-3, 0.01), (0.5, 0.0, 2e-3, 1e-3), (0.73, 0.1, 7e-3, 0.02)])
def test_schedule_matches_reference_scalars(zi, zf, dz, thr):
    zg = S.z_grid(zi, zf, dz)
    assert np.array_equal(zg, O.z_grid(zi, zf, dz))
    sch = S.make_schedule(zg, thr)
    assert np.array_equal(sch.z_window, np.asarray(O.window_starts(zg, thr)))
    for k in range(sch.n_steps):
        z = zg[k]
        assert sch.h[k] == zg[k + 1] - z
        assert sch.dldz[k] == O.dldz(z)
        assert sch.hc[k] == H(z) * PRINCE_UNITS.cm2sec
        assert sch.finj[k] == O.dldz(z) * 1.0 * PRINCE_UNITS.cm2sec
        assert sch.z_window[sch.window[k]] <= z + thr + 1e-15


def test_vectorised_evolution_matches_scalar():
    from workloads import light_run, draw_points, point_source

    run = light_run()
    for pt in draw_points(run, 5, seed=4, species=(2212, 1000020040)):
        src = point_source(run, pt)
        zs = S.z_grid(1.0, 0.0, 1e-3)
        vec = src.evolution_array(zs)
        ref = np.array([src.evolution(z) for z in zs])
        # numpy's vectorised pow may differ from the scalar path by an ulp
        np.testing.assert_allclose(vec, ref, rtol=5e-16, atol=0)


def test_batched_coefficients_match_per_source_evolution():
    """The broadcast (1 + z)^m table equals each source's own evolution_array bit for bit."""
    from prince_b200 import cr_sources
    from prince_b200.solvers import _coefficients
    from workloads import light_run
    run = light_run()
    rng = np.random.default_rng(4)
    zs = S.z_grid(0.9, 0.0, 1e-3)[:-1]
    srcs = []
    for k in range(40):
        m = ("simple", float(rng.uniform(-3, 5))) if k % 4 else ("simple", 2.0) if k % 8 == 0 else "flat"
        srcs.append(cr_sources.RigdityCutoffSource(run, norm=float(rng.uniform(0.5, 2.0)),
                                                   params={2212: (2.0, 1e10, 1.0)}, m=m,
                                                   z_max=None if k % 5 == 0 else float(rng.uniform(0.1, 0.9))))
    table = _coefficients(srcs, zs)
    for i, s in enumerate(srcs):
        assert np.array_equal(table[:, i], s.norm * s.evolution_array(zs)), i


def test_column_order_and_active_prefix():
    """Columns are stepped in the order they switch on; the active set is a prefix."""
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    from workloads import light_run, draw_points, point_source

    run = light_run()
    K = 9
    solver = MultiRHSPropagationSolverETD2.__new__(MultiRHSPropagationSolverETD2)
    # exercise _prepare without a device context
    solver.initial_z, solver.final_z, solver.recomp_z_threshold = 1.0, 0.0, 0.01
    solver.enable_injection_jacobian = True
    solver.dim_states = run.dim_states
    from prince_b200.solvers import _MultiRHSView
    solver._K = K
    solver._views = [_MultiRHSView(solver, k) for k in range(K)]
    pts = draw_points(run, K, seed=9, species=(2212, 1000020040))
    for k, p in enumerate(pts):
        solver[k].add_source_class(point_source(run, p))
    sched, K2, coeff, rows, G, src_col, n_active, perm, use_inj = solver._prepare(1e-3)
    assert K2 == K and use_inj
    zmax_sorted = np.array([pts[j]["zmax"] for j in perm])
    assert np.all(np.diff(zmax_sorted) <= 0)
    assert np.all(np.diff(n_active) >= 0) and n_active[-1] == K
    zs = sched.z[:-1]
    for k in range(0, sched.n_steps, 50):
        assert n_active[k] == np.sum(zmax_sorted >= zs[k])
    assert np.all(np.diff(src_col) >= 0)


def test_host_correctly_rounded_exp():
    """oracle.crexp agrees bit for bit with exp evaluated in 60-digit decimal arithmetic."""
    from decimal import Decimal, getcontext
    from oracle import crexp

    getcontext().prec = 60
    rng = np.random.default_rng(5)
    xs = np.concatenate([-np.exp(rng.uniform(np.log(1e-9), np.log(708), 4000)),
                         np.exp(rng.uniform(np.log(1e-9), np.log(709), 1000)), [0.0, 1e-6, -1e-6]])
    exact = np.array([float(Decimal(float(x)).exp()) for x in xs])
    assert np.array_equal(crexp.exp(xs), exact)


def test_device_order_puts_the_shared_grid_blocks_first():
    """Decoupled EM grid: nuclei first on the device, the EM blocks as the tail; the
    permuted CSR keeps every entry and maps back to the run's entry order."""
    import scipy.sparse as sp
    from golden_io import light_network_em_decoupled
    from prince_b200.solvers import device_order, permute_csr

    z, run, em, source = light_network_em_decoupled()
    dev2run, nb = device_order(run)
    sm = run.spec_man
    assert nb == sum(s.uidx() - s.lidx() for s in sm.species_refs if s.grid_tag == "default")
    assert nb % run.cr_grid.d == 0
    assert sorted(dev2run.tolist()) == list(range(run.dim_states))
    g = sm.pdgid2sref[22]
    assert set(dev2run[nb:].tolist()) >= set(range(g.lidx(), g.uidx()))
    cm = run.int_rates.coupling_mat
    M = sp.csr_matrix((np.arange(1, cm.nnz + 1, dtype=float), cm.indices, cm.indptr), shape=cm.shape)
    Md, order = permute_csr(M, dev2run)
    assert Md.has_sorted_indices
    np.testing.assert_array_equal(Md.data, M.data[order])
    np.testing.assert_array_equal(Md.toarray(), M.toarray()[np.ix_(dev2run, dev2run)])
    assert device_order(light_run_shared())[0] is None


def light_run_shared():
    from golden_io import light_network_em
    return light_network_em()[1]


def test_coupled_em_run_layout():
    """The coupled-EM workload: nuclei in 350 blocks of 96 bins, gamma / e+- on the
    128-bin EM grid ahead of them in the run's order and as the device's tail."""
    from prince_b200.solvers import device_order
    from workloads import em_network_run

    run = em_network_run()
    sm = run.spec_man
    assert run.em_grid.d == 128 and np.isclose(run.em_grid.bins[0], 1e-3) and np.isclose(run.em_grid.bins[-1], 1e14)
    assert run.dim_states == 350 * 96 + 3 * 128
    assert [sm.pdgid2sref[p].lidx() for p in (-11, 11, 22)] == [0, 128, 256]
    dev2run, nb = device_order(run)
    assert nb == 350 * 96
    assert np.array_equal(np.sort(dev2run[nb:]), np.arange(384))
    assert np.array_equal(dev2run[:nb], np.arange(384, run.dim_states))
    E = run.adia_loss_rates_grid.energy_vector
    assert np.array_equal(E[256:384], run.em_grid.grid)
    assert np.array_equal(E[384:480], run.cr_grid.grid)
