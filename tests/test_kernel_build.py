"""The fold kernel as per-channel response samples (host side).

``tests/golden/kernel_spec_light.npz`` (``make_golden.py --kernel``) holds the
reference's own kernel-construction inputs for the light network: its
sampled response increments per channel and the channel of every kernel
row.  Expanded with the reference's operation order they must give the
reference's ``_batch_matrix`` (``light_network.npz``) bit for bit; the same
expansion runs on the device (``pb_build_fold_kernel``).
"""

import os

import numpy as np
import pytest

from golden_io import GOLDEN, light_network
from prince_b200.kernel_build import KIND_BC, KIND_DIFF, KIND_SEP, KernelSpec, cut_pairs


def spec_from_golden():
    z = dict(np.load(os.path.join(GOLDEN, "kernel_spec_light.npz")))
    return KernelSpec(d=int(z["d"]), dph=int(z["dph"]), f_mo=z["f_mo"], dE=z["dE"], resp=z["resp"],
                      ddr=z["ddr"], sep_a=z["sep_a"], sep_b=z["sep_b"], channels=z["channels"],
                      rows=z["rows"], cols=z["cols"], chan=z["chan"])


def test_reference_spec_expands_to_the_reference_kernel_bit_for_bit():
    spec = spec_from_golden()
    z, _, _ = light_network()
    bm = spec.materialize()
    order = np.lexsort((spec.cols, spec.rows))
    assert np.array_equal(spec.rows[order], z["batch_rows"])
    assert np.array_equal(spec.cols[order], z["batch_cols"])
    assert np.array_equal(bm[order], z["batch_matrix"])
    kinds = set(spec.channels[:, 0].tolist())
    assert KIND_BC in kinds and KIND_DIFF in kinds


def _direct(spec, e):
    """One kernel row from the channel formulas, element by element."""
    d, dph = spec.d, spec.dph
    kind, p1, p2, _ = spec.channels[spec.chan[e]]
    i, k = spec.cols[e] % d, spec.rows[e] % d
    out = np.empty(dph)
    for j in range(dph):
        f = spec.f_mo[i]
        if kind == KIND_BC:
            v = 0.0
            if p1 >= 0:
                v = v + f * spec.resp[p1][i + j]
            if p2 >= 0:
                v = v - f * spec.resp[p2][i + j]
        else:
            g = f * (spec.dE[i] / spec.dE[k])
            dd = (spec.ddr[p1][i + j, k - i + d - 1] if kind == KIND_DIFF
                  else spec.sep_a[p1][i + j] * spec.sep_b[p1][k - i + d - 1])
            v = max(g * dd, 0.0)
            if p2 >= 0 and i == k:
                v = v - f * spec.resp[p2][i + j]
        out[j] = v
    return out


def test_synthetic_spec_rows_follow_the_channel_formulas():
    from workloads import network_run
    run = network_run(max_mass=16, n_species=60, seed=5)
    spec = run.int_rates.kernel_spec
    assert KIND_SEP in set(spec.channels[:, 0].tolist())
    bm = spec.materialize()
    rng = np.random.default_rng(0)
    for e in rng.choice(spec.n_rows, 300, replace=False):
        np.testing.assert_array_equal(bm[e], _direct(spec, e))
    # the run's host kernel is the spec's expansion in CSR order
    np.testing.assert_array_equal(run.int_rates._batch_matrix, bm[run.int_rates.sortidx])


def test_cut_pairs_are_the_reference_x_cuts():
    from prince_b200.data import EnergyGrid
    g = EnergyGrid(5, 14, 96 / 9)
    for cut in (1e-4, 1e-1):
        i_mo, i_da = cut_pairs(g.bins, g.grid, cut)
        xl = g.bins[:-1][None, :] / g.grid[:, None]
        assert np.array_equal(np.argwhere((xl >= cut) & (xl <= 1)), np.stack([i_mo, i_da], 1))
