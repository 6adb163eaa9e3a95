"""Fold-kernel construction on the device (needs a B200).

``pb_build_fold_kernel`` expands per-channel response samples into the
``R x dph`` FP64 kernel in device memory, in coupling-CSR order.  It must
reproduce, bit for bit, the reference's own kernel of the light network
(from the reference's sampled responses, ``kernel_spec_light.npz``) and the
host expansion of the A <= 56 synthetic network (2.7M rows x 96).
"""

import time

import numpy as np
import pytest

from golden_io import light_network
from test_kernel_build import spec_from_golden

pytestmark = pytest.mark.gpu


def _context_with_pattern(n, rows, cols, ph_grid):
    from prince_b200 import _lib
    from prince_b200.operators import coupling_structure
    ctx = _lib.Context(0)
    indptr, indices, order = coupling_structure(rows, cols, n)
    ctx.set_coupling(n, indptr, indices)
    ctx.set_photon_grid(ph_grid)
    return ctx, order


def test_device_build_reproduces_the_reference_kernel():
    z, run, _ = light_network()
    spec = spec_from_golden()
    ctx, order = _context_with_pattern(run.dim_states, spec.rows, spec.cols, run.ph_grid.grid)
    ctx.build_fold_kernel(spec, spec.chan[order])
    K = ctx.fold_kernel(spec.n_rows, spec.dph)
    assert np.array_equal(K, z["batch_matrix"])


def test_device_build_of_the_a56_network_matches_the_host_expansion():
    from workloads import network_run
    run = network_run()
    ir = run.int_rates
    spec = ir.kernel_spec
    ctx, order = _context_with_pattern(run.dim_states, spec.rows, spec.cols, run.ph_grid.grid)
    assert np.array_equal(order, ir.sortidx)
    t0 = time.perf_counter()
    ctx.build_fold_kernel(spec, spec.chan[order])
    dt = time.perf_counter() - t0
    K = ctx.fold_kernel(spec.n_rows, spec.dph)
    assert K.shape == (2665233, 96)
    assert np.array_equal(K, ir._batch_matrix)
    print(f"device kernel build incl. spec upload: {dt * 1e3:.1f} ms")
