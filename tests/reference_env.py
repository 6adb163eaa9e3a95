"""Import the installed PriNCe reference (plug-in tests, the bench's reference arm).

The reference is installed (``pip install --no-deps --target baseline/_ref``)
beside the repository and travels with it; it is not part of this package.
At import it wants its HDF5 database and ``h5py``; neither is needed for the
ETD2 path, so the package is copied to a scratch directory with an empty
database file and a minimal ``h5py`` stand-in, exactly as
``tests/golden/make_golden.py`` does for the source tree.  The light-nuclei
run is then built with the golden recipe's synthetic cross sections and FP64
settings, so its states are the ones recorded in ``light_network.npz``.
"""

from __future__ import annotations

import importlib.util
import os
import shutil
import sys
import tempfile
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INSTALLED = os.path.join(ROOT, "baseline", "_ref", "prince_cr")


def available():
    return os.path.isdir(INSTALLED)


def _stub_h5py():
    h5 = types.ModuleType("h5py")

    class _File:
        def __init__(self, *a, **k):
            self.attrs = {"version": "stub"}

        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False

        def __contains__(self, k):
            return False

    h5.File = _File
    sys.modules.setdefault("h5py", h5)


def load_package():
    """Import the installed reference (``prince_cr``) from a scratch copy; returns its ``config``."""
    if "prince_cr" not in sys.modules:
        tmp = tempfile.mkdtemp(prefix="prince_ref_")
        shutil.copytree(INSTALLED, os.path.join(tmp, "prince_cr"))
        os.chmod(os.path.join(tmp, "prince_cr", "data"), 0o755)
        open(os.path.join(tmp, "prince_cr", "data", "prince_db_05.h5"), "wb").close()
        _stub_h5py()
        sys.path.insert(0, tmp)
    import prince_cr.config as config

    config.debug_level = 0
    return config


def load_light_run():
    """``(prince_cr package, reference PriNCeRun of the light network)``."""
    load_package()
    import prince_cr
    import prince_cr.config as config

    config.debug_level = 0
    config.cosmic_ray_grid = (6, 14, 8)
    config.photon_grid = (-15, -6, 8)
    config.tau_dec_threshold = 0.0
    config.max_mass = 4
    config.batch_matrix_format = "dense"
    config.xs_dtype = "float64"
    config.linear_algebra_backend = "scipy"
    from prince_cr.cross_sections.base import CrossSectionBase

    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(ROOT, "tests", "golden",
                                                                              "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    run = mg.build(config, CrossSectionBase)
    run.backend.xs_dtype = "float64"
    return prince_cr, run


def load_light_em_run(bins_dec=16):
    """``(prince_cr, reference PriNCeRun)`` of the light network with the
    co-evolved EM cascade on the reference's decoupled EM grid (from the
    electron mass to 1e14 GeV at ``bins_dec`` bins per decade) and the FP64
    cascade iteration; the EM switches are restored on the config afterwards."""
    load_package()
    import prince_cr.config as config

    keys = ("enable_em_cascade", "enable_em_decoupled_grid", "em_grid_bins_dec", "em_cascade_iter_dtype")
    saved = {k: getattr(config, k, None) for k in keys}
    config.enable_em_cascade = True
    config.enable_em_decoupled_grid = True
    config.em_grid_bins_dec = bins_dec
    config.em_cascade_iter_dtype = "float64"
    try:
        return load_light_run()
    finally:
        for k, v in saved.items():
            setattr(config, k, v)
