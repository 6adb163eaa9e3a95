"""Seeded synthetic workloads shared by the tests, the smoke check and the bench."""

from __future__ import annotations

import numpy as np

from prince_b200 import cr_sources, photonfields as pf, synth
from prince_b200.run import PriNCeRun

A56_GRID = (5, 14, 96 / 9)      # 96 bins, log step 0.09375
A56_PHOTON = (-15, -6, 96 / 9)  # 96 photon bins, same step
INJECTED = (2212, 1000020040, 1000070140, 1000140280, 1000260560)  # H, He, N, Si, Fe


def cib_field():
    return pf.CombinedPhotonField([pf.CMBPhotonSpectrum(), pf.ModifiedBlackBodyCIB()])


def network_run(max_mass=56, n_species=350, seed=2):
    """The A <= max_mass network on the 96-bin grid, CMB + synthetic CIB."""
    species = synth.full_network_species(max_mass, n_species=n_species)
    model = synth.SyntheticPhotoNuclear(species, seed=seed, x_cut_proton=1e-4)
    return PriNCeRun(model, cib_field(), cosmic_ray_grid=A56_GRID, photon_grid=A56_PHOTON)


EM_GRID = (-3, 14, 128 / 17)    # 128 bins, 1e-3 to 1e14 GeV


def em_network_run(max_mass=56, n_species=350, seed=2, dz=1e-3):
    """The A <= max_mass network with the co-evolved EM cascade: gamma and e+- on
    the 128-bin EM grid, the cascade transfer and the Bethe-Heitler pair shape
    built on the device from the CMB + synthetic CIB."""
    from prince_b200.em_cascade import KineticCascadeModel

    species = synth.full_network_species(max_mass, n_species=n_species)
    model = synth.SyntheticPhotoNuclear(species, seed=seed, x_cut_proton=1e-4)
    run = PriNCeRun(model, cib_field(), cosmic_ray_grid=A56_GRID, photon_grid=A56_PHOTON,
                    enable_em_cascade=True, enable_em_decoupled_grid=True, em_grid=EM_GRID)
    run.em_cascade_model = KineticCascadeModel(run, dz)
    return run


def light_run(seed=1):
    """p, n, 2H, 3H, 3He, 4He on 1e6-1e14 GeV at 8 bins/decade, CMB only."""
    model = synth.SyntheticPhotoNuclear(synth.light_network_species(), seed=seed)
    return PriNCeRun(model, pf.CMBPhotonSpectrum(), cosmic_ray_grid=(6, 14, 8), photon_grid=(-15, -6, 8))


def draw_points(run, K, seed=7, z_range=(0.5, 1.0), species=INJECTED):
    """K seeded source-parameter points: spectral index U[-1.5, 2.5], log10 Rmax/V
    U[9, 11], composition fractions ~ Dirichlet(1), evolution (1+z)^m with m ~ U[-3, 5],
    z_max ~ U[z_range]."""
    rng = np.random.default_rng(seed)
    present = [p for p in species if p in run.spec_man.pdgid2sref]
    pts = []
    for _ in range(K):
        gamma = rng.uniform(-1.5, 2.5)
        rmax = 10 ** rng.uniform(9.0, 11.0)
        frac = rng.dirichlet(np.ones(len(present)))
        m = rng.uniform(-3.0, 5.0)
        zmax = rng.uniform(*z_range)
        pts.append(dict(gamma=gamma, rmax=rmax, frac=frac, m=m, zmax=zmax, species=present))
    return pts


def point_source(run, pt):
    params = {p: (pt["gamma"], pt["rmax"], float(f)) for p, f in zip(pt["species"], pt["frac"])}
    return cr_sources.RigdityCutoffSource(run, norm=1.0, params=params, m=("simple", pt["m"]),
                                          z_max=pt["zmax"])
