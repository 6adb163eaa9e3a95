"""Oracle solves run in spawned worker processes by the GPU tests.

A test process that holds a CUDA context must not fork, so oracle solves that
run beside the GPU solve go to spawned workers; their job functions live here
so that the workers can import them.
"""

PERTURB = 1e-15


def headline_oracle(args):
    """One oracle solve in a spawned process (the caller holds a CUDA context)."""
    kind, cols, zi, seed = args
    import os
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from oracle import etd2_oracle as O
    from workloads import INJECTED, network_run

    run = network_run()
    from prince_b200 import cr_sources

    if kind == "single":
        params = {p: (2.0, 1e10, 0.2) for p in INJECTED}
        srcs = [cr_sources.RigdityCutoffSource(run, norm=1.0, params=params)]
        K = None
    else:
        from workloads import draw_points, point_source

        pts = draw_points(run, 512, seed=1000, z_range=(0.5, 1.0))
        srcs = [[point_source(run, pts[k])] for k in cols]
        K = len(cols)
    perturb = None if seed is None else (PERTURB, seed)
    return O.OracleSolver(run, zi, 0.0, K=K, exp="cr", perturb=perturb).solve(srcs, dz=1e-3)


def coupled_em_oracle(args):
    """One oracle solve of the coupled-EM network (decoupled 128-bin EM grid) in a
    spawned process; ``em_table`` maps each window's redshift to the device-built
    (T_gamma, T_electron, R_BH) the GPU solve used."""
    cols, zi, seed, em_table, size = args
    import os
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from oracle import etd2_oracle as O
    from prince_b200 import synth
    from prince_b200.run import PriNCeRun
    from workloads import A56_GRID, A56_PHOTON, EM_GRID, cib_field, draw_points, point_source

    species = synth.full_network_species(56, n_species=350)
    model = synth.SyntheticPhotoNuclear(species, seed=2, x_cut_proton=1e-4)
    run = PriNCeRun(model, cib_field(), cosmic_ray_grid=A56_GRID, photon_grid=A56_PHOTON,
                    enable_em_cascade=True, enable_em_decoupled_grid=True, em_grid=EM_GRID)
    pts = draw_points(run, 2048, seed=5000, z_range=(0.5, 4.0))
    srcs = [[point_source(run, pts[k])] for k in cols]
    perturb = None if seed is None else (size, seed)

    def em(z):
        return em_table[float(z)]

    return O.OracleSolver(run, zi, 0.0, K=len(cols), exp="cr", perturb=perturb, em=em).solve(srcs, dz=1e-3)
