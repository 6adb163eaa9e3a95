"""CPU restatement of the kinetic EM-cascade transfer -- TEST INFRASTRUCTURE ONLY.

The checker of the device build (``pb_em_transfer``): the per-redshift
cascade transfer ``(T_gamma, T_electron)`` of PriNCe's
``kinetic_cascade_transfer_batched`` (``src/prince_cr/cascade/cascade.py:444-589``)
restated in numpy with an FP64 iteration, pinned to the reference's own
output (``tests/golden/em_cascade_transfer.npz``).  Only ``tests/`` import it.

Steps (reference lines):

* photon stacks on a target grid ``eps`` (IC, pair) and an opacity grid
  ``eps_o``, non-finite / non-positive densities as zero (``cascade.py:474-480``);
* field-free kernels: inverse-Compton emission (``cascade.py:78-104``, the
  Blumenthal-Gould function of ``kernels.py:68-75``), IC energy loss on a
  per-electron sub-grid (``cascade.py:107-138``), gamma-gamma pair injection
  (``cascade.py:141-171``), and the angle-averaged Breit-Wheeler opacity
  (``cascade.py:425-441``, ``opacity.py:44-75``); each with the trapezoid
  weights of its integration grid folded in;
* per-z contractions with the photon stacks; energy-conserving pair matrix;
  IC single-scatter shape, its mean photon energy and the cold-electron mask;
  the continuous-energy-loss shift matrix by cloud-in-cell; the cooled-IC
  matrix from the cumulative trapezoid of emission / loss; the per-step escape
  probability ``exp(-dtau dl)`` (``cascade.py:494-556``);
* the scattering iteration with per-z convergence and the final electron
  transfer (``cascade.py:558-589``).
"""

from __future__ import annotations

import numpy as np

from prince_b200.constants import PRINCE_UNITS as U

# unit constants of the reference's unit table (data.py:722-740, kernels.py:23-25)
M_E = U.m_electron                                        # GeV
SIGMA_T = 8.0 / 3.0 * np.pi * U.r_electron ** 2            # cm^2
C_CM = U.c                                                # cm/s
PREF_IC = 0.75 * SIGMA_T * C_CM


def trapz_weights(x):
    """w with sum(w * y) == trapezoid(y, x)."""
    w = np.empty_like(x)
    w[1:-1] = (x[2:] - x[:-2]) / 2.0
    w[0] = (x[1] - x[0]) / 2.0
    w[-1] = (x[-1] - x[-2]) / 2.0
    return w


def bg_f(q, G):
    """Blumenthal-Gould isotropic inverse-Compton function f(q, Gamma)."""
    return 2.0 * q * np.log(q) + (1.0 + 2.0 * q) * (1.0 - q) + 0.5 * (G * q) ** 2 * (1.0 - q) / (1.0 + G * q)


def ic_kernel(E_out, E_e, eps):
    """A[i, j, k] (photon i from electron j on target k, weights folded) and pref[j]."""
    g = (E_e / M_E)[None, :, None]
    Eo = E_out[:, None, None]
    Ee = E_e[None, :, None]
    ep = eps[None, None, :]
    with np.errstate(all="ignore"):
        G = 4.0 * ep * g / M_E
        q = Eo / (G * (Ee - Eo))
        ok = (q >= 1.0 / (4.0 * g ** 2)) & (q <= 1.0) & (Eo < Ee) & (ep > 0) & (g > 1.0)
        A = np.where(ok, bg_f(q, G) / ep, 0.0) * trapz_weights(eps)[None, None, :]
    pref = np.where(E_e / M_E > 1.0, PREF_IC / (E_e / M_E) ** 2, 0.0)
    return A, pref


def ic_loss_kernel(E_e, eps, n_E1=400):
    """B[j, m, k] on the per-electron sub-grid E1[j, m], and pref[j]."""
    n = E_e.size
    lo = np.log10(eps.min())
    E1 = np.empty((n, n_E1))
    for j in range(n):
        E1[j] = np.logspace(lo, np.log10(0.9999 * E_e[j]), n_E1)
    g = (E_e / M_E)[:, None, None]
    Eo = E1[:, :, None]
    Ee = E_e[:, None, None]
    ep = eps[None, None, :]
    with np.errstate(all="ignore"):
        G = 4.0 * ep * g / M_E
        q = Eo / (G * (Ee - Eo))
        ok = (q >= 1.0 / (4.0 * g ** 2)) & (q <= 1.0) & (Eo < Ee) & (ep > 0) & (g > 1.0)
        B = np.where(ok, bg_f(q, G) / ep, 0.0) * trapz_weights(eps)[None, None, :]
    pref = np.where(E_e / M_E > 1.0, PREF_IC / (E_e / M_E) ** 2, 0.0)
    return B, E1, pref


def pair_kernel(E_e, E0, eps):
    """A[i, j, k] (lepton i from photon j on target k, weights folded) and pref[j]."""
    ge = (E_e / M_E)[:, None, None]
    eg = (E0 / M_E)[None, :, None]
    w = (eps / M_E)[None, None, :]
    denom = ge * (eg - ge)
    valid = (ge > 1.0) & (ge < eg - 1.0) & (denom > 0)
    with np.errstate(all="ignore"):
        wmin = eg / (4.0 * denom)
        r = wmin / w
        F = (4.0 * eg ** 2 / denom * np.log(4.0 * w * denom / eg) - 8.0 * eg * w
             + 2.0 * (2.0 * eg * w - 1.0) * eg ** 2 / denom
             - (1.0 - 1.0 / (eg * w)) * eg ** 4 / denom ** 2)
        ok = valid & (w > wmin) & (r < 1.0)
        A = np.where(ok, F / (w ** 2) / M_E, 0.0) * trapz_weights(eps)[None, None, :]
    return A, PREF_IC / (E0 / M_E) ** 3


def sigma_gg(s):
    """Breit-Wheeler cross section [cm^2] of the squared CM energy s [GeV^2]."""
    s = np.atleast_1d(np.asarray(s, dtype=np.float64))
    out = np.zeros_like(s)
    thr = s > 4.0 * M_E ** 2
    w = 4.0 * M_E ** 2 / s[thr]
    beta = np.sqrt(1.0 - w)
    b2 = 1.0 - w
    out[thr] = 3.0 / 16.0 * SIGMA_T * w * ((3.0 - b2 * b2) * np.log((1.0 + beta) ** 2 / w)
                                           - 2.0 * beta * (2.0 - b2))
    return out


def tau_kernel(E, eps_o, mu):
    """K[i, k]: d tau / dl of photon i on target k (angle-averaged, weights folded)."""
    from scipy.integrate import trapezoid

    omm = 1.0 - mu
    s = 2.0 * E[:, None, None] * eps_o[None, :, None] * omm[None, None, :]
    sig = sigma_gg(s.ravel()).reshape(s.shape)
    ang = 0.5 * trapezoid(omm[None, None, :] * sig, mu, axis=2)
    return ang * trapz_weights(eps_o)[None, :]


def default_grids():
    return np.logspace(-15, -9, 400), np.logspace(-12, -7, 256), np.linspace(-1.0, 1.0, 128)


def hubble(z):
    """cosmology.py:10-21."""
    from prince_b200.cosmology import H
    return H(z)


def transfer(E, zs, field, dz, eps=None, eps_o=None, mu=None, cool_floor_frac=0.1, max_scatter=4000, tol=1e-4):
    """``[(T_gamma, T_electron)]`` per redshift in ``zs`` (FP64 throughout)."""
    d_eps, d_epso, d_mu = default_grids()
    eps = d_eps if eps is None else eps
    eps_o = d_epso if eps_o is None else eps_o
    mu = d_mu if mu is None else mu
    n = E.size
    dE = np.gradient(E)
    Nz = len(zs)

    def stack(grid):
        out = np.empty((grid.size, Nz))
        for i, z in enumerate(zs):
            ne = np.asarray(field.get_photon_density(grid, z), dtype=np.float64)
            out[:, i] = np.where(np.isfinite(ne) & (ne > 0), ne, 0.0)
        return out

    N, No = stack(eps), stack(eps_o)
    A_e, pe = ic_kernel(E, E, eps)
    A_p, pp = pair_kernel(E, E, eps)
    B_l, E1, pl = ic_loss_kernel(E, eps)
    K_tau = tau_kernel(E, eps_o, mu)
    w1 = np.stack([trapz_weights(E1[j]) for j in range(n)])
    epsw = trapz_weights(eps)

    emis = np.einsum("ijk,kz->zij", A_e, N) * pe[None, None, :]
    pair = np.einsum("ijk,kz->zij", A_p, N) * pp[None, None, :]
    dN = np.einsum("jmk,kz->zjm", B_l, N) * pl[None, :, None]
    power_out = np.sum(w1[None] * E1[None] * dN, axis=2)
    rate = np.sum(w1[None] * dN, axis=2)
    eps_mean = (epsw * eps) @ N / (epsw @ N)
    loss = power_out - rate * eps_mean[:, None]
    dtau = np.einsum("ik,kz->zi", K_tau, No)
    dl = np.array([C_CM * abs(dz) / ((1.0 + z) * hubble(z)) for z in zs])

    def trapz_E(M):
        y = E[None, :, None] * M
        return np.sum((y[:, 1:, :] + y[:, :-1, :]) * (E[1:] - E[:-1])[None, :, None] / 2.0, axis=1)

    outE = trapz_E(pair)
    P = np.where(outE[:, None, :] > 0, pair * (E[None, None, :] / np.where(outE > 0, outE, 1.0)[:, None, :]), 0.0)
    R = np.sum(emis * dE[None, :, None], axis=1)
    Sg = np.where(R[:, None, :] > 0, emis / np.where(R > 0, R, 1.0)[:, None, :], 0.0)
    Egam = np.sum(E[None, :, None] * Sg * dE[None, :, None], axis=1)
    cold = (Egam < cool_floor_frac * E[None, :]) | (R <= 0)
    # continuous-loss shift: electron j scatters photon k, keeps E_j - E_k (cloud in cell)
    Eep = E[None, :] - E[:, None]
    valid = Eep > E[0]
    b = np.clip(np.searchsorted(E, Eep.ravel()) - 1, 0, n - 2).reshape(n, n)
    fr = np.clip((E[b + 1] - Eep) / (E[b + 1] - E[b]), 0.0, 1.0)
    vk, vj = np.nonzero(valid)
    bv, fv = b[vk, vj], fr[vk, vj]
    W = Sg[:, vk, vj] * dE[vk][None, :]
    De = np.zeros((Nz, n * n))
    np.add.at(De, (slice(None), bv * n + vj), W * (fv / dE[bv])[None, :])
    np.add.at(De, (slice(None), (bv + 1) * n + vj), W * ((1.0 - fv) / dE[bv + 1])[None, :])
    De = De.reshape(Nz, n, n)
    # cooled inverse-Compton photon matrix
    gg = np.where(loss[:, None, :] > 0, emis / np.where(loss > 0, loss, 1.0)[:, None, :], 0.0)
    dEm = E[1:] - E[:-1]
    incr = (gg[:, :, 1:] + gg[:, :, :-1]) * dEm[None, None, :] / 2.0
    Cum = np.concatenate([np.zeros((Nz, n, 1)), np.cumsum(incr, axis=2)], axis=2)
    diag = Cum[:, np.arange(n), np.arange(n)]
    Mraw = np.where((np.arange(n)[None, :] >= np.arange(n)[:, None])[None], Cum - diag[:, :, None], 0.0)
    outEm = trapz_E(Mraw)
    Mic = np.where(outEm[:, None, :] > 0, Mraw * (E[None, None, :] / np.where(outEm > 0, outEm, 1.0)[:, None, :]),
                   0.0)
    Pe = np.exp(-dtau * dl[:, None])[:, :, None]
    # scattering iteration
    G = np.broadcast_to(np.eye(n), (Nz, n, n)).copy()
    e = np.zeros_like(G)
    escaped = np.zeros_like(G)
    final = np.zeros_like(G)
    E_in = E * dE
    tot0 = np.einsum("i,zij->zj", E_in, G)
    done = np.zeros(Nz, dtype=bool)
    notcold = ~cold
    for _ in range(max_scatter):
        escaped = escaped + Pe * G
        inter = G - Pe * G
        e = e + P @ (inter * dE[None, :, None])
        e_cold = e * cold[:, :, None]
        e_hot = e * notcold[:, :, None]
        G_cold = Mic @ (e_cold * dE[None, :, None])
        G_hot = Sg @ (e_hot * dE[None, :, None])
        e = De @ (e_hot * dE[None, :, None])
        G = G_hot + G_cold
        escaped = escaped + Pe * G_cold
        G = G - Pe * G_cold
        in_box = np.einsum("i,zij->zj", E_in, G) + np.einsum("i,zij->zj", E_in, e)
        conv = np.max(in_box / tot0, axis=1) < tol
        newly = conv & ~done
        if newly.any():
            final = np.where(newly[:, None, None], escaped + Pe * G, final)
            done = done | newly
        if done.all():
            break
    final = np.where(done[:, None, None], final, escaped)
    T_e = final @ (Mic * dE[None, None, :])
    return [(final[i], T_e[i]) for i in range(Nz)]


# ---------------------------------------------------------------------------
# Bethe-Heitler e+- pair shape (bethe_heitler.py:27-172 for the differential
# Born cross section and its nested fourth-order integrations, 180-240 for the
# field-free kernel tensor, 240-297 for the per-redshift shape).
# ---------------------------------------------------------------------------
M_P = U.m_proton


def dsigma_bh(k, g, u):
    """d^2 sigma / (d gamma_e d xi) in (3 / 16 pi) sigma_T alpha units; 0 outside 2.0001 <= k <= 600."""
    REG = 1e-30
    with np.errstate(all="ignore"):
        p = np.sqrt(np.maximum(g * g - 1.0, 0.0) + REG)
        g1 = k - g
        p1 = np.sqrt(np.maximum(g1 * g1 - 1.0, 0.0) + REG)
        D = g - u * p
        T = np.sqrt(np.maximum(k * k + p * p - 2.0 * k * p * u, 0.0))
        d1T = np.log((T + p1) / np.maximum(T - p1, REG))
        y1 = np.log(np.maximum((g1 + p1) / np.maximum(g1 - p1, REG), REG)) / np.maximum(p1, REG)
        Y = 2.0 * np.log(np.maximum((g * g1 + p * p1 + 1.0) / k, REG)) / np.maximum(p * p, REG)
        A0 = p * p1 / (k * k * k)
        A1 = -4.0 * (1.0 - u * u) * (2.0 * g * g + 1.0) / np.maximum(p * p * D ** 4, REG)
        A2 = (5.0 * g * g - 2.0 * g * g1 + 3.0) / np.maximum(p * p * D * D, REG)
        A3 = (p * p - k * k) / np.maximum(T * T * D * D, REG)
        A4 = 2.0 * g1 / np.maximum(p * p * D, REG)
        A50 = Y / np.maximum(p * p1, REG)
        A51 = 2.0 * g * (1.0 - u * u) * (3.0 * k + p * p * g1) / np.maximum(D ** 4, REG)
        A52 = (2.0 * g * g * (g * g + g1 * g1) - 7.0 * g * g - 3.0 * g * g1 - g1 * g1 + 1.0) / np.maximum(D * D, REG)
        A53 = k * (g * g - g * g1 - 1.0) / np.maximum(D, REG)
        A6 = -(d1T / np.maximum(p1 * T, REG)) * (2.0 / np.maximum(D * D, REG) - 3.0 * k / np.maximum(D, REG)
                                                 - k * (p * p - k * k) / np.maximum(T * T * D, REG))
        A7 = -2.0 * y1 / np.maximum(D, REG)
        res = A0 * (A1 + A2 + A3 + A4 + A50 * (A51 + A52 + A53) + A6 + A7)
    return np.where((k >= 2.0001) & (k <= 600.0) & (T >= 1e-30), res, 0.0)


def rk4(fn, lo, hi, n_bins=5):
    """Simpson-weighted fourth-order rule over [lo, hi] in n_bins steps; 0 where hi <= lo."""
    valid = hi > lo
    dx = np.where(valid, (hi - lo) / n_bins, 0.0)
    y = np.zeros_like(lo)
    x = lo.copy()
    for _ in range(n_bins):
        k1 = dx * fn(x)
        k2 = dx * fn(x + 0.5 * dx)
        k4 = dx * fn(x + dx)
        y = y + (k1 + k4) / 6.0 + 2.0 * k2 / 3.0
        x = x + dx
    return np.where(valid, y, 0.0)


def bh_kernel(E_e, E_p, eps):
    """Field-free K[i, j, k]: lepton i from nucleon j on target photon k."""
    ge = (E_e / M_E)[:, None, None]
    gp = (E_p / M_P)[None, :, None]
    ke = (eps / M_E)[None, None, :]
    GE, GP, KE = np.broadcast_arrays(ge, gp, ke)

    def inner(omega, ee):
        REG = 1e-20
        with np.errstate(all="ignore"):
            p_ = np.sqrt(np.maximum(ee * ee - 1.0, 0.0) + REG)
            xi = (GP * ee - GE) / (GP * p_)
            val = omega * dsigma_bh(omega, ee, xi) / p_
        ok = (p_ >= REG) & (xi >= -1.0) & (xi <= 1.0) & (ee >= 1.0) & (ee <= omega - 1.0)
        return np.where(ok, val, 0.0)

    def outer(omega):
        REG = 1e-5
        lo = (GP * GP + GE * GE) / (2.0 * GP * GE) + REG
        hi = omega - 1.0 - REG
        ok = ((hi - lo) >= -1e-4 * lo) & ((hi - lo) / lo >= 1e-4)
        res = rk4(lambda ee: inner(omega, ee), np.where(ok, lo, 1.0), np.where(ok, hi, 0.0))
        return np.where(ok, res, 0.0)

    upper = 2.0 * GP * KE
    lower = (GP + GE) ** 2 / (2.0 * GP * GE)
    ok = (upper - lower) / np.maximum(lower, 1e-30) >= 1e-8
    y = rk4(outer, np.where(ok, lower, 1.0), np.where(ok, upper, 0.0))
    return np.where(ok, y * GE / (2.0 * GP ** 3 * KE ** 2), 0.0)


def bh_shape(E_e, E_p, eps, n_eps, e_p_min=1e5):
    """R[i, j]: one-sign e+- spectrum of a nucleon at E_p[j], energy-normalised so
    the pair carries E_p[j]; the eps integral runs over the points with n > 0."""
    from scipy.integrate import trapezoid

    ln_eps = np.log(eps)
    ok = (n_eps > 0) & (eps > 0)
    R = np.zeros((E_e.size, E_p.size))
    if not ok.any():
        return R
    K = bh_kernel(E_e, E_p, eps)
    col = trapezoid((K * (n_eps * eps)[None, None, :])[:, :, ok], ln_eps[ok], axis=2)
    band = (E_e[:, None] <= E_p[None, :]) & (E_e[:, None] > 1e-6 * E_p[None, :])
    col = np.where(band & (E_p[None, :] >= e_p_min), col, 0.0)
    carried = 2.0 * trapezoid(E_e[:, None] * col, E_e, axis=0)
    good = carried > 0
    R[:, good] = col[:, good] * (E_p[good] / carried[good])[None, :]
    return R
