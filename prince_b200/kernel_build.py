"""The photo-nuclear fold kernel as per-channel response samples.

The fold kernel (``R x dph`` FP64, one row per coupling entry) is a Toeplitz
expansion of a few short arrays per interaction channel
(``src/prince_cr/interaction_rates.py:251-646``).  With the cosmic-ray and
photon grids on one log step, mother bin ``i`` (energy ``E_i``), photon bin
``j`` and daughter bin ``k``:

* boost-conserving channel ``(mo, da)`` and the non-elastic diagonal:
  ``f_i dR_incl[i + j] - f_i dR_nonel[i + j]`` (either term may be absent),
  with ``f_i = m_p / E_i``;
* redistributed channel (daughter energy spread in ``x``):
  ``max(g_ik ddR[i + j, k - i + d - 1], 0)`` with
  ``g_ik = f_i (dE_i / dE_k)``, minus ``f_i dR_nonel[i + j]`` on the diagonal
  ``i = k`` of a channel into the mother itself.  ``ddR`` is either a full
  ``(d + dph - 1) x (2d - 1)`` table or the outer product of two vectors
  (``a[i + j] b[k - i + d - 1]``).

``KernelSpec`` holds those arrays (a few MB) and the ``(channel, row, col)``
of every kernel row; ``materialize`` expands it on the host with the
reference's operation order (the CPU oracle's kernel), and
``pb_build_fold_kernel`` expands it on the GPU straight into device memory in
coupling-CSR order (no host kernel, no 2 GB upload).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

KIND_BC = 0     # f dR_incl - f dR_nonel
KIND_DIFF = 1   # max(g ddR, 0) [- f dR_nonel on the diagonal], ddR a full table
KIND_SEP = 2    # as KIND_DIFF with ddR[a, b] = sep_a[a] * sep_b[b]


@dataclass
class KernelSpec:
    d: int                    # cosmic-ray bins
    dph: int                  # photon bins
    f_mo: np.ndarray          # (d,) m_p / E_i
    dE: np.ndarray            # (d,) bin widths
    resp: np.ndarray          # (n1, d + dph - 1) 1-D increments dR (incl and nonel)
    ddr: np.ndarray           # (n2, d + dph - 1, 2 d - 1) full 2-D increments
    sep_a: np.ndarray         # (n3, d + dph - 1)
    sep_b: np.ndarray         # (n3, 2 d - 1)
    channels: np.ndarray      # (n_ch, 4) int32: kind, incl/ddr/sep index, nonel index, -
    rows: np.ndarray = field(default=None)   # (R,) daughter state index of each kernel row
    cols: np.ndarray = field(default=None)   # (R,) mother state index
    chan: np.ndarray = field(default=None)   # (R,) channel of each kernel row

    @property
    def n_rows(self):
        return int(self.rows.size)

    def materialize(self):
        """``(R, dph)`` FP64 kernel on the host, rows in emission order, with the
        reference's operation order (``interaction_rates.py:490-646``)."""
        d, dph = self.d, self.dph
        out = np.empty((self.n_rows, dph))
        hank = np.arange(d)[:, None] + np.arange(dph)[None, :]          # i + j
        chan = np.asarray(self.chan)
        starts = np.concatenate([[0], np.flatnonzero(np.diff(chan)) + 1, [chan.size]])
        for s0, s1 in zip(starts[:-1], starts[1:]):
            if s1 <= s0:
                continue
            kind, p1, p2, _ = self.channels[chan[s0]]
            i_mo = np.asarray(self.cols[s0:s1]) % d
            i_da = np.asarray(self.rows[s0:s1]) % d
            a = hank[i_mo]
            f = self.f_mo[i_mo][:, None]
            if kind == KIND_BC:
                v = np.zeros((s1 - s0, dph))
                if p1 >= 0:
                    v += f * self.resp[p1][a]
                if p2 >= 0:
                    v -= f * self.resp[p2][a]
            else:
                b = (i_da - i_mo + d - 1)[:, None]
                g = f * (self.dE[i_mo] / self.dE[i_da])[:, None]
                dd = self.ddr[p1][a, b] if kind == KIND_DIFF else self.sep_a[p1][a] * self.sep_b[p1][b]
                v = g * dd
                np.clip(v, 0.0, None, out=v)
                if p2 >= 0:
                    dg = i_mo == i_da
                    v[dg] -= f[dg] * self.resp[p2][a[dg]]
            out[s0:s1] = v
        return out


class SpecBuilder:
    """Collects channels and their kernel rows in emission order."""

    def __init__(self, d, dph, f_mo, dE):
        self.d, self.dph = int(d), int(dph)
        self.f_mo = np.asarray(f_mo, dtype=np.float64)
        self.dE = np.asarray(dE, dtype=np.float64)
        self.resp, self.ddr, self.sep_a, self.sep_b = [], [], [], []
        self.channels, self.rows, self.cols, self.chan = [], [], [], []
        self._resp_index = {}

    def response(self, arr, key=None):
        """Index of a 1-D increment array (shared when ``key`` repeats)."""
        if key is not None and key in self._resp_index:
            return self._resp_index[key]
        self.resp.append(np.asarray(arr, dtype=np.float64))
        i = len(self.resp) - 1
        if key is not None:
            self._resp_index[key] = i
        return i

    def _add(self, kind, p1, p2, rows, cols):
        c = len(self.channels)
        self.channels.append((kind, p1, p2, 0))
        self.rows.append(np.asarray(rows, dtype=np.int64))
        self.cols.append(np.asarray(cols, dtype=np.int64))
        self.chan.append(np.full(len(rows), c, dtype=np.int32))

    def bc(self, incl, nonel, da_lo, mo_lo):
        """Boost-conserving rows ``da_lo + i`` from ``mo_lo + i`` (indices of ``response``, or -1)."""
        i = np.arange(self.d)
        self._add(KIND_BC, incl, nonel, da_lo + i, mo_lo + i)

    def diff(self, kept_mo, kept_da, da_lo, mo_lo, nonel=-1, table=None, sep=None):
        """Redistributed rows at the kept ``(i_mo, i_da)`` pairs; ``table`` (full 2-D) or
        ``sep = (a, b)``."""
        if table is not None:
            self.ddr.append(np.asarray(table, dtype=np.float64))
            kind, p1 = KIND_DIFF, len(self.ddr) - 1
        else:
            self.sep_a.append(np.asarray(sep[0], dtype=np.float64))
            self.sep_b.append(np.asarray(sep[1], dtype=np.float64))
            kind, p1 = KIND_SEP, len(self.sep_a) - 1
        self._add(kind, p1, nonel, da_lo + np.asarray(kept_da), mo_lo + np.asarray(kept_mo))

    def spec(self):
        na, nb = self.d + self.dph - 1, 2 * self.d - 1
        cat = lambda xs, shape, dt: np.stack(xs).astype(dt) if xs else np.zeros(shape, dtype=dt)
        return KernelSpec(
            d=self.d, dph=self.dph, f_mo=self.f_mo, dE=self.dE,
            resp=cat(self.resp, (0, na), np.float64), ddr=cat(self.ddr, (0, na, nb), np.float64),
            sep_a=cat(self.sep_a, (0, na), np.float64), sep_b=cat(self.sep_b, (0, nb), np.float64),
            channels=np.asarray(self.channels, dtype=np.int32).reshape(-1, 4),
            rows=np.concatenate(self.rows) if self.rows else np.zeros(0, np.int64),
            cols=np.concatenate(self.cols) if self.cols else np.zeros(0, np.int64),
            chan=np.concatenate(self.chan) if self.chan else np.zeros(0, np.int32))


def cut_pairs(bins, centres, x_lo):
    """Kept ``(i_mo, i_da)`` of a redistributed channel: ``x_lo <= bins[i_da] / E[i_mo] <= 1``
    (``interaction_rates.py:579-593``), in row-major ``(i_mo, i_da)`` order."""
    xl = bins[:-1][None, :] / centres[:, None]
    keep = (xl >= x_lo) & (xl <= 1)
    i_mo, i_da = np.nonzero(keep)
    return i_mo, i_da
