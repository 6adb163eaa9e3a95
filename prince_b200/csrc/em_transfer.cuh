// Kinetic EM-cascade transfer built on the device (included by prince_b200.cu).
//
// The per-redshift cascade transfer (T_gamma, T_electron) of an EM grid E
// (n bins) on the context's photon field, as PriNCe's
// kinetic_cascade_transfer_batched (src/prince_cr/cascade/cascade.py:444-589)
// computes it, in FP64 throughout:
//   1. photon densities on a target grid eps (IC, pair) and an opacity grid
//      eps_o for every redshift (non-finite / non-positive as zero);
//   2. field-free kernels with the trapezoid weights of their integration grid
//      folded in: IC emission A_e[i][j][k], IC loss B_l[j][m][k] on the
//      per-electron sub-grid E1[j][m], pair injection A_p[i][j][k]
//      (cascade.py:78-171, the Blumenthal-Gould function kernels.py:68-75),
//      Breit-Wheeler opacity K[i][k] averaged over mu (cascade.py:425-441,
//      opacity.py:44-75);
//   3. the contractions with the photon stacks as FP64 tensor-core GEMMs (DMMA);
//   4. per redshift: the energy-conserving pair matrix, the IC single-scatter
//      shape and its cold mask, the loss-shift matrix (cloud in cell), the
//      cooled-IC matrix from a cumulative trapezoid, the escape probability;
//   5. the scattering iteration, four batched n x n GEMMs per pass, with the
//      per-redshift convergence test on the device, and the electron transfer.

namespace {

// ---------------------------------------------------------------------------
// Batched FP64 GEMM on the tensor pipe: C[b] (=|+=) A[b] B[b], row-major,
// DMMA m8n8k4.  CTA tile (16 WM) x 32 (2 WM warps of 16 x 16 each; WM = 4 for
// large grids, 2 when 64-row tiles would leave most SMs idle), k in chunks of
// 16 through shared memory (zero-padded at the edges).
// ---------------------------------------------------------------------------
struct BGemm {
  const double* A;
  const double* B;
  double* C;
  int M, N, K, lda, ldb, ldc;
  long long sA, sB, sC;
  int accumulate;
};

constexpr int kGn = 32, kGk = 16;

template <int WM>
__global__ void __launch_bounds__(WM * 64) k_bgemm(BGemm g) {
  constexpr int kGm = 16 * WM;
  __shared__ double As[kGm][kGk + 1];
  __shared__ double Bs[kGk][kGn + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wm = wid % WM, wn = wid / WM;
  const int m0 = blockIdx.y * kGm, n0 = blockIdx.x * kGn;
  const double* __restrict__ A = g.A + (size_t)blockIdx.z * g.sA;
  const double* __restrict__ B = g.B + (size_t)blockIdx.z * g.sB;
  double* __restrict__ C = g.C + (size_t)blockIdx.z * g.sC;
  double acc[2][2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  for (int k0 = 0; k0 < g.K; k0 += kGk) {
    for (int t = threadIdx.x; t < kGm * kGk; t += blockDim.x) {
      const int r = t / kGk, c = t - r * kGk;
      As[r][c] = (m0 + r < g.M && k0 + c < g.K) ? A[(size_t)(m0 + r) * g.lda + k0 + c] : 0.0;
    }
    for (int t = threadIdx.x; t < kGk * kGn; t += blockDim.x) {
      const int r = t / kGn, c = t - r * kGn;
      Bs[r][c] = (k0 + r < g.K && n0 + c < g.N) ? B[(size_t)(k0 + r) * g.ldb + n0 + c] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGk / 4; ++kk) {
      double af[2], bf[2];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) af[mi] = As[wm * 16 + mi * 8 + (lane >> 2)][kk * 4 + (lane & 3)];
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) bf[ni] = Bs[kk * 4 + (lane & 3)][wn * 16 + ni * 8 + (lane >> 2)];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) dmma884(acc[mi][ni][0], acc[mi][ni][1], af[mi], bf[ni]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni) {
      const int row = m0 + wm * 16 + mi * 8 + (lane >> 2);
      if (row >= g.M) continue;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int col = n0 + wn * 16 + ni * 8 + (lane & 3) * 2 + h;
        if (col >= g.N) continue;
        double* out = C + (size_t)row * g.ldc + col;
        *out = g.accumulate ? __dadd_rn(*out, acc[mi][ni][h]) : acc[mi][ni][h];
      }
    }
}

void bgemm(cudaStream_t st, const double* A, const double* B, double* C, int M, int N, int K, int lda, int ldb,
           int ldc, long long sA, long long sB, long long sC, int batch, bool accumulate) {
  BGemm g{A, B, C, M, N, K, lda, ldb, ldc, sA, sB, sC, accumulate ? 1 : 0};
  const long long ctas64 = (long long)((N + kGn - 1) / kGn) * ((M + 63) / 64) * batch;
  if (ctas64 < 256)
    k_bgemm<2><<<dim3((N + kGn - 1) / kGn, (M + 31) / 32, batch), 128, 0, st>>>(g);
  else
    k_bgemm<4><<<dim3((N + kGn - 1) / kGn, (M + 63) / 64, batch), 256, 0, st>>>(g);
}

// ---------------------------------------------------------------------------
// Field-free kernels and photon stacks
// ---------------------------------------------------------------------------
struct EmConst {
  double me;       // electron mass [GeV]
  double pref_ic;  // 3/4 sigma_T c
  double sigma_t;
};

// Blumenthal-Gould isotropic inverse-Compton function (kernels.py:68-75).
__device__ __forceinline__ double bg_f(double q, double G) {
  const double gq = G * q;
  return 2.0 * q * log(q) + (1.0 + 2.0 * q) * (1.0 - q) + 0.5 * gq * gq * (1.0 - q) / (1.0 + gq);
}

// IC emission of a photon Eo from an electron Ee on target e (weight w folded in).
__device__ __forceinline__ double ic_term(const EmConst& k, double Eo, double Ee, double e, double w) {
  const double g = Ee / k.me;
  const double G = 4.0 * e * g / k.me;
  const double q = Eo / (G * (Ee - Eo));
  const bool ok = (q >= 1.0 / (4.0 * g * g)) && (q <= 1.0) && (Eo < Ee) && (e > 0) && (g > 1.0);
  return ok ? bg_f(q, G) / e * w : 0.0;
}

// A_e[i][j][k], row (i, j), column k: photon i from electron j (cascade.py:78-104).
__global__ void k_em_ic(EmConst k, const double* __restrict__ E, int n, const double* __restrict__ eps,
                        const double* __restrict__ wk, int neps, double* __restrict__ A) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * n * neps) return;
  const int kk = (int)(t % neps);
  const int64_t ij = t / neps;
  const int i = (int)(ij / n), j = (int)(ij % n);
  A[t] = ic_term(k, E[i], E[j], eps[kk], wk[kk]);
}

// B_l[j][m][k]: photon E1[j][m] from electron j (cascade.py:107-138).
__global__ void k_em_icloss(EmConst k, const double* __restrict__ E, const double* __restrict__ E1, int n, int nE1,
                            const double* __restrict__ eps, const double* __restrict__ wk, int neps,
                            double* __restrict__ B) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * nE1 * neps) return;
  const int kk = (int)(t % neps);
  const int64_t jm = t / neps;
  const int j = (int)(jm / nE1);
  B[t] = ic_term(k, E1[jm], E[j], eps[kk], wk[kk]);
}

// A_p[i][j][k]: lepton i from photon j on target k (cascade.py:141-171).
__global__ void k_em_pair(EmConst k, const double* __restrict__ E, int n, const double* __restrict__ eps,
                          const double* __restrict__ wk, int neps, double* __restrict__ A) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * n * neps) return;
  const int kk = (int)(t % neps);
  const int64_t ij = t / neps;
  const int i = (int)(ij / n), j = (int)(ij % n);
  const double ge = E[i] / k.me, eg = E[j] / k.me, w = eps[kk] / k.me;
  const double denom = ge * (eg - ge);
  double v = 0.0;
  if (ge > 1.0 && ge < eg - 1.0 && denom > 0) {
    const double wmin = eg / (4.0 * denom);
    const double r = wmin / w;
    if (w > wmin && r < 1.0) {
      const double F = 4.0 * eg * eg / denom * log(4.0 * w * denom / eg) - 8.0 * eg * w +
                       2.0 * (2.0 * eg * w - 1.0) * eg * eg / denom -
                       (1.0 - 1.0 / (eg * w)) * (eg * eg * eg * eg) / (denom * denom);
      v = F / (w * w) / k.me * wk[kk];
    }
  }
  A[t] = v;
}

// Breit-Wheeler cross section [cm^2] at squared CM energy s (opacity.py:44-75).
__device__ __forceinline__ double sigma_gg(const EmConst& k, double s) {
  if (!(s > 4.0 * k.me * k.me)) return 0.0;
  const double w = 4.0 * k.me * k.me / s;
  const double beta = sqrt(1.0 - w), b2 = 1.0 - w;
  return 3.0 / 16.0 * k.sigma_t * w * ((3.0 - b2 * b2) * log((1.0 + beta) * (1.0 + beta) / w) - 2.0 * beta * (2.0 - b2));
}

// K[i][k] = 0.5 trapz_mu((1 - mu) sigma(2 E_i eps_k (1 - mu))) * w_k (cascade.py:425-441).
__global__ void k_em_tau(EmConst k, const double* __restrict__ E, int n, const double* __restrict__ epso,
                         const double* __restrict__ wo, int nepso, const double* __restrict__ mu, int nmu,
                         double* __restrict__ K) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * nepso) return;
  const int i = (int)(t / nepso), kk = (int)(t % nepso);
  double acc = 0.0, yprev = 0.0;
  for (int m = 0; m < nmu; ++m) {
    const double omm = 1.0 - mu[m];
    const double y = omm * sigma_gg(k, 2.0 * E[i] * epso[kk] * omm);
    if (m > 0) acc += (mu[m] - mu[m - 1]) * (y + yprev) / 2.0;
    yprev = y;
  }
  K[t] = 0.5 * acc * wo[kk];
}

// Photon densities at grid points for every redshift: out[k][z] (cascade.py:474-480).
__global__ void k_em_stack(FieldDesc f, const double* __restrict__ grid, int ng, const double* __restrict__ zs, int nz,
                           double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ng * nz) return;
  const int kk = t / nz, z = t % nz;
  const double v = field_density(f, grid[kk], zs[z]);
  out[t] = (isfinite(v) && v > 0) ? v : 0.0;
}

// ---------------------------------------------------------------------------
// Per-redshift matrices (cascade.py:494-556).  Layout: [z][i][j] row-major.
// ---------------------------------------------------------------------------
// emis[z][i][j] = raw[(i n + j)][z] * pref[j] (the contraction result, transposed)
__global__ void k_em_scatter_contraction(const double* __restrict__ raw, int n, int nz, const double* __restrict__ pref,
                                         double* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nz * n * n) return;
  const int z = (int)(t / ((int64_t)n * n));
  const int64_t ij = t - (int64_t)z * n * n;
  const int j = (int)(ij % n);
  out[t] = raw[ij * nz + z] * pref[j];
}

// loss[z][j] = power_out - rate * eps_mean, from dN[j][m][z] (raw contraction) * pref[j]
__global__ void k_em_loss(const double* __restrict__ rawdN, int n, int nE1, int nz, const double* __restrict__ pref,
                          const double* __restrict__ E1, const double* __restrict__ w1,
                          const double* __restrict__ eps_mean, double* __restrict__ loss) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nz) return;
  const int z = t / n, j = t % n;
  double p = 0.0, r = 0.0;
  for (int m = 0; m < nE1; ++m) {
    const double dn = rawdN[((size_t)j * nE1 + m) * nz + z] * pref[j];
    const double wm = w1[(size_t)j * nE1 + m];
    p += wm * E1[(size_t)j * nE1 + m] * dn;
    r += wm * dn;
  }
  loss[t] = p - r * eps_mean[z];
}

// column trapezoid of E * M over the row axis: out[z][j] = sum_i (y_i + y_{i+1}) (E_{i+1} - E_i) / 2
__device__ __forceinline__ double trapz_E_col(const double* __restrict__ M, const double* __restrict__ E, int n, int j) {
  double acc = 0.0;
  for (int i = 0; i + 1 < n; ++i)
    acc += (E[i + 1] * M[(size_t)(i + 1) * n + j] + E[i] * M[(size_t)i * n + j]) * (E[i + 1] - E[i]) / 2.0;
  return acc;
}

// P (energy-conserving pair), R, Sg, cold: one thread per (z, column j).
__global__ void k_em_columns(const double* __restrict__ pair, const double* __restrict__ emis,
                             const double* __restrict__ E, const double* __restrict__ dE, int n, int nz,
                             double cool_floor, double* __restrict__ P, double* __restrict__ Sg,
                             unsigned char* __restrict__ cold) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nz) return;
  const int z = t / n, j = t % n;
  const double* pz = pair + (size_t)z * n * n;
  const double* ez = emis + (size_t)z * n * n;
  const double outE = trapz_E_col(pz, E, n, j);
  const double sc = outE > 0 ? E[j] / outE : 0.0;
  double R = 0.0;
  for (int i = 0; i < n; ++i) {
    P[(size_t)z * n * n + (size_t)i * n + j] = outE > 0 ? pz[(size_t)i * n + j] * sc : 0.0;
    R += ez[(size_t)i * n + j] * dE[i];
  }
  double Eg = 0.0;
  for (int i = 0; i < n; ++i) {
    const double s = R > 0 ? ez[(size_t)i * n + j] / R : 0.0;
    Sg[(size_t)z * n * n + (size_t)i * n + j] = s;
    Eg += E[i] * s * dE[i];
  }
  cold[t] = (Eg < cool_floor * E[j]) || (R <= 0);
}

// De[z][r][j]: the loss-shift matrix.  Electron j emitting photon k keeps
// E_j - E_k, split between bins b and b+1 (cloud in cell); gathered per
// output in the order the reference's scatter-add visits it (all b terms by
// ascending k, then all b+1 terms by ascending k).
__global__ void k_em_shift(const double* __restrict__ Sg, const double* __restrict__ E, const double* __restrict__ dE,
                           const int* __restrict__ bidx, const double* __restrict__ frac, int n, int nz,
                           double* __restrict__ De) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nz * n * n) return;
  const int z = (int)(t / ((int64_t)n * n));
  const int r = (int)((t / n) % n), j = (int)(t % n);
  const double* S = Sg + (size_t)z * n * n;
  double acc = 0.0;
  for (int k = 0; k < n; ++k) {
    const int b = bidx[(size_t)k * n + j];
    if (b == r) acc += S[(size_t)k * n + j] * dE[k] * (frac[(size_t)k * n + j] / dE[b]);
  }
  for (int k = 0; k < n; ++k) {
    const int b = bidx[(size_t)k * n + j];
    if (b >= 0 && b + 1 == r) acc += S[(size_t)k * n + j] * dE[k] * ((1.0 - frac[(size_t)k * n + j]) / dE[b + 1]);
  }
  De[t] = acc;
}

// Cooled-IC matrix: Cum[z][i][m] = cumulative trapezoid over m of emis/loss,
// Mraw = Cum - diag on and above the diagonal; Mic = Mraw energy-normalised per column.
__global__ void k_em_cooled(const double* __restrict__ emis, const double* __restrict__ loss,
                            const double* __restrict__ E, int n, int nz, double* __restrict__ Mraw) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nz) return;
  const int z = t / n, i = t % n;
  const double* ez = emis + (size_t)z * n * n + (size_t)i * n;
  const double* lz = loss + (size_t)z * n;
  double* out = Mraw + (size_t)z * n * n + (size_t)i * n;
  double cum = 0.0, gprev = lz[0] > 0 ? ez[0] / lz[0] : 0.0, diag = 0.0;
  out[0] = 0.0;
  if (i == 0) diag = 0.0;
  for (int m = 1; m < n; ++m) {
    const double gm = lz[m] > 0 ? ez[m] / lz[m] : 0.0;
    cum += (gm + gprev) * (E[m] - E[m - 1]) / 2.0;
    gprev = gm;
    out[m] = cum;
    if (m == i) diag = cum;
  }
  for (int m = 0; m < n; ++m) out[m] = m >= i ? out[m] - diag : 0.0;
}

__global__ void k_em_normalise(double* __restrict__ M, const double* __restrict__ E, int n, int nz) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nz) return;
  const int z = t / n, j = t % n;
  double* Mz = M + (size_t)z * n * n;
  const double outE = trapz_E_col(Mz, E, n, j);
  const double sc = outE > 0 ? E[j] / outE : 0.0;
  for (int i = 0; i < n; ++i) Mz[(size_t)i * n + j] = outE > 0 ? Mz[(size_t)i * n + j] * sc : 0.0;
}

// dtau[z][i] from the raw contraction K No (raw[i][z]); Pe = exp(-dtau dl)
__global__ void k_em_escape(const double* __restrict__ rawtau, const double* __restrict__ dl, int n, int nz,
                            double* __restrict__ Pe) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nz) return;
  const int z = t / n, i = t % n;
  Pe[t] = exp(-rawtau[(size_t)i * nz + z] * dl[z]);
}

// ---------------------------------------------------------------------------
// The scattering iteration (cascade.py:558-589), all redshifts at once.
// ---------------------------------------------------------------------------
__global__ void k_em_iter_init(int n, int nz, double* __restrict__ G, double* __restrict__ e,
                               double* __restrict__ esc, double* __restrict__ fin) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nz * n * n) return;
  const int i = (int)((t / n) % n), j = (int)(t % n);
  G[t] = i == j ? 1.0 : 0.0;
  e[t] = esc[t] = fin[t] = 0.0;
}

// escaped += Pe G; T1 = (G - Pe G) dE_row (rows scaled by dE)
__global__ void k_em_iter_a(const double* __restrict__ Pe, const double* __restrict__ dE, int n, int nz,
                            const double* __restrict__ G, double* __restrict__ esc, double* __restrict__ T1) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nz * n * n) return;
  const int z = (int)(t / ((int64_t)n * n)), i = (int)((t / n) % n);
  const double pe = Pe[(size_t)z * n + i];
  const double pg = pe * G[t];
  esc[t] = esc[t] + pg;
  T1[t] = (G[t] - pg) * dE[i];
}

// e_cold dE, e_hot dE
__global__ void k_em_iter_b(const double* __restrict__ e, const unsigned char* __restrict__ cold,
                            const double* __restrict__ dE, int n, int nz, double* __restrict__ ec,
                            double* __restrict__ eh) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nz * n * n) return;
  const int z = (int)(t / ((int64_t)n * n)), i = (int)((t / n) % n);
  const bool c = cold[(size_t)z * n + i];
  ec[t] = (c ? e[t] : 0.0) * dE[i];
  eh[t] = (c ? 0.0 : e[t]) * dE[i];
}

// G = G_hot + G_cold; escaped += Pe G_cold; G -= Pe G_cold
__global__ void k_em_iter_c(const double* __restrict__ Pe, int n, int nz, const double* __restrict__ Gh,
                            const double* __restrict__ Gc, double* __restrict__ G, double* __restrict__ esc) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nz * n * n) return;
  const int z = (int)(t / ((int64_t)n * n)), i = (int)((t / n) % n);
  const double pe = Pe[(size_t)z * n + i];
  const double pg = pe * Gc[t];
  G[t] = Gh[t] + Gc[t];
  esc[t] = esc[t] + pg;
  G[t] = G[t] - pg;
}

// Convergence per redshift: max_j (E_in G + E_in e)_j / tot0_j < tol; a newly
// converged redshift freezes final = escaped + Pe G.  One CTA per redshift.
__global__ void k_em_iter_conv(const double* __restrict__ Ein, const double* __restrict__ Pe, int n, double tol,
                               const double* __restrict__ G, const double* __restrict__ e,
                               const double* __restrict__ esc, double* __restrict__ fin, int* __restrict__ done) {
  const int z = blockIdx.x;
  __shared__ double red[256];
  __shared__ int newly;
  const double* Gz = G + (size_t)z * n * n;
  const double* ez = e + (size_t)z * n * n;
  double mx = -1e300;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < n; ++i) {
      a += Ein[i] * Gz[(size_t)i * n + j];
      b += Ein[i] * ez[(size_t)i * n + j];
    }
    const double tot0 = Ein[j];  // E_in^T I
    mx = fmax(mx, (a + b) / tot0);
  }
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) newly = (red[0] < tol && !done[z]) ? 1 : 0;
  __syncthreads();
  if (!newly) return;
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
    const int i = t / n;
    fin[(size_t)z * n * n + t] = esc[(size_t)z * n * n + t] + Pe[(size_t)z * n + i] * Gz[t];
  }
  if (threadIdx.x == 0) done[z] = 1;
}

// final = done ? final : escaped; Mic dE (columns scaled) for T_e = final (Mic dE)
__global__ void k_em_finish(const int* __restrict__ done, const double* __restrict__ esc, const double* __restrict__ Mic,
                            const double* __restrict__ dE, int n, int nz, double* __restrict__ fin,
                            double* __restrict__ micd) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nz * n * n) return;
  const int z = (int)(t / ((int64_t)n * n)), j = (int)(t % n);
  if (!done[z]) fin[t] = esc[t];
  micd[t] = Mic[t] * dE[j];
}


// ---------------------------------------------------------------------------
// Bethe-Heitler e+- pair shape (bethe_heitler.py:27-297): the differential
// Born cross section, its nested fourth-order integrations into the
// field-free kernel K[i][j][k] (lepton i, nucleon j, target photon k), and per
// redshift the contraction with the photon density over ln eps (on the points
// where the density is positive), the kinematic band and the per-column
// energy normalisation.  Energies in units of m_e (leptons, photons) and the
// nucleon Lorentz factor.
// ---------------------------------------------------------------------------
__device__ double dsigma_bh(double k, double g, double u) {
  const double REG = 1e-30;
  const double p = sqrt(fmax(g * g - 1.0, 0.0) + REG);
  const double g1 = k - g;
  const double p1 = sqrt(fmax(g1 * g1 - 1.0, 0.0) + REG);
  const double D = g - u * p;
  const double T = sqrt(fmax(k * k + p * p - 2.0 * k * p * u, 0.0));
  if (!(k >= 2.0001 && k <= 600.0 && T >= 1e-30)) return 0.0;
  const double d1T = log((T + p1) / fmax(T - p1, REG));
  const double y1 = log(fmax((g1 + p1) / fmax(g1 - p1, REG), REG)) / fmax(p1, REG);
  const double Y = 2.0 * log(fmax((g * g1 + p * p1 + 1.0) / k, REG)) / fmax(p * p, REG);
  const double D4 = pow(D, 4.0);
  const double A0 = p * p1 / (k * k * k);
  const double A1 = -4.0 * (1.0 - u * u) * (2.0 * g * g + 1.0) / fmax(p * p * D4, REG);
  const double A2 = (5.0 * g * g - 2.0 * g * g1 + 3.0) / fmax(p * p * D * D, REG);
  const double A3 = (p * p - k * k) / fmax(T * T * D * D, REG);
  const double A4 = 2.0 * g1 / fmax(p * p * D, REG);
  const double A50 = Y / fmax(p * p1, REG);
  const double A51 = 2.0 * g * (1.0 - u * u) * (3.0 * k + p * p * g1) / fmax(D4, REG);
  const double A52 = (2.0 * g * g * (g * g + g1 * g1) - 7.0 * g * g - 3.0 * g * g1 - g1 * g1 + 1.0) / fmax(D * D, REG);
  const double A53 = k * (g * g - g * g1 - 1.0) / fmax(D, REG);
  const double A6 = -(d1T / fmax(p1 * T, REG)) *
                    (2.0 / fmax(D * D, REG) - 3.0 * k / fmax(D, REG) - k * (p * p - k * k) / fmax(T * T * D, REG));
  const double A7 = -2.0 * y1 / fmax(D, REG);
  return A0 * (A1 + A2 + A3 + A4 + A50 * (A51 + A52 + A53) + A6 + A7);
}

__device__ __forceinline__ double bh_inner(double ge, double gp, double omega, double ee) {
  const double REG = 1e-20;
  const double p_ = sqrt(fmax(ee * ee - 1.0, 0.0) + REG);
  const double xi = (gp * ee - ge) / (gp * p_);
  const bool ok = (p_ >= REG) && (xi >= -1.0) && (xi <= 1.0) && (ee >= 1.0) && (ee <= omega - 1.0);
  return ok ? omega * dsigma_bh(omega, ee, xi) / p_ : 0.0;
}

// Simpson-weighted fourth-order rule in 5 steps over [lo, hi] (0 when hi <= lo).
template <class F>
__device__ __forceinline__ double rk4_5(F f, double lo, double hi) {
  if (!(hi > lo)) return 0.0;
  const double dx = (hi - lo) / 5;
  double y = 0.0, x = lo;
  for (int s = 0; s < 5; ++s) {
    const double k1 = dx * f(x), k2 = dx * f(x + 0.5 * dx), k4 = dx * f(x + dx);
    y = y + (k1 + k4) / 6.0 + 2.0 * k2 / 3.0;
    x = x + dx;
  }
  return y;
}

__device__ double bh_outer(double ge, double gp, double omega) {
  const double REG = 1e-5;
  const double lo = (gp * gp + ge * ge) / (2.0 * gp * ge) + REG;
  const double hi = omega - 1.0 - REG;
  const bool ok = ((hi - lo) >= -1e-4 * lo) && ((hi - lo) / lo >= 1e-4);
  if (!ok) return 0.0;
  return rk4_5([&](double ee) { return bh_inner(ge, gp, omega, ee); }, lo, hi);
}

__global__ void k_bh_kernel(double me, double mp, const double* __restrict__ Ee, int ne,
                            const double* __restrict__ Ep, int np, const double* __restrict__ eps, int nk,
                            double* __restrict__ K) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)ne * np * nk) return;
  const int kk = (int)(t % nk);
  const int j = (int)((t / nk) % np), i = (int)(t / ((int64_t)nk * np));
  const double ge = Ee[i] / me, gp = Ep[j] / mp, ke = eps[kk] / me;
  const double upper = 2.0 * gp * ke;
  const double lower = (gp + ge) * (gp + ge) / (2.0 * gp * ge);
  double v = 0.0;
  if ((upper - lower) / fmax(lower, 1e-30) >= 1e-8) {
    const double y = rk4_5([&](double om) { return bh_outer(ge, gp, om); }, lower, upper);
    v = y * ge / (2.0 * pow(gp, 3.0) * (ke * ke));
  }
  K[t] = v;
}

// col[z][i][j] = trapezoid over ln eps (points with n > 0) of K n eps, in the band
__global__ void k_bh_col(const double* __restrict__ K, const double* __restrict__ Ee, int ne,
                         const double* __restrict__ Ep, int np, const double* __restrict__ eps,
                         const double* __restrict__ neps, int nk, int nz, double e_p_min,
                         double* __restrict__ col) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nz * ne * np) return;
  const int z = (int)(t / ((int64_t)ne * np));
  const int i = (int)((t / np) % ne), j = (int)(t % np);
  const bool band = Ee[i] <= Ep[j] && Ee[i] > 1e-6 * Ep[j] && Ep[j] >= e_p_min;
  double acc = 0.0, yprev = 0.0, xprev = 0.0;
  bool have = false;
  if (band) {
    const double* Kij = K + ((size_t)i * np + j) * nk;
    for (int k = 0; k < nk; ++k) {
      const double n = neps[(size_t)k * nz + z];
      if (!(n > 0 && eps[k] > 0)) continue;
      const double y = Kij[k] * (n * eps[k]);
      const double x = log(eps[k]);
      if (have) acc += (x - xprev) * (y + yprev) / 2.0;
      yprev = y;
      xprev = x;
      have = true;
    }
  }
  col[t] = band ? acc : 0.0;
}

// R[z][i][j] = col * (E_p[j] / carried) with carried = 2 trapezoid_i(E_e col)
__global__ void k_bh_norm(const double* __restrict__ col, const double* __restrict__ Ee, int ne,
                          const double* __restrict__ Ep, int np, int nz, double* __restrict__ R) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nz * np) return;
  const int z = t / np, j = t % np;
  const double* c = col + (size_t)z * ne * np;
  double acc = 0.0;
  for (int i = 0; i + 1 < ne; ++i)
    acc += (Ee[i + 1] - Ee[i]) * (Ee[i + 1] * c[(size_t)(i + 1) * np + j] + Ee[i] * c[(size_t)i * np + j]) / 2.0;
  const double carried = 2.0 * acc;
  for (int i = 0; i < ne; ++i)
    R[(size_t)z * ne * np + (size_t)i * np + j] = carried > 0 ? c[(size_t)i * np + j] * (Ep[j] / carried) : 0.0;
}
}  // namespace
