// prince_b200 -- B200-native ETD2 propagation core (sm_100a).
//
// One solve of the transport equation dn/dz = L(z) n + b(z) runs entirely on the
// device, in one CUDA graph:
//
//   1. photon matrix   PT[w][j] = s * n_gamma(E_ph[j], z_w)          (all windows)
//   2. pair-loss rate  kp[w][r] = scale[r] * trapz_xi(...)            (all windows)
//   3. first-window fold (GEMV) -> which coupling entries survive the
//      diagonal/off-diagonal split -> prefix sum -> M_off CSR pattern
//   4. fold GEMM over all windows on the FP64 tensor pipe (DMMA), written
//      straight into M_off values [w][nnz] and the diagonal [w][n]
//   5. ETD2 steps: two fused kernels per step (stage 1 -> a, F(x);
//      stage 2 -> x), each an SpMV/SpMM of M_off with the FD loss stencil,
//      the explicit-decay term, the injection and the phi-function epilogue.
//
// The algorithm follows the reference CPU solver of PriNCe:
//   src/prince_cr/solvers/etd2.py:329-439 (phi functions, step),
//   src/prince_cr/solvers/propagation.py:1017-1120 (per-window refresh),
//   propagation.py:1360-1508 (per-step operator and apply_F),
//   propagation.py:2495-2618 (multi-RHS),
//   src/prince_cr/interaction_rates.py:966-1067 (fold), 1277-1294 (pair loss).
// The data layout, the kernels and the launch structure are this project's own.

#include <cuda.h>  // CUtensorMap (the encoder is reached through cudaGetDriverEntryPoint)
#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/prince_b200.h"

namespace {

constexpr int kAbiVersion = 2;
constexpr int kLongRow = 256;      // rows with more coupling entries are cut into segments
constexpr int kMaxPhoton = 200;    // photon bins held in shared memory by the fold (208 KB tile)
constexpr int kColTile = 32;       // state columns per warp in the batched step
constexpr int kSegLen = 256;       // coupling entries per long-row segment
constexpr int kMaxEmBins = 1024;   // EM / nucleon bins of the cascade hook (as the transfer build)
constexpr int kMaxBhSpecies = 3072;  // charged nuclei of the hook's pair weights (their table in shared memory)

thread_local std::string g_error;

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t want) {
    if (want <= bytes && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (want == 0) want = 16;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace

constexpr long long kWaitTries = 1ll << 24;  // polls of a bounded wait (well above any staging time)
constexpr int kSlabPreDefault = 2;           // k_slab's default prefetch depth (row quartets)
struct pb_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
  std::string err;

  // problem dimensions
  int64_t n = 0;          // states
  int64_t R = 0;          // coupling entries (fold-kernel rows)
  int32_t dph = 0;        // photon bins
  bool have_coupling = false, have_kernel = false, have_photon_grid = false;
  bool have_field = false, have_fd = false, have_losses = false;

  // coupling pattern
  DBuf cpl_indptr, cpl_indices, cpl_row, cpl_is_diag;
  std::vector<int32_t> h_short_rows, h_long_rows;
  DBuf short_rows, long_rows;
  // long-row segments over the coupling entries
  int32_t n_seg = 0;
  DBuf seg_cb, seg_ce, seg_lr, lr_seg0, lr_nseg, seg_mb, seg_me, partial, counter;
  // fold kernel and photon grid
  DBuf kernel, eph;
  // photon field
  int32_t n_comp = 0;
  int32_t comp_kind[8];
  double comp_par[8][3];
  DBuf tab_z, tab_le, tab_v;        // tabulated photon field (kind 3)
  int32_t tab_nz = 0, tab_ne = 0;
  // FD operator
  int64_t nnzD = 0;
  DBuf d_indptr, d_indices, d_vals, d_diag;
  // losses
  DBuf adia_E, pair_scale, pair_bin, xi, phi_xi2, pair_pg;
  int32_t n_cr_bins = 0, n_xi = 0;
  // decay
  bool have_decay = false;
  int64_t nnzL = 0;
  DBuf l_diag, l_indptr, l_indices, l_vals;
  // injection
  int32_t n_src = 0, n_inj_rows = 0, n_src_cols = 0;
  DBuf inj_slot, inj_G, src_ptr;

  // per-solve workspace
  DBuf PT, zwin, rs, kp, keep, pos, dest, m_indptr, m_indices, m_vals, m_diag;
  DBuf s_h, s_dldz, s_hc, s_finj, s_win, s_coeff;
  DBuf X, A, F, rowf;
  DBuf scan_tmp;
  size_t scan_tmp_bytes = 0;
  int32_t last_W = 0;
  bool have_solution = false;
  std::vector<int32_t> h_win;   // window of each step of the current solve (host copy)
  std::vector<int32_t> h_nact;  // active columns of each step of the last solve (host copy)
  int64_t band_nnz = 0, slab_nnz = 0;  // coupling entries of the band rows and the bin-local rows

  // bin-blocked batched path (pb_set_layout): species blocks of `lay_d` bins
  std::vector<int64_t> h_cpl_indptr;
  std::vector<int32_t> h_cpl_indices;
  int32_t lay_d = 0, lay_nsp = 0;
  int64_t lay_nu = 0;               // rows of the species blocks [0, lay_nu); rows [lay_nu, n) are the tail
  int32_t n_tail = 0;               // tail rows (species on another grid), stepped by the general row kernel
  DBuf tail_rows;
  bool blocked_ok = false;          // the coupling pattern admits the band + slab kernels
  int32_t band_nb = 0, band_RT = 0, band_J = 0, n_slab_spec = 0;
  int64_t band_stride = 0;          // band-tile doubles per window
  int32_t band_npairs = 0;
  DBuf band_slot, band_spec, slab_spec, band_vals, band_part;
  // bin-local rows: coupling entries in bin-major order
  DBuf slab_rp, slab_sidx, slab_slot, slab_vals, slab_quart, slab_wrp, slab_rowslot, slab_fac;
  int64_t slab_nslots = 0;          // quartet slots over all bins (four per quartet)  // slab_rp: quad base per bin; slab_sidx: quads
  int64_t slab_nent = 0;            // value slots per window (4 per quad)
  int32_t slab_maxbin = 0;          // quads of the largest bin
  size_t slab_smem = 0, band_smem = 0;
  // FD stencil per bin (same in every species block): host copy of D and the table
  std::vector<int64_t> h_d_indptr;
  std::vector<int32_t> h_d_indices;
  std::vector<double> h_d_vals;
  bool fd_tab_ok = false;
  DBuf fd_cnt, fd_off, fd_val, fdbuf, fdkp, fd_dense, fdT_dense;
  bool fd_dense_ok = false;         // the stencil fits k_fd_dense's halo
  bool fdT_dense_ok = false;        // the transposed stencil fits k_fdT_dense's halo
  // transposed bin-blocked structures of the adjoint sweep (one band pair)
  bool blockedT_ok = false, fdT_ok = false;
  DBuf bandT_slot, slabT_rp, slabT_offs, slabT_slot, bandT_vals, slabT_vals, fdT_cnt, fdT_off, fdT_val;
  DBuf slabT_pairs, slabT_wrp;  // slabT_rp: quad base per bin; slabT_offs: quads
  DBuf vbuf, vbuf2, bTbuf, fdTbuf, outcols;
  int64_t slabT_nent = 0;
  int32_t slabT_maxbin = 0;
  size_t slabT_smem = 0, bandT_smem = 0;
  int32_t batched_mode = 1;         // 0: general row kernels; 1: bin-blocked kernels when the layout allows
  int32_t tma_mode = 1;             // 1: k_slab stages by TMA when tensor maps can be encoded; 0: cp.async
  long long staging_wait_tries = kWaitTries;  // k_slab's first staging wait (PB_OPT_STAGING_WAIT_TRIES)
  int32_t band_warps = 8;           // warps of a k_band CTA (PB_OPT_BAND_WARPS: 8 or 4)
  int32_t slab_pre = kSlabPreDefault;  // k_slab prefetch depth in row quartets (PB_OPT_SLAB_PREFETCH: 1..3)
  bool last_blocked = false;
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // the EM hook of a step beside the next step's nuclear stage (decoupled EM grid)
  cudaStream_t stream3 = nullptr;
  cudaEvent_t ev_hook_fork = nullptr, ev_hook_done = nullptr;
  bool tail_wait = false;           // the next tail launch waits for ev_hook_done
  int num_sms = 148;
  DBuf tmaps;                       // [4] CUtensorMap of X and A for k_slab's and k_band_tma's TMA staging
  bool tma_ok = false;              // tmaps hold k_slab's maps of the current X / A / ld
  bool tma_band_ok = false;         // tmaps also hold k_band_tma's maps (entries 2, 3)
  bool band_tma_fits = false;       // k_band_tma's shared memory fits the layout's band tiles
  bool last_tma = false;            // the last solve staged k_slab by TMA
  const void* tma_key[3] = {nullptr, nullptr, nullptr};
  DBuf tmapsT;                      // [2] CUtensorMap of the adjoint's v buffers for k_slabT's TMA staging
  bool tmaT_ok = false;             // tmapsT hold maps of the current vbuf / vbuf2 / ld
  const void* tmaT_key[3] = {nullptr, nullptr, nullptr};
  DBuf d_err;                       // int: a bounded wait of a kernel gave up
  // caller's row order: device row i holds the caller's row row_map[i] (none: identity)
  bool have_row_map = false;
  DBuf row_map;

  // EM cascade
  bool have_em = false;
  int32_t em_n = 0, em_ncr = 0, em_nbh = 0, em_W = 0;
  int64_t em_g = -1, em_m = -1, em_p = -1;
  DBuf em_bh_off, em_bh_A, em_invE, em_dE, em_Tg, em_Te, em_R, em_wbuf, em_es, em_lep, em_y;
  DBuf em_TgT, em_TeT, em_RT;       // per-window transposes (adjoint)
  std::vector<double> em_dl;

  // transposed constant operators (adjoint)
  DBuf dt_indptr, dt_indices, dt_vals, lt_indptr, lt_indices, lt_vals;
  DBuf inj_rows, src_col_d, nact;
  // checkpoints of the last solve and adjoint work buffers
  DBuf ckpt, lam, lam2, mu, rec_rf, rec_P, rec_Q, rec_sx, dsig, gb_inj, gs, g_out;
  DBuf erow, tkeys, tvals, skeys, svals, t_indptr, t_indices, t_perm, sort_tmp;
  int32_t last_ckpt = 0, last_K = 0;
  int64_t last_S = 0;
  uint32_t last_flags = 0;
  double last_scale = 1.0;

  // CUDA graph of the last solve's device work and the shape it was captured for
  cudaGraphExec_t graph_exec = nullptr, graph_exec2 = nullptr;
  std::vector<uint64_t> graph_key;
  int64_t graph_launches = 0;

  // timing
  float last_solve_ms = 0.f, last_device_ms = 0.f, last_steps_ms = 0.f;
  int64_t last_launches = 0;
};

namespace {

int fail(pb_context* c, int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf; else g_error = buf;
  return code;
}

unsigned blocks_for(int64_t work, int per_block) {
  return (unsigned)((work + per_block - 1) / per_block);
}

#define PB_CUDA(ctx, call)                                                              \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail((ctx), PB_ERR_CUDA, "%s failed: %s (%s:%d)", #call,                  \
                  cudaGetErrorString(e_), __FILE__, __LINE__);                          \
  } while (0)

// ---------------------------------------------------------------------------
// photon field on the device (prince_b200/photonfields.py kinds)
// ---------------------------------------------------------------------------
struct FieldDesc {
  int n;
  int kind[8];
  double p[8][3];
  double scale;
  // kind 3: a tabulated field, log10 dn/de on a regular (z, log10 E) grid
  const double* tz;    // tnz redshifts, increasing
  const double* tle;   // tne log10 energies [GeV], increasing
  const double* tv;    // tnz x tne log10 densities [GeV^-1 cm^-3]
  int tnz, tne;
};

// Interval of x on an increasing grid g[0..m-1] for linear interpolation:
// i with g[i] < x <= g[i+1], clamped to [0, m-2] (x = g[0] falls in the first).
__device__ __forceinline__ int grid_interval(const double* __restrict__ g, int m, double x) {
  int lo = 0, hi = m;  // first index with g[idx] >= x
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (g[mid] < x) lo = mid + 1; else hi = mid;
  }
  return min(max(lo - 1, 0), m - 2);
}

// Tabulated field (photonfields.py:227-345, the corrected EBL classes):
// log10 dn/de interpolated bilinearly in (z, log10 E), zero outside the table.
__device__ double table_density(const FieldDesc& f, double E, double z) {
  const double x = log10(E);
  if (!(z >= f.tz[0] && z <= f.tz[f.tnz - 1] && x >= f.tle[0] && x <= f.tle[f.tne - 1])) return 0.0;
  const int i = grid_interval(f.tz, f.tnz, z), j = grid_interval(f.tle, f.tne, x);
  const double u = __ddiv_rn(__dadd_rn(z, -f.tz[i]), __dadd_rn(f.tz[i + 1], -f.tz[i]));
  const double w = __ddiv_rn(__dadd_rn(x, -f.tle[j]), __dadd_rn(f.tle[j + 1], -f.tle[j]));
  const double* v0 = f.tv + (size_t)i * f.tne + j;
  const double* v1 = v0 + f.tne;
  const double cu = __dadd_rn(1.0, -u), cw = __dadd_rn(1.0, -w);
  double y = __dmul_rn(__dmul_rn(v0[0], cu), cw);
  y = __dadd_rn(y, __dmul_rn(__dmul_rn(v0[1], cu), w));
  y = __dadd_rn(y, __dmul_rn(__dmul_rn(v1[0], u), cw));
  y = __dadd_rn(y, __dmul_rn(__dmul_rn(v1[1], u), w));
  return exp10(y);
}

__device__ __forceinline__ double field_density(const FieldDesc& f, double E, double z) {
  double total = 0.0;
  const double opz = 1.0 + z;
  for (int c = 0; c < f.n; ++c) {
    double v;
    if (f.kind[c] == 1) {  // flat: (1+z)^2 * n0
      v = __dmul_rn(__dmul_rn(opz, opz), f.p[c][0]);
    } else if (f.kind[c] == 3) {  // tabulated
      v = table_density(f, E, z);
    } else {  // black / grey body: ((p0 (1+z)^2) Ered^p2) / (exp(Ered/p1) - 1)
      const double ered = __ddiv_rn(E, opz);
      const double eratio = __ddiv_rn(ered, f.p[c][1]);
      if (eratio < 709.0) {
        const double pz = __dmul_rn(f.p[c][0], __dmul_rn(opz, opz));
        const double pw = (f.kind[c] == 0) ? __dmul_rn(ered, ered) : pow(ered, f.p[c][2]);
        v = __ddiv_rn(__dmul_rn(pz, pw), __dadd_rn(exp(eratio), -1.0));
      } else {
        v = 0.0;
      }
    }
    total = (c == 0) ? v : __dadd_rn(total, v);
  }
  return (f.scale == 1.0) ? total : __dmul_rn(f.scale, total);
}

__global__ void k_photon_matrix(FieldDesc f, const double* __restrict__ eph, int dph,
                                const double* __restrict__ zwin, int W, double* __restrict__ PT) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W * dph) return;
  int w = i / dph, j = i % dph;
  PT[i] = field_density(f, eph[j], zwin[w]);
}

// Bethe-Heitler rate per (window, cosmic-ray bin): trapz over xi of
// n(pg[i][m], z) * phi_xi2[m] (interaction_rates.py:1280-1282).
__global__ void k_pair_rate(FieldDesc f, const double* __restrict__ pg, const double* __restrict__ xi,
                            const double* __restrict__ phi_xi2, int nxi, int ncr,
                            const double* __restrict__ zwin, double* __restrict__ rs) {
  const int w = blockIdx.y, i = blockIdx.x;
  const double z = zwin[w];
  double acc = 0.0;
  for (int m = threadIdx.x; m < nxi - 1; m += blockDim.x) {
    const double y0 = __dmul_rn(field_density(f, pg[(size_t)i * nxi + m], z), phi_xi2[m]);
    const double y1 = __dmul_rn(field_density(f, pg[(size_t)i * nxi + m + 1], z), phi_xi2[m + 1]);
    const double d = __dadd_rn(xi[m + 1], -xi[m]);
    acc += __ddiv_rn(__dmul_rn(d, __dadd_rn(y1, y0)), 2.0);
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) rs[(size_t)w * ncr + i] = v;
  }
}

// Fold kernel from per-channel response samples, one thread per (coupling
// entry, photon bin), rows in coupling-CSR order (interaction_rates.py:490-611,
// with the reference's operation order so the values are bit-identical):
//   kind 0:  0 [+ f_i dR_incl[i + j]] [- f_i dR_nonel[i + j]]
//   kind 1/2: max(g_ik ddR[i + j, k - i + d - 1], 0) [- f_i dR_nonel[i + j] if i = k]
// with i / k the mother / daughter bin, f_i = m_p / E_i, g_ik = f_i (dE_i / dE_k)
// and ddR a full table (kind 1) or sep_a[.] sep_b[.] (kind 2).
__global__ void k_build_kernel(const int* __restrict__ row, const int* __restrict__ col,
                               const int* __restrict__ ent_ch, const int* __restrict__ chan,
                               const double* __restrict__ f_mo, const double* __restrict__ dE,
                               const double* __restrict__ resp, const double* __restrict__ ddr,
                               const double* __restrict__ sep_a, const double* __restrict__ sep_b,
                               int d, int dph, int64_t total, double* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const int64_t e = t / dph;
  const int j = (int)(t - e * dph);
  const int i_mo = col[e] % d, i_da = row[e] % d;
  const int q = ent_ch[e];
  const int kind = chan[4 * q], p1 = chan[4 * q + 1], p2 = chan[4 * q + 2];
  const size_t na = (size_t)d + dph - 1, nb = 2 * (size_t)d - 1;
  const int a = i_mo + j;
  const double f = f_mo[i_mo];
  double v;
  if (kind == 0) {
    v = 0.0;
    if (p1 >= 0) v = __dadd_rn(v, __dmul_rn(f, resp[p1 * na + a]));
    if (p2 >= 0) v = __dadd_rn(v, -__dmul_rn(f, resp[p2 * na + a]));
  } else {
    const int b = i_da - i_mo + d - 1;
    const double g = __dmul_rn(f, __ddiv_rn(dE[i_mo], dE[i_da]));
    const double dd = kind == 1 ? ddr[(p1 * na + a) * nb + b] : __dmul_rn(sep_a[p1 * na + a], sep_b[p1 * nb + b]);
    v = __dmul_rn(g, dd);
    if (v < 0.0) v = 0.0;
    if (p2 >= 0 && i_mo == i_da) v = __dadd_rn(v, -__dmul_rn(f, resp[p2 * na + a]));
  }
  out[t] = v;
}

__global__ void k_pair_expand(const double* __restrict__ rs, const double* __restrict__ scale,
                              const int* __restrict__ bin, int ncr, int64_t n, int W,
                              double* __restrict__ kp) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * W) return;
  int64_t w = i / n, r = i % n;
  int b = bin[r];
  double rate = (b >= 0) ? rs[w * ncr + b] : 0.0;
  kp[i] = __dmul_rn(scale[r], rate);
}

// ---------------------------------------------------------------------------
// operator pattern: first-window fold and compaction
// ---------------------------------------------------------------------------
__global__ void k_coupling_rows(const int64_t* __restrict__ indptr, int64_t n,
                                const int* __restrict__ indices, int* __restrict__ row,
                                int* __restrict__ is_diag) {
  int64_t r = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (r >= n) return;
  for (int64_t j = indptr[r] + (threadIdx.x & 31); j < indptr[r + 1]; j += 32) {
    row[j] = (int)r;
    is_diag[j] = indices[j] == (int)r;
  }
}

// keep[i] = 1 where coupling entry i is off-diagonal and its first-window fold
// value is non-zero (the entries split_operator + eliminate_zeros retain).
__global__ void k_fold_first(const double* __restrict__ K, int64_t R, int dph,
                             const double* __restrict__ p0, const int* __restrict__ is_diag,
                             int* __restrict__ keep) {
  int64_t r = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  int lane = threadIdx.x & 31;
  if (r > R) return;
  if (r == R) {  // sentinel for the exclusive scan
    if (lane == 0) keep[R] = 0;
    return;
  }
  const double* row = K + (size_t)r * dph;
  double s = 0.0;
  for (int j = lane; j < dph; j += 32) s += row[j] * p0[j];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) keep[r] = (!is_diag[r] && s != 0.0) ? 1 : 0;
}

__global__ void k_compact(const int* __restrict__ keep, const int* __restrict__ pos,
                          const int* __restrict__ cpl_indices, const int* __restrict__ is_diag,
                          const int* __restrict__ row, int64_t R, int* __restrict__ dest,
                          int* __restrict__ diag_row, int* __restrict__ m_indices) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R) return;
  if (keep[i]) {
    dest[i] = pos[i];
    m_indices[pos[i]] = cpl_indices[i];
  } else {
    dest[i] = -1;
  }
  diag_row[i] = is_diag[i] ? row[i] : -1;
}

__global__ void k_m_indptr(const int64_t* __restrict__ cpl_indptr, const int* __restrict__ pos,
                           int64_t n, int64_t* __restrict__ m_indptr) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  m_indptr[i] = pos[cpl_indptr[i]];
}

// M_off range of each long-row segment from its coupling-entry range: the
// exclusive prefix count of kept entries maps coupling index -> M_off index.
__global__ void k_seg_map(const int64_t* __restrict__ cb, const int64_t* __restrict__ ce,
                          const int* __restrict__ pos, int nseg, int64_t* __restrict__ mb,
                          int64_t* __restrict__ me) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nseg) return;
  mb[i] = pos[cb[i]];
  me[i] = pos[ce[i]];
}

// ---------------------------------------------------------------------------
// fold GEMM on the FP64 tensor pipe: out[w][r] = sum_j K[r][j] * PT[w][j]
// mma.sync m8n8k4 f64 (DMMA).  CTA tile 64 entries x 64 windows, whole photon
// axis in shared memory; the epilogue scatters into M_off values / diagonal.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma884(double& c0, double& c1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

constexpr int kFoldBM = 64, kFoldBN = 64;

__global__ void __launch_bounds__(256) k_fold_gemm(const double* __restrict__ K, int64_t R, int dph,
                                                   int kpad, const double* __restrict__ PT, int W,
                                                   const int* __restrict__ dest,
                                                   const int* __restrict__ diag_row,
                                                   double* __restrict__ mv, int64_t mv_stride,
                                                   double* __restrict__ md, int64_t n,
                                                   const int* __restrict__ band_slot,
                                                   double* __restrict__ band, int64_t band_stride,
                                                   const int* __restrict__ slab_slot,
                                                   double* __restrict__ slab, int64_t slab_stride) {
  extern __shared__ double smem[];
  const int lda = kpad + 4;  // +4 doubles: 8-row fragments spread over all banks
  double* As = smem;
  double* Bs = smem + kFoldBM * lda;
  const int64_t r0 = (int64_t)blockIdx.x * kFoldBM;
  const int w0 = blockIdx.y * kFoldBN;
  for (int i = threadIdx.x; i < kFoldBM * kpad; i += blockDim.x) {
    int rr = i / kpad, kk = i % kpad;
    As[rr * lda + kk] = (r0 + rr < R && kk < dph) ? K[(size_t)(r0 + rr) * dph + kk] : 0.0;
  }
  for (int i = threadIdx.x; i < kFoldBN * kpad; i += blockDim.x) {
    int ww = i / kpad, kk = i % kpad;
    Bs[ww * lda + kk] = (w0 + ww < W && kk < dph) ? PT[(size_t)(w0 + ww) * dph + kk] : 0.0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wm = wid & 1, wn = wid >> 1;  // warp tile: 32 entries x 16 windows
  const int g = lane >> 2, t = lane & 3;
  double acc[4][2][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  for (int k0 = 0; k0 < kpad; k0 += 4) {
    double af[4], bf[2];
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) af[mt] = As[(wm * 32 + mt * 8 + g) * lda + k0 + t];
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) bf[nt] = Bs[(wn * 16 + nt * 8 + g) * lda + k0 + t];
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) dmma884(acc[mt][nt][0], acc[mt][nt][1], af[mt], bf[nt]);
  }
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    const int64_t r = r0 + wm * 32 + mt * 8 + g;
    if (r >= R) continue;
    const int de = dest[r];
    const int dr = diag_row[r];
    const int bs = (band_slot && de >= 0) ? band_slot[r] : -1;
    const int ss = (slab_slot && de >= 0) ? slab_slot[r] : -1;
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int w = w0 + wn * 16 + nt * 8 + t * 2 + i;
        if (w >= W) continue;
        const double v = acc[mt][nt][i];
        if (de >= 0) mv[(size_t)w * mv_stride + de] = v;
        if (dr >= 0) md[(size_t)w * n + dr] = v;
        if (bs >= 0) band[(size_t)w * band_stride + bs] = v;
        if (ss >= 0) slab[(size_t)w * slab_stride + ss] = v;
      }
  }
}

// ---------------------------------------------------------------------------
// correctly rounded exp (double-double; same operation sequence as oracle/crexp.py)
//
// x = k ln2 + r, s = r / 2^10, expm1(s) by a degree-9 Taylor polynomial in
// double-double, ten squarings E <- 2E + E^2, then (1 + E) 2^k rounded once.
// Double-double arithmetic after Dekker and Knuth (QD library, Hida/Li/Bailey);
// every operation is an explicitly rounded intrinsic so the sequence cannot be
// contracted into FMAs and matches the host form bit for bit.
// ---------------------------------------------------------------------------
struct DD {
  double h, l;
};

__device__ __forceinline__ DD dd_two_sum(double a, double b) {
  const double s = __dadd_rn(a, b);
  const double bb = __dadd_rn(s, -a);
  return {s, __dadd_rn(__dadd_rn(a, -__dadd_rn(s, -bb)), __dadd_rn(b, -bb))};
}
__device__ __forceinline__ DD dd_quick(double a, double b) {
  const double s = __dadd_rn(a, b);
  return {s, __dadd_rn(b, -__dadd_rn(s, -a))};
}
__device__ __forceinline__ DD dd_two_prod(double a, double b) {
  const double p = __dmul_rn(a, b);
  return {p, __fma_rn(a, b, -p)};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
  DD s = dd_two_sum(a.h, b.h);
  const DD t = dd_two_sum(a.l, b.l);
  s.l = __dadd_rn(s.l, t.h);
  s = dd_quick(s.h, s.l);
  s.l = __dadd_rn(s.l, t.l);
  return dd_quick(s.h, s.l);
}
__device__ __forceinline__ DD dd_mul(DD a, DD b) {
  DD p = dd_two_prod(a.h, b.h);
  p.l = __dadd_rn(p.l, __dadd_rn(__dmul_rn(a.h, b.l), __dmul_rn(a.l, b.h)));
  return dd_quick(p.h, p.l);
}

__constant__ double c_expcoef[9][2] = {
    {1.0, 0.0},
    {0.5, 0.0},
    {0x1.5555555555555p-3, 0x1.5555555555555p-57},
    {0x1.5555555555555p-5, 0x1.5555555555555p-59},
    {0x1.1111111111111p-7, 0x1.1111111111111p-63},
    {0x1.6c16c16c16c17p-10, -0x1.f49f49f49f49fp-65},
    {0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-73},
    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
};

__device__ double cr_exp(double x) {
  if (isnan(x)) return x;
  if (x > 709.782712893384) return CUDART_INF;
  if (x < -745.1332191019412) return 0.0;
  const double ln2_hi = 0x1.62e42fefa39efp-1, ln2_lo = 0x1.abc9e3b39803fp-56;
  const double k = rint(__dmul_rn(x, 1.4426950408889634));
  const DD p = dd_two_prod(k, ln2_hi);
  DD r = dd_two_sum(x, -p.h);
  r = dd_add(r, DD{-p.l, 0.0});
  r = dd_add(r, DD{-__dmul_rn(k, ln2_lo), 0.0});
  const DD s{__dmul_rn(r.h, 0.0009765625), __dmul_rn(r.l, 0.0009765625)};
  DD t{c_expcoef[8][0], c_expcoef[8][1]};
#pragma unroll
  for (int i = 7; i >= 0; --i) {
    t = dd_mul(t, s);
    t = dd_add(t, DD{c_expcoef[i][0], c_expcoef[i][1]});
  }
  DD e = dd_mul(t, s);
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const DD q = dd_mul(e, e);
    e = dd_add(DD{__dmul_rn(e.h, 2.0), __dmul_rn(e.l, 2.0)}, q);
  }
  const DD v = dd_add(e, DD{1.0, 0.0});
  return ldexp(__dadd_rn(v.h, v.l), (int)k);
}

__global__ void k_eval_exp(const double* __restrict__ x, double* __restrict__ y, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = cr_exp(x[i]);
}

// ---------------------------------------------------------------------------
// ETD2 step kernels
//
// Per step, two launches (stage 1 and 2) over the rows; short rows get a warp,
// rows with more than kLongRow coupling entries a whole CTA.  The per-row
// factors of a step (kappa, eD, phi1, phi2) are computed once per row by the
// stage-2 launch of the previous step (k_prep for the first step) into a
// buffer pair indexed by the step's parity, so the column tiles of the batched
// kernel never recompute them.
// ---------------------------------------------------------------------------
struct StepParams {
  int64_t n;
  int ld;            // leading dimension of the (n x ld) state buffers
  int ncols;         // active columns this step
  int64_t step;
  int step_w;        // rate window of this step (k_slab's entry values), set with step
  const CUtensorMap* tmap_src;  // k_slab: tensor map of src for the TMA staging, or null (cp.async staging)
  const CUtensorMap* tmap_band;  // k_band_tma: tensor map of src as (64 columns x d bins) boxes, or null
  long long wait_tries;         // k_slab: polls of the staging wait before it gives up (the drain keeps kWaitTries)
  int* err;          // set to a nonzero code when a bounded wait gives up
  int64_t n_steps;
  uint32_t flags;
  const double* h;
  const double* dldz;
  const double* hc;
  const double* finj;
  const int* win;
  // operator
  const int64_t* m_indptr;
  const int* m_indices;
  const double* m_vals;
  int64_t m_wstride;
  const double* m_diag;
  const int64_t* d_indptr;
  const int* d_indices;
  const double* d_vals;
  const double* d_diag;
  const double* E;
  const double* kp;  // W x n or null
  const int64_t* l_indptr;
  const int* l_indices;
  const double* l_vals;
  const double* l_diag;
  // injection
  const int* inj_slot;
  const double* G;
  int n_src;
  const int* src_ptr;
  const double* coeff;
  // per-row step factors, [2][n] each (parity of the step)
  double* eD;
  double* phi1;
  double* phi2;
  double* kap;
  // states
  const double* src;  // stage 1: x ; stage 2: a
  const double* x;    // stage 1: x
  double* a;          // stage 1 writes, stage 2 reads
  double* f;          // F(x): stage 1 writes, stage 2 reads
  double* xout;       // stage 2 writes
  const int* rows;    // short rows
  int nrows;
  int nsb;            // blocks of the launch that work on short rows
  // long rows: segments of at most kSegLen coupling entries
  const int* seg_lr;        // long-row index of each segment
  const int64_t* seg_mb;    // M_off range of each segment
  const int64_t* seg_me;
  int nseg;
  const int* lr_row;        // state row of each long row
  const int* lr_seg0;       // first segment of each long row
  const int* lr_nseg;       // number of segments of each long row
  double* partial;          // nseg x ld partial sums
  int* counter;             // finished segments per (long row, column tile)
  int ctiles;               // column tiles per long row in `counter`
  // recording for the adjoint (all null in a plain solve)
  double inv_scale;         // 1 / photon scale
  double* dsig;             // [2][n] d(d)/d(scale)
  double* dphi1;            // [2][n] phi1'(h d)
  double* dphi2;            // [2][n] phi2'(h d)
  double* rec_rf;           // [rec_len][4][n]: eD, phi1, phi2, kappa of each recorded step
  double* rec_P;            // [rec_len][n x ld]
  double* rec_Q;            // [rec_len][n x ld]
  double* rec_sx;           // n x ld: S x of the current step (stage 1 -> stage 2)
  int64_t rec_k0;
  int rec_len;
  // bin-blocked batched path
  int d;                    // bins per species block
  int nsp;                  // species blocks
  const int* slab_spec;     // species whose coupling rows are bin-local
  int n_slab_spec;
  const int* slab_qbase;    // [d + 1] first entry quad of each bin (even)
  const unsigned long long* slab_q;  // per quad: byte offsets of the 4 entries' mother rows in k_slab's slab, 16 bits each
  const int4* slab_quart;   // row quartets of k_slab's warps: species 0 | 1 << 16, 2 | 3 << 16 (0xffff: none), first quad, quads per row
  const int* slab_wrp;      // [d][kSlabWarps + 1] first quartet of each warp of a bin's CTA
  const double* slab_vals;  // [W][slab_stride] M_off values of the quads (4 per quad, zero padding)
  int64_t slab_stride;
  int slab_maxq;            // quads of the largest bin (shared-memory sizing)
  int slab_maxp;            // row quartets of a bin
  const int* slab_rowslot;  // [n] quartet slot of each bin-local row (-1: other rows)
  double* slab_fac;         // [2][3][slab_nslots] eD, phi1, phi2 of the bin-local rows in quartet-slot order
  int64_t slab_nslots;
  const int* fd_cnt;        // per bin: FD stencil entries, row offsets and values
  const int* fd_off;
  const double* fd_val;
  const double* fd_dense;   // [d][kFdDenseW] stencil weights of offsets -kFdHalo..kFdHalo (k_fd_dense)
  double* fdbuf;            // n x ld: D_off (kappa v) of the stage
  double* fdkp;             // n x ld: D_off (kappa_pair v), adjoint record pass with the photon scale, or null
  const int* band_spec;     // species with cross-bin coupling rows
  int nb;
  const double* band_vals;  // [W][nsp][band pair][2][RT][J][32] DMMA A fragments
  int64_t band_stride;
  double* band_part;        // [G][nb][d][ld] partial sums of the band rows
  int ngroups;              // mother-species groups of the band launch
  int spg;                  // species per group
};

struct StepScalars {
  double h, dl, hc, finj;
  int w;
  bool kap, adia, pair, photohad, inj, decay;
};

__device__ __forceinline__ StepScalars load_scalars(const StepParams& p, int64_t step) {
  StepScalars s;
  s.h = p.h[step];
  s.dl = p.dldz[step];
  s.hc = p.hc[step];
  s.finj = p.finj[step];
  s.w = p.win[step];
  s.kap = (p.flags & PB_PARTIAL_DIFF) != 0;
  s.adia = (p.flags & PB_ADIABATIC) != 0;
  s.pair = (p.flags & PB_PAIRPROD) != 0 && p.kp != nullptr;
  s.photohad = (p.flags & PB_PHOTOHAD) != 0;
  s.inj = (p.flags & PB_INJECTION) != 0 && p.G != nullptr;
  s.decay = (p.flags & PB_DECAY) != 0 && p.l_diag != nullptr;
  return s;
}

// phi functions with the Taylor patches of etd2.py:43-46, 329-390
__device__ __forceinline__ void phi_of(double h, double d, double& eD, double& phi1, double& phi2) {
  const double hd = __dmul_rn(d, h);
  const double e = cr_exp(hd);
  eD = e;
  const double ahd = fabs(hd);
  if (ahd > 1e-6) {
    phi1 = __ddiv_rn(__dadd_rn(e, -1.0), hd);
  } else {
    phi1 = __dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(hd, 1.0 / 6.0), 0.5), hd), 1.0);
  }
  if (ahd > 1e-3) {
    phi2 = __ddiv_rn(__dadd_rn(__dadd_rn(e, -1.0), -hd), __dmul_rn(hd, hd));
  } else {
    phi2 = __dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(hd, 1.0 / 24.0), 1.0 / 6.0), hd), 0.5);
  }
}

// phi1'(w) = (e^w - phi1)/w and phi2'(w) = (phi1 - 2 phi2)/w; for |w| < 0.1 their
// power series sum_n (n+1) w^n/(n+2)! and sum_n (n+1) w^n/(n+3)! (13 terms).
__device__ __forceinline__ void dphi_of(double w, double e, double f1, double f2, double& d1, double& d2) {
  if (fabs(w) < 0.1) {
    double a = 0.0, b = 0.0;
    double fact2 = 87178291200.0;    // (12 + 2)!
    double fact3 = 1307674368000.0;  // (12 + 3)!
    for (int n = 12; n >= 0; --n) {  // Horner from the top
      a = a * w + (n + 1) / fact2;
      b = b * w + (n + 1) / fact3;
      fact2 /= (n + 2);
      fact3 /= (n + 3);
    }
    d1 = a;
    d2 = b;
  } else {
    d1 = (e - f1) / w;
    d2 = (f1 - 2.0 * f2) / w;
  }
}

// kappa (propagation.py:1393-1401) and d = dldz (M_diag + kappa D_diag [+ Lambda_diag])
// (propagation.py:1408-1422) of row r at `step`, then its phi factors.
__device__ __forceinline__ void row_prep(const StepParams& p, int64_t step, int64_t r) {
  const StepScalars s = load_scalars(p, step);
  double k = 0.0;
  if (s.adia) k = __dmul_rn(s.hc, p.E[r]);
  if (s.pair) k = __dadd_rn(k, p.kp[(size_t)s.w * p.n + r]);
  double d = __dmul_rn(p.m_diag[(size_t)s.w * p.n + r], s.dl);
  if (s.kap) d = __dadd_rn(d, __dmul_rn(__dmul_rn(k, p.d_diag[r]), s.dl));
  if (s.decay) d = __dadd_rn(d, __dmul_rn(p.l_diag[r], s.dl));
  double e, f1, f2;
  phi_of(s.h, d, e, f1, f2);
  const size_t o = (size_t)(step & 1) * p.n + r;
  p.eD[o] = e;
  p.phi1[o] = f1;
  p.phi2[o] = f2;
  p.kap[o] = k;
  if (p.slab_rowslot) {  // k_slab stages the factors of a bin's rows as three contiguous runs
    const int sl = p.slab_rowslot[r];
    if (sl >= 0) {
      double* fc = p.slab_fac + (size_t)(step & 1) * 3 * p.slab_nslots + sl;
      fc[0] = e;
      fc[p.slab_nslots] = f1;
      fc[2 * p.slab_nslots] = f2;
    }
  }
  if (p.dsig) {  // derivatives with respect to the photon scale (adjoint record pass)
    const double md = p.m_diag[(size_t)s.w * p.n + r] * p.inv_scale;
    double ds = md;
    if (s.kap && s.pair) ds += (p.kp[(size_t)s.w * p.n + r] * p.inv_scale) * p.d_diag[r];
    ds *= s.dl;
    double d1, d2;
    dphi_of(s.h * d, e, f1, f2, d1, d2);
    p.dsig[o] = ds;
    p.dphi1[o] = d1;
    p.dphi2[o] = d2;
  }
  if (p.rec_rf) {
    const int64_t j = step - p.rec_k0;
    if (j >= 0 && j < p.rec_len) {
      double* rf = p.rec_rf + (size_t)j * 4 * p.n;
      rf[r] = e;
      rf[p.n + r] = f1;
      rf[2 * p.n + r] = f2;
      rf[3 * p.n + r] = k;
    }
  }
}

__global__ void k_prep(StepParams p) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < p.n) row_prep(p, p.step, r);
}

// ---------------------------------------------------------------------------
// Scratch of pb_integrate_const_noalloc: one file-scope device array (every
// GPU that loads the library holds it until exit).  Layout, in bytes from the
// start: a and F(x) (n doubles each), the row factors (8 n doubles), the
// per-step h and dl/dz (s doubles each), the window index (s ints), the row
// list (n ints), an all-zero row pointer (n + 1 int64) and a 256-byte status
// block (the CSR check's flag), for n = the state limit and s = the step limit.
// ---------------------------------------------------------------------------
constexpr int64_t kNaMaxStates = PB_NOALLOC_MAX_STATES;
constexpr int64_t kNaMaxSteps = PB_NOALLOC_MAX_STEPS;
constexpr size_t kNaBytes = (size_t)kNaMaxStates * 10 * sizeof(double) + (size_t)kNaMaxSteps * 2 * sizeof(double) +
                            (size_t)kNaMaxSteps * sizeof(int) + (size_t)kNaMaxStates * sizeof(int) +
                            (size_t)(kNaMaxStates + 1) * sizeof(int64_t) + 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

// Validates a caller's CSR before any step kernel reads through it: indptr
// starts at 0, never decreases and ends at nnz, and every column index lies in
// [0, n).  Reads stay inside the sizes the caller declared (n + 1 row
// pointers, nnz indices); a violation sets bit 0 (row pointers) or bit 1
// (indices) of *flag.
__global__ void k_noalloc_check_csr(int64_t n, int64_t nnz, const int64_t* __restrict__ indptr,
                                    const int32_t* __restrict__ indices, unsigned int* __restrict__ flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && indptr[i] > indptr[i + 1]) atomicOr(flag, 1u);
  if (i == 0 && indptr[0] != 0) atomicOr(flag, 1u);
  if (i == n && indptr[n] != nnz) atomicOr(flag, 1u);
  if (i < nnz) {
    const int32_t c = indices[i];
    if (c < 0 || (int64_t)c >= n) atomicOr(flag, 2u);
  }
}

__global__ void k_noalloc_fill(int64_t n, int64_t n_steps, const double* __restrict__ z, double* __restrict__ h,
                               double* __restrict__ ones, int* __restrict__ win, int* __restrict__ rows,
                               int64_t* __restrict__ zero_indptr) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_steps) {
    h[i] = __dadd_rn(z[i + 1], -z[i]);
    ones[i] = 1.0;
    win[i] = 0;
  }
  if (i < n) rows[i] = (int)i;
  if (i <= n) zero_indptr[i] = 0;
}

// b(z) at (row r, column k): finj * sum_s coeff_s * g_s[r] (propagation.py:363-370, 2476-2488)
__device__ __forceinline__ double inj_at(const StepParams& p, const StepScalars& s, int64_t r, int k) {
  const int slot = p.inj_slot[r];
  if (slot < 0) return 0.0;
  const int s0 = p.src_ptr[k], s1 = p.src_ptr[k + 1];
  if (s0 == s1) return 0.0;
  const double* c = p.coeff + (size_t)p.step * p.n_src;
  const double* g = p.G + (size_t)slot * p.n_src;
  double acc = __dmul_rn(c[s0], g[s0]);
  for (int q = s0 + 1; q < s1; ++q) acc = __dadd_rn(acc, __dmul_rn(c[q], g[q]));
  return __dmul_rn(s.finj, acc);
}

// The rest of apply_F for one (row, column): the FD loss term, the decay term,
// the dl/dz scale and the injection (propagation.py:1473-1486).  Sums run in
// CSR order without contraction, as the host sparse products do.
__device__ __forceinline__ double finish_F(const StepParams& p, const StepScalars& s, int64_t r,
                                           int k, const double* __restrict__ v, double sM) {
  const double* kap = p.kap + (size_t)(p.step & 1) * p.n;
  double out = sM;
  if (s.kap) {
    double sD = 0.0;
    for (int64_t j = p.d_indptr[r]; j < p.d_indptr[r + 1]; ++j) {
      const int c = p.d_indices[j];
      sD = __dadd_rn(sD, __dmul_rn(p.d_vals[j], __dmul_rn(kap[c], v[(size_t)c * p.ld + k])));
    }
    out = __dadd_rn(out, sD);
  }
  if (s.decay) {
    double sL = 0.0;
    for (int64_t j = p.l_indptr[r]; j < p.l_indptr[r + 1]; ++j)
      sL = __dadd_rn(sL, __dmul_rn(p.l_vals[j], v[(size_t)p.l_indices[j] * p.ld + k]));
    out = __dadd_rn(out, sL);
  }
  out = __dmul_rn(out, s.dl);
  if (s.inj) out = __dadd_rn(out, inj_at(p, s, r, k));
  return out;
}

// S v = (1/scale) dl/dz (M_off v + D_off (kappa_pair v)): the derivative of the
// operator with respect to the photon scale applied to v, from the M_off sum.
__device__ __forceinline__ double scale_deriv_apply(const StepParams& p, const StepScalars& s, int64_t r, int k,
                                                    const double* __restrict__ v, double sM) {
  double out = sM;
  if (s.kap && s.pair) {
    const double* kp = p.kp + (size_t)s.w * p.n;
    double sD = 0.0;
    for (int64_t j = p.d_indptr[r]; j < p.d_indptr[r + 1]; ++j) {
      const int c = p.d_indices[j];
      sD += p.d_vals[j] * (kp[c] * v[(size_t)c * p.ld + k]);
    }
    out += sD;
  }
  return out * s.dl * p.inv_scale;
}

template <int STAGE>
__device__ __forceinline__ void record(const StepParams& p, const StepScalars& s, int64_t r, int k, double sM,
                                       double F) {
  const size_t o = (size_t)(p.step & 1) * p.n + r;
  const size_t idx = (size_t)r * p.ld + k;
  const int64_t j = p.step - p.rec_k0;
  if (j < 0 || j >= p.rec_len) return;
  const size_t ro = (size_t)j * p.n * p.ld + idx;
  const double h = s.h, ds = p.dsig[o];
  if (STAGE == 1) {
    const double Sx = scale_deriv_apply(p, s, r, k, p.src, s.photohad ? sM : 0.0);
    p.rec_sx[idx] = Sx;
    p.rec_P[ro] = p.eD[o] * h * ds * p.x[idx] + h * h * p.dphi1[o] * ds * F + h * p.phi1[o] * Sx;
  } else {
    const double Sa = scale_deriv_apply(p, s, r, k, p.src, s.photohad ? sM : 0.0);
    const double dF = F - p.f[idx];
    p.rec_Q[ro] = h * h * p.dphi2[o] * ds * dF + h * p.phi2[o] * (Sa - p.rec_sx[idx]);
  }
}

template <int STAGE>
__device__ __forceinline__ void row_epilogue(const StepParams& p, const StepScalars& s, int64_t r,
                                             int k, double sM) {
  const size_t o = (size_t)(p.step & 1) * p.n + r;
  const size_t idx = (size_t)r * p.ld + k;
  const double F = finish_F(p, s, r, k, p.src, sM);
  if (p.rec_P) record<STAGE>(p, s, r, k, sM, F);
  if (STAGE == 1) {
    // a = eD x + (phi1 F(x)) h  (etd2.py:427-430)
    const double a = __dadd_rn(__dmul_rn(p.eD[o], p.x[idx]), __dmul_rn(__dmul_rn(p.phi1[o], F), s.h));
    p.a[idx] = a;
    p.f[idx] = F;
  } else {
    // x = a + ((F(a) - F(x)) h) phi2  (etd2.py:435-438)
    const double dF = __dmul_rn(__dadd_rn(F, -p.f[idx]), s.h);
    p.xout[idx] = __dadd_rn(p.a[idx], __dmul_rn(dF, p.phi2[o]));
  }
}

// stage 2 of step k prepares the row factors of step k + 1 (one thread per row)
__device__ __forceinline__ void prep_next(const StepParams& p, int64_t r) {
  if (p.step + 1 < p.n_steps) row_prep(p, p.step + 1, r);
}

// Long rows are cut into segments of at most kSegLen coupling entries.  A warp
// sums one segment into `partial`; the last warp to finish a (row, column tile)
// -- found with a fence and an atomic ticket, no waiting -- adds the row's
// partials in segment order and runs the row epilogue.
__device__ __forceinline__ bool last_of_row(const StepParams& p, int lr, int tile, int lane) {
  __syncwarp();      // every lane's partial is written before lane 0 publishes the ticket
  __threadfence();
  int t = 0;
  if (lane == 0) t = atomicAdd(&p.counter[(size_t)lr * p.ctiles + tile], 1);
  t = __shfl_sync(0xffffffffu, t, 0);
  const bool last = t == p.lr_nseg[lr] - 1;
  if (last) {
    __threadfence();
    if (lane == 0) p.counter[(size_t)lr * p.ctiles + tile] = 0;  // ready for the next launch
  }
  return last;
}

// Single column.  Blocks [0, nsb): a thread per short row, summing the row in
// CSR order without contraction (as the host CSR product does).  Blocks
// [nsb, ...): a warp per long-row segment.
template <int STAGE>
__global__ void __launch_bounds__(256) k_step_plain(StepParams p) {
  const StepScalars s = load_scalars(p, p.step);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const double* __restrict__ v = p.src;
  const double* __restrict__ mv = p.m_vals + (size_t)s.w * p.m_wstride;
  if ((int)blockIdx.x < p.nsb) {
    const int64_t ri = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ri >= p.nrows) return;
    const int64_t r = p.rows[ri];
    double acc = 0.0;
    if (s.photohad) {
      const int64_t j1 = p.m_indptr[r + 1];
#pragma unroll 4
      for (int64_t j = p.m_indptr[r]; j < j1; ++j) acc = __dadd_rn(acc, __dmul_rn(mv[j], v[p.m_indices[j]]));
    }
    row_epilogue<STAGE>(p, s, r, 0, acc);
    if (STAGE == 2) prep_next(p, r);
    return;
  }
  const int seg = (blockIdx.x - p.nsb) * (blockDim.x >> 5) + wid;
  if (seg >= p.nseg) return;
  double acc = 0.0;
  if (s.photohad)
    for (int64_t j = p.seg_mb[seg] + lane; j < p.seg_me[seg]; j += 32) acc += mv[j] * v[p.m_indices[j]];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) p.partial[seg] = acc;
  const int lr = p.seg_lr[seg];
  if (!last_of_row(p, lr, 0, lane)) return;
  if (lane == 0) {
    const int s0 = p.lr_seg0[lr], ns = p.lr_nseg[lr];
    double t = 0.0;
    for (int q = 0; q < ns; ++q) t += __ldcg(p.partial + s0 + q);
    const int64_t r = p.lr_row[lr];
    row_epilogue<STAGE>(p, s, r, 0, t);
    if (STAGE == 2) prep_next(p, r);
  }
}

// Sum of M_off[j] * v[col_j, kk] over j in [j0, j1) for one column per lane:
// the (value, column) pairs are loaded 32 at a time and broadcast by shuffles,
// so each gathered state row is one coalesced 256-byte load; the lane adds in
// CSR order without contraction (the order of a CSR sparse x dense product).
__device__ __forceinline__ double gather_sum(const double* __restrict__ mv, const int* __restrict__ idx,
                                             const double* __restrict__ v, int ld, int kk, int64_t j0,
                                             int64_t j1, int lane) {
  double acc = 0.0;
  for (int64_t base = j0; base < j1; base += 32) {
    const int64_t j = base + lane;
    const double mvl = (j < j1) ? mv[j] : 0.0;
    const int cl = (j < j1) ? idx[j] : 0;
    const int cnt = (int)min((int64_t)32, j1 - base);
#pragma unroll 4
    for (int q = 0; q < cnt; ++q) {
      const double mq = __shfl_sync(0xffffffffu, mvl, q);
      const int cq = __shfl_sync(0xffffffffu, cl, q);
      acc = __dadd_rn(acc, __dmul_rn(mq, v[(size_t)cq * ld + kk]));
    }
  }
  return acc;
}

// Many columns: lane = column inside a 32-column tile (blockIdx.y).  Blocks
// [0, nsb): a warp per short row; blocks [nsb, ...): a warp per long-row segment.
template <int STAGE>
__global__ void __launch_bounds__(256) k_step_multi(StepParams p) {
  const StepScalars s = load_scalars(p, p.step);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int k = blockIdx.y * kColTile + lane;
  const bool active = k < p.ncols;
  const int kk = active ? k : 0;
  const double* __restrict__ v = p.src;
  const double* __restrict__ mv = p.m_vals + (size_t)s.w * p.m_wstride;
  if ((int)blockIdx.x < p.nsb) {
    const int64_t ri = (int64_t)blockIdx.x * (blockDim.x >> 5) + wid;
    if (ri >= p.nrows) return;
    const int64_t r = p.rows[ri];
    const double acc = s.photohad ? gather_sum(mv, p.m_indices, v, p.ld, kk, p.m_indptr[r], p.m_indptr[r + 1], lane)
                                  : 0.0;
    if (active) row_epilogue<STAGE>(p, s, r, k, acc);
    if (STAGE == 2 && blockIdx.y == 0 && lane == 0) prep_next(p, r);
    return;
  }
  const int seg = (blockIdx.x - p.nsb) * (blockDim.x >> 5) + wid;
  if (seg >= p.nseg) return;
  const double acc = s.photohad ? gather_sum(mv, p.m_indices, v, p.ld, kk, p.seg_mb[seg], p.seg_me[seg], lane) : 0.0;
  p.partial[(size_t)seg * p.ld + blockIdx.y * kColTile + lane] = acc;
  const int lr = p.seg_lr[seg];
  if (!last_of_row(p, lr, blockIdx.y, lane)) return;
  const int s0 = p.lr_seg0[lr], ns = p.lr_nseg[lr];
  double t = 0.0;
  for (int q = 0; q < ns; ++q) t = __dadd_rn(t, __ldcg(p.partial + (size_t)(s0 + q) * p.ld + blockIdx.y * kColTile + lane));
  const int64_t r = p.lr_row[lr];
  if (active) row_epilogue<STAGE>(p, s, r, k, t);
  if (STAGE == 2 && blockIdx.y == 0 && lane == 0) prep_next(p, r);
}

// ---------------------------------------------------------------------------
// Bin-blocked batched stage kernels.
//
// States are species blocks of d energy bins.  The coupling rows split in two
// classes (pb_set_layout):
//  * bin-local rows: every M_off entry couples bin e to bin e of another
//    species (boost-conserving fragments).  Their entries are stored
//    bin-major (all rows of bin e contiguous).  k_slab stages the state slab
//    of one bin -- all species x 32 columns -- and the bin's entries in shared
//    memory and sums each row from there, so a state value is read from DRAM
//    once per stage instead of once per coupling entry.
//  * band rows (species with cross-bin entries: the redistributed nucleons):
//    their block rows against each mother species form a band of d x d tiles.
//    k_band multiplies them on the FP64 tensor pipe (DMMA m8n8k4) with the
//    tiles stored in fragment order per window, split over groups of mother
//    species into partial sums that k_band_finish adds in group order.
// The FD loss term D_off (kappa v) couples neighbouring bins of one species;
// k_fd evaluates it species-major (one species block per CTA, in shared
// memory) into fdbuf before the row kernels read it.  A stage is
// k_band (second stream) || k_fd -> k_slab, then k_band_finish.
// ---------------------------------------------------------------------------
constexpr int kFdMax = 4;           // off-diagonal FD stencil entries per row (bin-blocked path)
constexpr int kFdHalo = 3;          // k_fd_dense: stencil offsets within +-kFdHalo bins
constexpr int kFdDenseW = 8;        // dense weights per bin (2 kFdHalo + 1, padded to 16 bytes)
constexpr int kFdChunk = 12;        // k_fd_dense: bins per warp pass
constexpr int kMaxBandGroups = 64;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// mbarrier and bulk-copy helpers of the TMA staging (CTA-local barrier, no cluster)
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
// Wait for phase `phase` of the barrier, giving up after `tries` polls.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned phase, long long tries) {
  for (long long i = 0; i < tries; ++i)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}
// Tiled 3-D tensor load (x = column, y = bin, z = species) into shared memory.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
      ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// Contiguous bulk copy (16-byte aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
constexpr int kErrStagingWait = 1;           // err code: a k_slab CTA's staging wait gave up

// fdbuf = D_off (kappa v) for every row.  CTA = (species block, 32-column
// tile): the block's d x 32 states and its kappa go to shared memory, then a
// thread per (bin, column) adds the stencil terms in CSR order (the stencil of
// bin e is the same in every species block; it is padded to kFdMax terms
// with zero weights on the row itself).
__global__ void __launch_bounds__(256) k_fd(StepParams p) {
  extern __shared__ double fsm[];
  const int sp = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int d = p.d, ld = p.ld;
  const int col = blockIdx.y * kColTile + lane;  // < ld
  double* vb = fsm;                  // d x 32
  double* kb = fsm + d * kColTile;   // d
  double* kpb = kb + d;              // d: kappa_pair of the window (recording only)
  const size_t o0 = (size_t)(p.step & 1) * p.n;
  const double* __restrict__ v = p.src + (size_t)sp * d * ld + blockIdx.y * kColTile;
  for (int t = threadIdx.x; t < d * (kColTile / 2); t += blockDim.x) {
    const int e = t / (kColTile / 2), c = 2 * (t - e * (kColTile / 2));
    cp_async16(vb + e * kColTile + c, v + (size_t)e * ld + c);
  }
  cp_async_commit();
  for (int e = threadIdx.x; e < d; e += blockDim.x) kb[e] = p.kap[o0 + (size_t)sp * d + e];
  const double* kpw = p.fdkp ? p.kp + (size_t)p.win[p.step] * p.n + (size_t)sp * d : nullptr;
  if (kpw)
    for (int e = threadIdx.x; e < d; e += blockDim.x) kpb[e] = kpw[e];
  cp_async_wait<0>();
  __syncthreads();
  for (int e = wid; e < d; e += blockDim.x >> 5) {
    const int* fo = p.fd_off + e * kFdMax;
    const double* fv = p.fd_val + e * kFdMax;
    double sD = __dmul_rn(fv[0], __dmul_rn(kb[e + fo[0]], vb[(e + fo[0]) * kColTile + lane]));
#pragma unroll
    for (int t = 1; t < kFdMax; ++t)
      sD = __dadd_rn(sD, __dmul_rn(fv[t], __dmul_rn(kb[e + fo[t]], vb[(e + fo[t]) * kColTile + lane])));
    p.fdbuf[((size_t)sp * d + e) * ld + col] = sD;
    if (kpw) {  // the photon-scale derivative's FD term, in the order of scale_deriv_apply
      double sK = 0.0;
#pragma unroll
      for (int t = 0; t < kFdMax; ++t) sK += fv[t] * (kpb[e + fo[t]] * vb[(e + fo[t]) * kColTile + lane]);
      p.fdkp[((size_t)sp * d + e) * ld + col] = sK;
    }
  }
}

// fdbuf = D_off (kappa v), register-blocked.  CTA = (species block, 32-column
// tile), lane = column: the block's d x 32 states, its kappa and the dense
// stencil weights go to shared memory; a warp then takes kFdChunk consecutive
// bins, holds kappa x of those bins and kFdHalo neighbours on each side in
// registers (zeros outside the block) and applies the dense stencil in
// ascending offset order.  The zero weights of absent offsets add exact zeros,
// so every row's sum equals the CSR-order sum of k_fd.  KP: the adjoint's
// record pass also needs D_off (kappa_pair v) of the step's window (fdkp).
template <bool KP>
__global__ void __launch_bounds__(256) k_fd_dense(StepParams p) {
  extern __shared__ double fsm[];
  const int sp = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int d = p.d, ld = p.ld;
  const int col = blockIdx.y * kColTile + lane;  // < ld
  double* vb = fsm;                              // d x 32
  double* wt = vb + (size_t)d * kColTile;        // d x kFdDenseW
  double* kb = wt + (size_t)d * kFdDenseW;       // d
  double* kpb = kb + d;                          // d: kappa_pair of the window (KP)
  const size_t o0 = (size_t)(p.step & 1) * p.n + (size_t)sp * d;
  const double* __restrict__ v = p.src + (size_t)sp * d * ld + blockIdx.y * kColTile;
  for (int t = threadIdx.x; t < d * (kColTile / 2); t += blockDim.x) {
    const int e = t / (kColTile / 2), c = 2 * (t - e * (kColTile / 2));
    cp_async16(vb + e * kColTile + c, v + (size_t)e * ld + c);
  }
  for (int t = threadIdx.x; t < d * (kFdDenseW / 2); t += blockDim.x) cp_async16(wt + 2 * t, p.fd_dense + 2 * t);
  cp_async_commit();
  for (int e = threadIdx.x; e < d; e += blockDim.x) kb[e] = p.kap[o0 + e];
  if (KP)
    for (int e = threadIdx.x; e < d; e += blockDim.x) kpb[e] = p.kp[(size_t)p.step_w * p.n + (size_t)sp * d + e];
  cp_async_wait<0>();
  __syncthreads();
  constexpr int U = kFdChunk + 2 * kFdHalo;
  for (int c0 = wid * kFdChunk; c0 < d; c0 += (blockDim.x >> 5) * kFdChunk) {
#pragma unroll 1
    for (int pass = 0; pass < (KP ? 2 : 1); ++pass) {  // pass 1: kappa_pair into fdkp
      const double* kk = pass ? kpb : kb;
      double* __restrict__ out = (pass ? p.fdkp : p.fdbuf) + (size_t)sp * d * ld + col;
      double u[U];
#pragma unroll
      for (int i = 0; i < U; ++i) {
        const int e = c0 - kFdHalo + i;
        u[i] = (e >= 0 && e < d) ? __dmul_rn(kk[e], vb[e * kColTile + lane]) : 0.0;
      }
#pragma unroll
      for (int i = 0; i < kFdChunk; ++i) {
        const int e = c0 + i;
        if (e >= d) break;
        const double2* w2 = reinterpret_cast<const double2*>(wt + e * kFdDenseW);
        const double2 wa = w2[0], wb = w2[1], wc = w2[2], wd = w2[3];
        double sD = __dmul_rn(wa.x, u[i]);
        sD = __dadd_rn(sD, __dmul_rn(wa.y, u[i + 1]));
        sD = __dadd_rn(sD, __dmul_rn(wb.x, u[i + 2]));
        sD = __dadd_rn(sD, __dmul_rn(wb.y, u[i + 3]));
        sD = __dadd_rn(sD, __dmul_rn(wc.x, u[i + 4]));
        sD = __dadd_rn(sD, __dmul_rn(wc.y, u[i + 5]));
        sD = __dadd_rn(sD, __dmul_rn(wd.x, u[i + 6]));
        out[(size_t)e * ld] = sD;
      }
    }
  }
}

// Record pass of the adjoint in the bin-blocked kernels: the photon-scale
// sensitivities P (stage 1) and Q (stage 2) of one (row, column), as record()
// computes them, with the M_off sum sM, the stage result F, the own state
// (x in stage 1) and F(x) (stage 2).
template <int STAGE>
__device__ __forceinline__ void record_blocked(const StepParams& p, const StepScalars& s, int64_t r, int k,
                                               double sM, double F, double own, double fprev) {
  const int64_t j = p.step - p.rec_k0;
  if (j < 0 || j >= p.rec_len) return;
  const size_t o = (size_t)(p.step & 1) * p.n + r;
  const size_t idx = (size_t)r * p.ld + k;
  const size_t ro = (size_t)j * p.n * p.ld + idx;
  const double h = s.h, ds = p.dsig[o];
  double S = s.photohad ? sM : 0.0;
  if (s.kap && s.pair) S += p.fdkp[idx];
  S = S * s.dl * p.inv_scale;
  if (STAGE == 1) {
    p.rec_sx[idx] = S;
    p.rec_P[ro] = p.eD[o] * h * ds * own + h * h * p.dphi1[o] * ds * F + h * p.phi1[o] * S;
  } else {
    p.rec_Q[ro] = h * h * p.dphi2[o] * ds * (F - fprev) + h * p.phi2[o] * (S - p.rec_sx[idx]);
  }
}

// The record inputs of one (row, column), loaded by k_slab with the row's
// other inputs ahead of its sum: the scale derivatives, the step factors, the
// FD term with kappa_pair and (stage 2) the stage-1 S x.
struct RecIn {
  double ds, d12, f0, f1, kp, sx;
  bool on;
};
// record_blocked with preloaded inputs (same arithmetic)
template <int STAGE>
__device__ __forceinline__ void record_pre(const StepParams& p, const StepScalars& s, int64_t r, int k, double sM,
                                           double F, double own, double fprev, const RecIn& in) {
  if (!in.on) return;
  const size_t idx = (size_t)r * p.ld + k;
  const size_t ro = (size_t)(p.step - p.rec_k0) * p.n * p.ld + idx;
  const double h = s.h, ds = in.ds;
  double S = s.photohad ? sM : 0.0;
  if (s.kap && s.pair) S += in.kp;
  S = S * s.dl * p.inv_scale;
  if (STAGE == 1) {
    p.rec_sx[idx] = S;
    p.rec_P[ro] = in.f0 * h * ds * own + h * h * in.d12 * ds * F + h * in.f1 * S;
  } else {
    p.rec_Q[ro] = h * h * in.d12 * ds * (F - fprev) + h * in.f0 * (S - in.sx);
  }
}

// k_slab's shared memory: the state slab of one bin (nsp x 16 columns), the
// bin's entry values (4 per quad), mother-row byte offsets (4 x 16 bits per
// quad), the row quartets of the bin and the row factors (eD, phi1, phi2) of
// each quartet slot.  Every block starts on a 16-byte boundary (the quad count
// of a bin is a multiple of 4).
constexpr int kSlabCols = 16;       // state columns of a k_slab CTA
constexpr int kSlabRows = 4;        // rows per warp: a quarter-warp per row, two columns per lane
constexpr int kSlabWarps = 12;      // two CTAs per SM: 24 warps of 80 registers (loads in flight per warp)
struct SlabSmem {
  double* slab;
  double* vals;
  unsigned long long* sidx;
  int4* quart;
  double* fac;  // [3][kSlabRows maxg]
  unsigned long long* bar;  // the TMA staging barrier
  // species rows of the slab, padded to whole TMA boxes of at most 256 species
  __host__ __device__ static int nbox(int nsp) { return (nsp + 255) / 256; }
  __host__ __device__ static int box_rows(int nsp) { return (nsp + nbox(nsp) - 1) / nbox(nsp); }
  __host__ __device__ static int rows(int nsp) { return nbox(nsp) * box_rows(nsp); }
  __host__ __device__ static size_t bytes(int nsp, int maxq, int maxg) {
    return (size_t)rows(nsp) * kSlabCols * sizeof(double) +
           (size_t)maxq * (4 * sizeof(double) + sizeof(unsigned long long)) +
           (size_t)maxg * (sizeof(int4) + 3 * kSlabRows * sizeof(double)) + sizeof(unsigned long long);
  }
  __device__ SlabSmem(double* base, int nsp, int maxq, int maxg) {
    slab = base;
    vals = slab + (size_t)rows(nsp) * kSlabCols;
    sidx = reinterpret_cast<unsigned long long*>(vals + (size_t)maxq * 4);
    quart = reinterpret_cast<int4*>(sidx + maxq);
    fac = reinterpret_cast<double*>(quart + maxg);
    bar = reinterpret_cast<unsigned long long*>(fac + 3 * kSlabRows * (size_t)maxg);
  }
};

// Species of row g of a quartet descriptor (0xffff: no row).
__device__ __forceinline__ unsigned quart_species(const int4& qd, int g) {
  return ((unsigned)(g < 2 ? qd.x : qd.y) >> (16 * (g & 1))) & 0xffffu;
}
__device__ __forceinline__ double2 dadd2(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
// The injection of one column (rows of injected species only).
__device__ __forceinline__ double slab_inj(const StepParams& p, int slot, int src0, int src1) {
  const double* cf = p.coeff + (size_t)p.step * p.n_src;
  const double* g = p.G + (size_t)slot * p.n_src;
  double a = __dmul_rn(cf[src0], g[src0]);
  for (int q = src0 + 1; q < src1; ++q) a = __dadd_rn(a, __dmul_rn(cf[q], g[q]));
  return a;
}

// Bin-local rows.  CTA = (bin e, 16-column tile); a warp takes four rows at
// a time (a quartet), a quarter-warp per row, and lane j of the quarter owns
// columns col0 + 2j and col0 + 2j + 1.  The state slab of bin e, the bin's
// entry quads, its quartets and their row factors (written in slot order by
// the row preparation) arrive in shared memory by asynchronous copies; a
// warp then walks its quartets (balanced over the warps when the layout is
// built), sums each row from shared memory (four accumulators per column, one
// per quad position, in the row's CSR order) and applies the stage update.
// The four rows' quads interleave, so that one 16-byte value load and one
// offset load serve four rows without bank conflicts, and a slab load of
// 16 bytes per lane serves two columns; a quad's offsets are loaded one quad
// ahead.  The row's FD term (fdbuf), F(x) in stage 2 and its injection slot
// are loaded PREF quartets ahead into registers.  REC: the adjoint's record
// pass (P / Q sensitivities); its row and (row, column) inputs are loaded with
// the others, a quartet less ahead.  Offsets into the (n x ld) state buffers
// are 32-bit (n ld < 2^31, checked at launch).
template <int STAGE, bool REC, int PREF>
__global__ void __launch_bounds__(kSlabWarps * 32, 2) k_slab(StepParams p) {
  extern __shared__ __align__(128) double sm[];  // TMA boxes land at 128-byte boundaries
  const int e = blockIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int g = lane >> 3, j = lane & 7;
  const int col0 = blockIdx.y * kSlabCols;
  const int colA = col0 + 2 * j;  // this lane's columns colA, colA + 1 (< ld)
  const bool actA = colA < p.ncols, actB = colA + 1 < p.ncols;
  const StepScalars s = load_scalars(p, p.step);
  const size_t o0 = (size_t)(p.step & 1) * p.n;
  const int ld = p.ld, d = p.d;
  SlabSmem L(sm, p.nsp, p.slab_maxq, p.slab_maxp);
  const int qb = p.slab_qbase[e], nqb = p.slab_qbase[e + 1] - qb;
  const int gb0 = p.slab_wrp[e * (kSlabWarps + 1)], ngb = p.slab_wrp[e * (kSlabWarps + 1) + kSlabWarps] - gb0;
  const int fs = kSlabRows * p.slab_maxp;  // stride of the three row-factor arrays
  unsigned long long* stage_bar = L.bar;
  const double* mv = p.slab_vals + (size_t)p.step_w * p.slab_stride + (size_t)qb * 4;
  const double* fc = p.slab_fac + (size_t)(p.step & 1) * 3 * p.slab_nslots + (size_t)kSlabRows * gb0;
  if (p.tmap_src) {  // TMA: the slab as tensor boxes, the rest as bulk copies, one barrier
    if (threadIdx.x == 0) mbar_init(stage_bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      const int nb = SlabSmem::nbox(p.nsp), br = SlabSmem::box_rows(p.nsp);
      unsigned bytes = (unsigned)(nb * br * kSlabCols * sizeof(double)) + (unsigned)(ngb * sizeof(int4)) +
                       (unsigned)(3 * kSlabRows * ngb * sizeof(double));
      if (s.photohad) bytes += (unsigned)(nqb * (4 * sizeof(double) + sizeof(unsigned long long)));
      mbar_expect_tx(stage_bar, bytes);
      for (int b = 0; b < nb; ++b) tma_load_3d(L.slab + (size_t)b * br * kSlabCols, p.tmap_src, col0, e, b * br, stage_bar);
      if (s.photohad && nqb > 0) {
        bulk_load(L.vals, mv, (unsigned)(nqb * 4 * sizeof(double)), stage_bar);
        bulk_load(L.sidx, p.slab_q + qb, (unsigned)(nqb * sizeof(unsigned long long)), stage_bar);
      }
      if (ngb > 0) {
        bulk_load(L.quart, p.slab_quart + gb0, (unsigned)(ngb * sizeof(int4)), stage_bar);
        for (int k = 0; k < 3; ++k)
          bulk_load(L.fac + k * fs, fc + (size_t)k * p.slab_nslots, (unsigned)(kSlabRows * ngb * sizeof(double)), stage_bar);
      }
    }
  } else {
    const double* vs = p.src + (size_t)e * ld + col0;
    for (int t = threadIdx.x; t < p.nsp * (kSlabCols / 2); t += blockDim.x) {
      const int q = t / (kSlabCols / 2), cc = 2 * (t - q * (kSlabCols / 2));
      cp_async16(L.slab + q * kSlabCols + cc, vs + (size_t)q * d * ld + cc);
    }
    if (s.photohad) {
      for (int t = threadIdx.x; t < 2 * nqb; t += blockDim.x) cp_async16(L.vals + 2 * t, mv + 2 * t);
      const unsigned long long* mq = p.slab_q + qb;
      for (int t = threadIdx.x; t < nqb / 2; t += blockDim.x) cp_async16(L.sidx + 2 * t, mq + 2 * t);
    }
    for (int t = threadIdx.x; t < ngb; t += blockDim.x) cp_async16(L.quart + t, p.slab_quart + gb0 + t);
    for (int t = threadIdx.x; t < 3 * 2 * ngb; t += blockDim.x) {  // kSlabRows ngb slots per factor, 16 bytes a copy
      const int k = t / (2 * ngb), u = t - k * 2 * ngb;
      cp_async16(L.fac + k * fs + 2 * u, fc + (size_t)k * p.slab_nslots + 2 * u);
    }
    cp_async_commit();
  }
  const int w0 = p.slab_wrp[e * (kSlabWarps + 1) + wid], w1 = p.slab_wrp[e * (kSlabWarps + 1) + wid + 1];
  const bool need_fd = s.kap, need_f = STAGE == 2;
  constexpr int PRE = (REC && PREF > 1) ? PREF - 1 : PREF;  // the record inputs take registers too
  const double2 z2 = make_double2(0.0, 0.0);
  double2 fdr[PRE], fxr[PRE];
  int slr[PRE];
  // record pass: dsigma and phi1' / phi2' of the row, D_off (kappa_pair v) and S x of (row, column)
  const int64_t rj = p.step - p.rec_k0;
  const bool rec_on = REC && rj >= 0 && rj < p.rec_len;
  double rds[PRE], rd12[PRE];
  double2 rkp[PRE], rsx[PRE];
  // the FD term, F(x) and injection slot of quartet pi's row g (staged: the
  // quartet comes from shared memory; the first ones are read from global memory)
#define PB_SLAB_LOAD(U, PI, QD)                                                                          \
  do {                                                                                                   \
    fdr[U] = z2;                                                                                         \
    fxr[U] = z2;                                                                                         \
    slr[U] = -1;                                                                                         \
    if ((PI) < w1) {                                                                                     \
      const unsigned sp_ = quart_species((QD), g);                                                       \
      if (sp_ != 0xffffu) {                                                                              \
        const int r_ = (int)sp_ * d + e;                                                                 \
        if (need_fd) fdr[U] = *reinterpret_cast<const double2*>(p.fdbuf + r_ * ld + colA);               \
        if (need_f) fxr[U] = *reinterpret_cast<const double2*>(p.f + r_ * ld + colA);                    \
        if (s.inj) slr[U] = p.inj_slot[r_];                                                              \
        if (rec_on) {                                                                                    \
          rds[U] = p.dsig[o0 + r_];                                                                      \
          rd12[U] = STAGE == 1 ? p.dphi1[o0 + r_] : p.dphi2[o0 + r_];                                    \
          rkp[U] = (s.kap && s.pair) ? *reinterpret_cast<const double2*>(p.fdkp + r_ * ld + colA) : z2;  \
          rsx[U] = STAGE == 2 ? *reinterpret_cast<const double2*>(p.rec_sx + r_ * ld + colA) : z2;       \
        }                                                                                                \
      }                                                                                                  \
    }                                                                                                    \
  } while (0)
#pragma unroll
  for (int u = 0; u < PRE; ++u) {
    const int pi = w0 + u;
    PB_SLAB_LOAD(u, pi, pi < w1 ? __ldg(p.slab_quart + pi) : make_int4(-1, -1, 0, 0));
  }
  int srcA0 = 0, srcA1 = 0, srcB1 = 0;
  if (s.inj && actA) {
    srcA0 = p.src_ptr[colA];
    srcA1 = p.src_ptr[colA + 1];
    if (actB) srcB1 = p.src_ptr[colA + 2];
  }
  if (p.tmap_src) {
    if (!mbar_wait_bounded(stage_bar, 0, p.wait_tries)) {  // the copies did not land: report and leave
      if (threadIdx.x == 0) atomicExch(p.err, kErrStagingWait);
      mbar_wait_bounded(stage_bar, 0, kWaitTries);
      return;
    }
  } else {
    cp_async_wait<0>();
  }
  __syncthreads();

  const char* slb = reinterpret_cast<const char*>(L.slab + 2 * j);
  const double2* vq = reinterpret_cast<const double2*>(L.vals);
  for (int pb = w0; pb < w1; pb += PRE) {
#pragma unroll
    for (int u = 0; u < PRE; ++u) {
      const int pi = pb + u;
      if (pi >= w1) break;
      const int4 qd = L.quart[pi - gb0];
      const unsigned spw = quart_species(qd, g);
      double2 acc0 = z2, acc1 = z2, acc2 = z2, acc3 = z2;
      if (s.photohad) {  // uniform over the warp: rows without entries walk zero quads
        const int q1 = qd.z + kSlabRows * qd.w;
        unsigned long long mn = qd.w > 0 ? L.sidx[qd.z + g] : 0ull;  // the offsets one quad ahead
#pragma unroll 1
        for (int q = qd.z + g; q < q1; q += kSlabRows) {
          const unsigned long long m = mn;
          if (q + kSlabRows < q1) mn = L.sidx[q + kSlabRows];
          const double2 va = vq[2 * q], vb = vq[2 * q + 1];
          const double2 x0 = *reinterpret_cast<const double2*>(slb + ((unsigned)m & 0xffffu));
          const double2 x1 = *reinterpret_cast<const double2*>(slb + ((unsigned)(m >> 16) & 0xffffu));
          const double2 x2 = *reinterpret_cast<const double2*>(slb + ((unsigned)(m >> 32) & 0xffffu));
          const double2 x3 = *reinterpret_cast<const double2*>(slb + (unsigned)(m >> 48));
          acc0.x = __fma_rn(va.x, x0.x, acc0.x);
          acc0.y = __fma_rn(va.x, x0.y, acc0.y);
          acc1.x = __fma_rn(va.y, x1.x, acc1.x);
          acc1.y = __fma_rn(va.y, x1.y, acc1.y);
          acc2.x = __fma_rn(vb.x, x2.x, acc2.x);
          acc2.y = __fma_rn(vb.x, x2.y, acc2.y);
          acc3.x = __fma_rn(vb.y, x3.x, acc3.x);
          acc3.y = __fma_rn(vb.y, x3.y, acc3.y);
        }
      }
      if (spw != 0xffffu && actA) {
        const int sp = (int)spw;
        const int r = sp * d + e;
        const double2 sM = dadd2(dadd2(acc0, acc1), dadd2(acc2, acc3));
        double2 out = sM;
        if (s.kap) out = dadd2(out, fdr[u]);
        if (s.decay) {
          double2 sL = z2;
          for (int64_t jj = p.l_indptr[r]; jj < p.l_indptr[r + 1]; ++jj) {
            const double lv = p.l_vals[jj];
            const double2 xv = *reinterpret_cast<const double2*>(p.src + (size_t)p.l_indices[jj] * ld + colA);
            sL.x = __dadd_rn(sL.x, __dmul_rn(lv, xv.x));
            sL.y = __dadd_rn(sL.y, __dmul_rn(lv, xv.y));
          }
          out = dadd2(out, sL);
        }
        out.x = __dmul_rn(out.x, s.dl);
        out.y = __dmul_rn(out.y, s.dl);
        if (slr[u] >= 0) {  // injection (rows of injected species only)
          if (srcA1 > srcA0) out.x = __dadd_rn(out.x, __dmul_rn(s.finj, slab_inj(p, slr[u], srcA0, srcA1)));
          if (actB && srcB1 > srcA1) out.y = __dadd_rn(out.y, __dmul_rn(s.finj, slab_inj(p, slr[u], srcA1, srcB1)));
        }
        const double2 own = *reinterpret_cast<const double2*>(L.slab + sp * kSlabCols + 2 * j);
        const int slot = kSlabRows * (pi - gb0) + g;
        const int ro = r * ld + colA;
        if (rec_on) {
          const double f0 = STAGE == 1 ? L.fac[slot] : L.fac[2 * fs + slot], f1 = L.fac[fs + slot];
          record_pre<STAGE>(p, s, r, colA, sM.x, out.x, own.x, fxr[u].x, RecIn{rds[u], rd12[u], f0, f1, rkp[u].x, rsx[u].x, true});
          if (actB)
            record_pre<STAGE>(p, s, r, colA + 1, sM.y, out.y, own.y, fxr[u].y,
                              RecIn{rds[u], rd12[u], f0, f1, rkp[u].y, rsx[u].y, true});
        }
        if (STAGE == 1) {
          // a = eD x + (phi1 F(x)) h
          const double eD = L.fac[slot], p1 = L.fac[fs + slot];
          const double2 av = make_double2(__dadd_rn(__dmul_rn(eD, own.x), __dmul_rn(__dmul_rn(p1, out.x), s.h)),
                                          __dadd_rn(__dmul_rn(eD, own.y), __dmul_rn(__dmul_rn(p1, out.y), s.h)));
          if (actB) {
            *reinterpret_cast<double2*>(p.a + ro) = av;
            *reinterpret_cast<double2*>(p.f + ro) = out;
          } else {
            p.a[ro] = av.x;
            p.f[ro] = out.x;
          }
        } else {
          // x = a + ((F(a) - F(x)) h) phi2
          const double p2 = L.fac[2 * fs + slot];
          const double2 xv = make_double2(__dadd_rn(own.x, __dmul_rn(__dmul_rn(__dadd_rn(out.x, -fxr[u].x), s.h), p2)),
                                          __dadd_rn(own.y, __dmul_rn(__dmul_rn(__dadd_rn(out.y, -fxr[u].y), s.h), p2)));
          if (actB) *reinterpret_cast<double2*>(p.xout + ro) = xv;
          else p.xout[ro] = xv.x;
        }
      }
      const int pn = pi + PRE;
      PB_SLAB_LOAD(u, pn, pn < w1 ? L.quart[pn - gb0] : make_int4(-1, -1, 0, 0));
    }
  }
#undef PB_SLAB_LOAD
}

// k_slab instance for (stage, record pass, prefetch depth in quartets).
using SlabKernel = void (*)(StepParams);
template <int PREF>
SlabKernel slab_kernel_p(int stage, bool rec) {
  if (stage == 1) return rec ? k_slab<1, true, PREF> : k_slab<1, false, PREF>;
  return rec ? k_slab<2, true, PREF> : k_slab<2, false, PREF>;
}
SlabKernel slab_kernel(int stage, bool rec, int pre) {
  switch (pre) {
    case 1: return slab_kernel_p<1>(stage, rec);
    case 3: return slab_kernel_p<3>(stage, rec);
    default: return slab_kernel_p<2>(stage, rec);
  }
}

// Stage 2: the row factors of the next step for the bin-local rows (one
// thread per row; the band rows are prepared by k_band_finish).
__global__ void k_slab_prep(StepParams p) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)p.n_slab_spec * p.d) return;
  const int i = (int)(t / p.d), e = (int)(t - (int64_t)i * p.d);
  prep_next(p, (int64_t)p.slab_spec[i] * p.d + e);
}

// Band partial sums.  CTA = (64-column block, mother-species group, pair of
// band species), 8 warps; warp = one 8-column DMMA tile x both band species
// of the pair x all d rows (accumulators in registers).  Per mother species
// the CTA copies the pair's A tiles (2 x RT x J fragments, fragment order)
// into shared memory with cp.async, double-buffered across species; each warp
// keeps the species' X fragments (2 RT k-tiles of 4 mother bins) in
// registers, loaded one species ahead.  Every tile of the static band is
// multiplied: tiles without coupling entries hold zeros and add exact zeros.
template <int RT, int J, int NW>
__global__ void __launch_bounds__(NW * 32, 1) k_band(StepParams p) {
  extern __shared__ double sm[];
  constexpr int KT = 2 * RT;
  constexpr int ABLK = 2 * RT * J * 32;  // doubles of one (species, band pair) block
  constexpr int AH = RT * J * 32;        // one band species of it
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int c0 = blockIdx.x * (NW * 8) + wid * 8;
  const bool wact = c0 < p.ncols;  // c0 + 7 < ld: ld is a multiple of 32
  const int pair = blockIdx.z, g = blockIdx.y;
  const int s0 = g * p.spg, s1 = min(p.nsp, s0 + p.spg);
  const int d = p.d, ld = p.ld;
  const int w = p.win[p.step];
  const double* __restrict__ A = p.band_vals + (size_t)w * p.band_stride;
  const int npairs = gridDim.z;
  double* As = sm;  // [2][ABLK]
  auto issue = [&](int sp, int stage) {
    const double* src = A + ((size_t)sp * npairs + pair) * ABLK;
    for (int c = threadIdx.x; c < ABLK / 2; c += blockDim.x) cp_async16(As + stage * ABLK + 2 * c, src + 2 * c);
    cp_async_commit();
  };
  double acc[2][RT][2];
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int rt = 0; rt < RT; ++rt) acc[b][rt][0] = acc[b][rt][1] = 0.0;
  const int kr = lane & 3;
  double xf[KT], xn[KT];
  auto load_x = [&](int sp, double (&x)[KT]) {
    const double* __restrict__ xs = p.src + (size_t)sp * d * ld + c0 + (lane >> 2);
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
      const int e = 4 * kt + kr;
      x[kt] = (wact && e < d) ? xs[(size_t)e * ld] : 0.0;
    }
  };
  if (NW == 8) {  // whole (species, pair) blocks, double-buffered
    if (s0 < s1) {
      issue(s0, 0);
      load_x(s0, xf);
    }
    for (int sp = s0; sp < s1; ++sp) {
      const int stage = (sp - s0) & 1;
      if (sp + 1 < s1) {
        issue(sp + 1, stage ^ 1);
        load_x(sp + 1, xn);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
      // a lane's fragments of row tiles 2p and 2p + 1 are one 16-byte word
      const double2* __restrict__ as = reinterpret_cast<const double2*>(As + stage * ABLK) + lane;
      // consecutive DMMAs go to different accumulators (k-tile outer, row tile inner)
#pragma unroll
      for (int jj = 0; jj < J; ++jj)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int rp = 0; rp < RT / 2; ++rp) {
            const int kt = 4 * rp + jj;
            if (kt >= KT) continue;
            const double2 a2 = as[((b * (RT / 2) + rp) * J + jj) * 32];
            dmma884(acc[b][2 * rp][0], acc[b][2 * rp][1], a2.x, xf[kt]);
            if (kt + 2 < KT) dmma884(acc[b][2 * rp + 1][0], acc[b][2 * rp + 1][1], a2.y, xf[kt + 2]);
          }
      __syncthreads();  // every warp is done with this stage before it is refilled
#pragma unroll
      for (int kt = 0; kt < KT; ++kt) xf[kt] = xn[kt];
    }
  } else {  // one band species at a time through a ring of two half blocks (half the shared memory)
    auto issue_h = [&](int sp, int b, int buf) {
      const double* src = A + ((size_t)sp * npairs + pair) * ABLK + (size_t)b * AH;
      for (int c = threadIdx.x; c < AH / 2; c += blockDim.x) cp_async16(As + buf * AH + 2 * c, src + 2 * c);
      cp_async_commit();
    };
    int buf = 0;
    if (s0 < s1) {
      issue_h(s0, 0, 0);
      load_x(s0, xf);
    }
    for (int sp = s0; sp < s1; ++sp) {
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const bool more = b == 0 || sp + 1 < s1;
        if (more) {
          issue_h(b == 0 ? sp : sp + 1, b ^ 1, buf ^ 1);
          if (b == 0 && sp + 1 < s1) load_x(sp + 1, xn);
          cp_async_wait<1>();
        } else {
          cp_async_wait<0>();
        }
        __syncthreads();
        const double2* __restrict__ as = reinterpret_cast<const double2*>(As + buf * AH) + lane;
#pragma unroll
        for (int jj = 0; jj < J; ++jj)
#pragma unroll
          for (int rp = 0; rp < RT / 2; ++rp) {
            const int kt = 4 * rp + jj;
            if (kt >= KT) continue;
            const double2 a2 = as[(rp * J + jj) * 32];
            dmma884(acc[b][2 * rp][0], acc[b][2 * rp][1], a2.x, xf[kt]);
            if (kt + 2 < KT) dmma884(acc[b][2 * rp + 1][0], acc[b][2 * rp + 1][1], a2.y, xf[kt + 2]);
          }
        __syncthreads();  // every warp is done with this half before it is refilled
        buf ^= 1;
      }
#pragma unroll
      for (int kt = 0; kt < KT; ++kt) xf[kt] = xn[kt];
    }
  }
  if (!wact) return;
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    if (2 * pair + b >= p.nb) continue;
    double* __restrict__ P = p.band_part + (size_t)(g * p.nb + 2 * pair + b) * d * ld;
#pragma unroll
    for (int rt = 0; rt < RT; ++rt) {
      const int row = 8 * rt + (lane >> 2);
      if (row >= d) continue;
      double2 o;
      o.x = acc[b][rt][0];
      o.y = acc[b][rt][1];
      *reinterpret_cast<double2*>(P + (size_t)row * ld + c0 + kr * 2) = o;
    }
  }
}

template <int RT, int J, int NW>
size_t band_smem_bytes() {
  return (size_t)2 * ((NW == 8 ? 2 : 1) * RT * J * 32) * sizeof(double);
}

// Band rows: add the group partials in group order, then the stage update
// with the FD term from fdbuf.
template <int STAGE>
__global__ void __launch_bounds__(256) k_band_finish(StepParams p) {
  const StepScalars s = load_scalars(p, p.step);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int rb = blockIdx.x * (blockDim.x >> 5) + wid;
  if (rb >= p.nb * p.d) return;
  const int b = rb / p.d, e = rb - b * p.d;
  const int64_t r = (int64_t)p.band_spec[b] * p.d + e;
  const int col = blockIdx.y * kColTile + lane;
  if (col < p.ncols) {
    double t = 0.0;
    for (int g = 0; g < p.ngroups; ++g)
      t = __dadd_rn(t, p.band_part[((size_t)(g * p.nb + b) * p.d + e) * p.ld + col]);
    const size_t idx = (size_t)r * p.ld + col;
    double out = t;
    if (s.kap) out = __dadd_rn(out, p.fdbuf[idx]);
    if (s.decay) {
      double sL = 0.0;
      for (int64_t j = p.l_indptr[r]; j < p.l_indptr[r + 1]; ++j)
        sL = __dadd_rn(sL, __dmul_rn(p.l_vals[j], p.src[(size_t)p.l_indices[j] * p.ld + col]));
      out = __dadd_rn(out, sL);
    }
    out = __dmul_rn(out, s.dl);
    if (s.inj) out = __dadd_rn(out, inj_at(p, s, r, col));
    const size_t o = (size_t)(p.step & 1) * p.n + r;
    if (p.rec_P) record_blocked<STAGE>(p, s, r, col, t, out, p.x[idx], STAGE == 2 ? p.f[idx] : 0.0);
    if (STAGE == 1) {
      p.a[idx] = __dadd_rn(__dmul_rn(p.eD[o], p.x[idx]), __dmul_rn(__dmul_rn(p.phi1[o], out), s.h));
      p.f[idx] = out;
    } else {
      const double dF = __dmul_rn(__dadd_rn(out, -p.f[idx]), s.h);
      p.xout[idx] = __dadd_rn(p.a[idx], __dmul_rn(dF, p.phi2[o]));
    }
  }
  if (STAGE == 2 && blockIdx.y == 0 && lane == 0) prep_next(p, r);
}

// Band partial sums with TMA staging (8 warps; the same tiles and arithmetic
// as k_band).  Per mother species one thread issues the pair's A tiles as one
// bulk copy (double-buffered) and the species' X block (d bins x 64 columns)
// as one tensor-map box; each warp reads its X fragments from shared memory,
// so no register copy of the next species is held.  One CTA barrier per
// species; every mbarrier wait is bounded: a CTA that gives up sets p.err,
// stops issuing, waits (bounded) for the copies it issued and leaves.
constexpr int kErrBandWait = 2;  // err code: a k_band CTA's staging wait gave up
template <int RT, int J>
__global__ void __launch_bounds__(256, 1) k_band_tma(StepParams p) {
  extern __shared__ __align__(128) double sm[];
  constexpr int KT = 2 * RT;
  constexpr int ABLK = 2 * RT * J * 32;  // doubles of one (species, band pair) block
  constexpr int XS = 8 * RT * 64;        // X of one species: bins x 64 columns
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int cb = blockIdx.x * 64, c0 = cb + wid * 8;
  const bool wact = c0 < p.ncols;  // c0 + 7 < ld: ld is a multiple of 32
  const int pair = blockIdx.z, g = blockIdx.y;
  const int s0 = g * p.spg, s1 = min(p.nsp, s0 + p.spg);
  const int d = p.d, ld = p.ld;
  const int w = p.win[p.step];
  const double* __restrict__ A = p.band_vals + (size_t)w * p.band_stride;
  const int npairs = gridDim.z;
  double* As = sm;             // [2][ABLK]
  double* Xs = As + 2 * ABLK;  // [bin][64 columns]
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(Xs + XS);  // A stage 0, A stage 1, X
  int* abort_s = reinterpret_cast<int*>(bar + 3);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    mbar_init(bar + 2, 1);
    *abort_s = 0;
  }
  __syncthreads();
  auto issue = [&](int sp, int stage) {  // thread 0
    mbar_expect_tx(bar + stage, (unsigned)(ABLK * sizeof(double)));
    bulk_load(As + stage * ABLK, A + ((size_t)sp * npairs + pair) * ABLK, (unsigned)(ABLK * sizeof(double)), bar + stage);
    mbar_expect_tx(bar + 2, (unsigned)(64 * d * sizeof(double)));
    tma_load_3d(Xs, p.tmap_band, cb, 0, sp, bar + 2);
  };
  if (threadIdx.x == 0 && s0 < s1) issue(s0, 0);
  double acc[2][RT][2];
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int rt = 0; rt < RT; ++rt) acc[b][rt][0] = acc[b][rt][1] = 0.0;
  const int kr = lane & 3;
  int last = s0 - 1;  // the last species whose copies were issued (thread 0)
  if (s0 < s1) last = s0;
  for (int sp = s0; sp < s1; ++sp) {
    const int it = sp - s0, stage = it & 1;
    bool ok = mbar_wait_bounded(bar + 2, (unsigned)(it & 1), p.wait_tries);
    double xf[KT];
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
      const int e = 4 * kt + kr;
      xf[kt] = (wact && e < d) ? Xs[e * 64 + wid * 8 + (lane >> 2)] : 0.0;
    }
    ok = mbar_wait_bounded(bar + stage, (unsigned)((it >> 1) & 1), p.wait_tries) && ok;
    if (!ok) {
      atomicExch(p.err, kErrBandWait);
      *abort_s = 1;
    }
    __syncthreads();  // every warp holds X(sp) and is done with A(sp - 1)
    if (*abort_s) break;
    if (threadIdx.x == 0 && sp + 1 < s1) {
      issue(sp + 1, stage ^ 1);
      last = sp + 1;
    }
    // a lane's fragments of row tiles 2p and 2p + 1 are one 16-byte word
    const double2* __restrict__ as = reinterpret_cast<const double2*>(As + stage * ABLK) + lane;
#pragma unroll
    for (int jj = 0; jj < J; ++jj)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int rp = 0; rp < RT / 2; ++rp) {
          const int kt = 4 * rp + jj;
          if (kt >= KT) continue;
          const double2 a2 = as[((b * (RT / 2) + rp) * J + jj) * 32];
          dmma884(acc[b][2 * rp][0], acc[b][2 * rp][1], a2.x, xf[kt]);
          if (kt + 2 < KT) dmma884(acc[b][2 * rp + 1][0], acc[b][2 * rp + 1][1], a2.y, xf[kt + 2]);
        }
  }
  if (*abort_s) {  // the copies this CTA issued land before it leaves
    if (threadIdx.x == 0 && last >= s0) {
      const int it = last - s0;
      mbar_wait_bounded(bar + 2, (unsigned)(it & 1), kWaitTries);
      mbar_wait_bounded(bar + (it & 1), (unsigned)((it >> 1) & 1), kWaitTries);
    }
    return;
  }
  if (!wact) return;
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    if (2 * pair + b >= p.nb) continue;
    double* __restrict__ P = p.band_part + (size_t)(g * p.nb + 2 * pair + b) * d * ld;
#pragma unroll
    for (int rt = 0; rt < RT; ++rt) {
      const int row = 8 * rt + (lane >> 2);
      if (row >= d) continue;
      double2 o;
      o.x = acc[b][rt][0];
      o.y = acc[b][rt][1];
      *reinterpret_cast<double2*>(P + (size_t)row * ld + c0 + kr * 2) = o;
    }
  }
}

template <int RT, int J>
size_t band_tma_smem_bytes() {
  return (size_t)(2 * 2 * RT * J * 32 + 8 * RT * 64) * sizeof(double) + 4 * sizeof(unsigned long long);
}

// Instances of k_band: row tiles RT (d <= 8 RT) x k-tiles per row tile J
// (band offsets up to 4 J - 8 bins).
using BandKernel = void (*)(StepParams);
constexpr int kBandRT[] = {4, 8, 12, 16};
constexpr int kBandJ[] = {5, 9, 13, 17};
struct BandInstance {
  BandKernel fn;
  size_t smem;
  int warps;
};
template <int RT, int NW>
BandInstance band_kernel_j(int J) {
  switch (J) {
    case 5: return {k_band<RT, 5, NW>, band_smem_bytes<RT, 5, NW>(), NW};
    case 9: return {k_band<RT, 9, NW>, band_smem_bytes<RT, 9, NW>(), NW};
    case 13: return {k_band<RT, 13, NW>, band_smem_bytes<RT, 13, NW>(), NW};
    case 17: return {k_band<RT, 17, NW>, band_smem_bytes<RT, 17, NW>(), NW};
  }
  return {nullptr, 0, 0};
}
template <int NW>
BandInstance band_kernel_w(int RT, int J) {
  switch (RT) {
    case 4: return band_kernel_j<4, NW>(J);
    case 8: return band_kernel_j<8, NW>(J);
    case 12: return band_kernel_j<12, NW>(J);
    case 16: return band_kernel_j<16, NW>(J);
  }
  return {nullptr, 0, 0};
}
// nw = 8: 64-column CTAs (one per SM); nw = 4: 32-column CTAs in half the
// registers and shared memory, so that a k_slab CTA fits beside one.
BandInstance band_kernel(int RT, int J, int nw = 8) {
  return nw == 4 ? band_kernel_w<4>(RT, J) : band_kernel_w<8>(RT, J);
}
// The TMA-staged 8-warp instance.
template <int RT>
BandInstance band_kernel_tma_j(int J) {
  switch (J) {
    case 5: return {k_band_tma<RT, 5>, band_tma_smem_bytes<RT, 5>(), 8};
    case 9: return {k_band_tma<RT, 9>, band_tma_smem_bytes<RT, 9>(), 8};
    case 13: return {k_band_tma<RT, 13>, band_tma_smem_bytes<RT, 13>(), 8};
    case 17: return {k_band_tma<RT, 17>, band_tma_smem_bytes<RT, 17>(), 8};
  }
  return {nullptr, 0, 0};
}
BandInstance band_kernel_tma(int RT, int J) {
  switch (RT) {
    case 4: return band_kernel_tma_j<4>(J);
    case 8: return band_kernel_tma_j<8>(J);
    case 12: return band_kernel_tma_j<12>(J);
    case 16: return band_kernel_tma_j<16>(J);
  }
  return {nullptr, 0, 0};
}

// ---------------------------------------------------------------------------
// Co-evolved EM cascade, applied after every ETD2 step (propagation.py:555-665):
//   w      = sum over charged nuclei s of (A_s kappa_pair_s dl_step / E dE) n_s   (per nucleon bin)
//   e_src  = R_BH(z_w) w                     added to e- and e+
//   gamma <- T_gamma gamma + T_electron (e- + e+),   e+- <- 0
// The pair weights by k_em_w, the products as batched DMMA GEMMs (em_hook_forward).
// ---------------------------------------------------------------------------
}  // namespace

// batched FP64 GEMM on the tensor pipe and the cascade-transfer kernels
#include "em_transfer.cuh"

namespace {

struct EmParams {
  int64_t n;
  int ld;
  int ncols;
  int n_em, n_cr, n_bh;
  int64_t g_off, em_off, ep_off;  // block offsets of gamma, e-, e+ (e+- may be -1)
  const int64_t* bh_off;          // block offset of each charged nucleus
  const double* bh_A;
  const double* invE;             // 1 / E on the nucleon grid
  const double* dE;               // gradient of E
  const double* kp;               // kappa_pair of the window (n)
  double dl_step;
  const double* Tg;               // n_em x n_em
  const double* Te;               // n_em x n_em
  const double* R;                // n_em x n_cr
  double* X;
  double* w;                      // n_cr x ld: Bethe-Heitler pair weights (forward) or their adjoint
  double* es;                     // n_em x ld: R w (forward) or Te^T lam_gamma (adjoint)
  double* lep;                    // n_em x ld: e- + e+ with the pairs (forward)
  double* y;                      // n_em x ld: the new gamma rows (forward) or Tg^T lam_gamma (adjoint)
  const double* TgT;              // transposes of the window's matrices (adjoint)
  const double* TeT;
  const double* RT;               // n_cr x n_em
};

// l = (e- + es) + (e+ + es) with es = R w, then e+- <- 0 (the lepton half of the hook).
__global__ void k_em_lep(EmParams e) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)e.n_em * e.ncols) return;
  const int j = (int)(t / e.ncols), k = (int)(t % e.ncols);
  const double es = e.es[(size_t)j * e.ld + k];
  double l = 0.0;
  if (e.em_off >= 0) {
    double* x = e.X + (size_t)(e.em_off + j) * e.ld + k;
    l = __dadd_rn(l, __dadd_rn(*x, es));
    *x = 0.0;
  }
  if (e.ep_off >= 0) {
    double* x = e.X + (size_t)(e.ep_off + j) * e.ld + k;
    l = __dadd_rn(l, __dadd_rn(*x, es));
    *x = 0.0;
  }
  e.lep[(size_t)j * e.ld + k] = l;
}

// Adjoint lepton rows: lam_e+- <- Te^T lam_gamma (e.es), and lw = n_lep R^T (that) is a GEMM after.
__global__ void k_em_lepT(EmParams e) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)e.n_em * e.ncols) return;
  const int j = (int)(t / e.ncols), k = (int)(t % e.ncols);
  const double m = e.es[(size_t)j * e.ld + k];
  if (e.em_off >= 0) e.X[(size_t)(e.em_off + j) * e.ld + k] = m;
  if (e.ep_off >= 0) e.X[(size_t)(e.ep_off + j) * e.ld + k] = m;
}

// Scales the first n_cr x ncols block of e.w by s (the lepton count of the adjoint pair weights).
__global__ void k_em_scale_w(EmParams e, double s) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)e.n_cr * e.ncols) return;
  const int i = (int)(t / e.ncols), k = (int)(t % e.ncols);
  e.w[(size_t)i * e.ld + k] *= s;
}


// w[i][k] = sum_s cw_si X[s, i][k] over the charged nuclei in species order, with
// cw_si = A_s kappa_pair dl_step / E_i dE_i: the Bethe-Heitler pair weights of the
// hook (propagation.py:640-661).  A warp per (bin, 32 V-column tile), each lane
// V adjacent columns (V = 2: 16-byte loads, used when the leading dimension is
// even; V = 1 for one-column solves, whose leading dimension is 1), so the
// nuclear state is read by many warps at once; the species table sits in
// shared memory and each warp loads kEmWBatch species' states ahead of the
// (ordered) sum.
constexpr int kEmWBatch = 8;

template <int V>
__global__ void __launch_bounds__(256, 3) k_em_w(EmParams e) {
  extern __shared__ unsigned char em_w_smem[];
  int64_t* soff = reinterpret_cast<int64_t*>(em_w_smem);
  double* sA = reinterpret_cast<double*>(soff + e.n_bh);
  for (int t = threadIdx.x; t < e.n_bh; t += blockDim.x) {
    soff[t] = e.bh_off[t];
    sA[t] = e.bh_A[t];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int i = blockIdx.x * 8 + wid;
  if (i >= e.n_cr) return;
  const int k = blockIdx.y * (32 * V) + V * lane;  // columns k .. k + V - 1
  const bool active = k < e.ncols;
  const int kk = active ? k : 0;
  const double ie = e.invE[i], de = e.dE[i];
  double acc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = 0.0;
  for (int s0 = 0; s0 < e.n_bh; s0 += kEmWBatch) {
    double xv[kEmWBatch][V];
    double kv[kEmWBatch];
#pragma unroll
    for (int u = 0; u < kEmWBatch; ++u) {
#pragma unroll
      for (int v = 0; v < V; ++v) xv[u][v] = 0.0;
      kv[u] = 0.0;
      if (s0 + u < e.n_bh) {
        const int64_t row = soff[s0 + u] + i;
        const double* src = e.X + (size_t)row * e.ld + kk;
        if (V == 2) {
          const double2 x2 = __ldg(reinterpret_cast<const double2*>(src));
          xv[u][0] = x2.x;
          xv[u][V - 1] = x2.y;
        } else {
          xv[u][0] = __ldg(src);
        }
        kv[u] = __ldg(e.kp + row);
      }
    }
#pragma unroll
    for (int u = 0; u < kEmWBatch; ++u) {
      const int s = s0 + u;
      if (s < e.n_bh) {
        const double cw = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(sA[s], kv[u]), e.dl_step), ie), de);
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const double t = __dmul_rn(cw, xv[u][v]);
          acc[v] = (s == 0) ? t : __dadd_rn(acc[v], t);
        }
      }
    }
  }
#pragma unroll
  for (int v = 0; v < V; ++v)
    if (k + v < e.ncols) e.w[(size_t)i * e.ld + k + v] = acc[v];
}

// Adjoint of the pair weights: X[s, i][k] += cw_si lw[i][k] (e.X = lam, e.w = lw).
__global__ void __launch_bounds__(256) k_em_wT(EmParams e) {
  extern __shared__ unsigned char em_w_smem[];
  int64_t* soff = reinterpret_cast<int64_t*>(em_w_smem);
  double* sA = reinterpret_cast<double*>(soff + e.n_bh);
  for (int t = threadIdx.x; t < e.n_bh; t += blockDim.x) {
    soff[t] = e.bh_off[t];
    sA[t] = e.bh_A[t];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int i = blockIdx.x * 8 + wid;
  if (i >= e.n_cr) return;
  const int k = blockIdx.y * 32 + lane;
  if (k >= e.ncols) return;
  const double l = e.w[(size_t)i * e.ld + k] * e.dl_step * e.invE[i] * e.dE[i];
  for (int s0 = 0; s0 < e.n_bh; s0 += kEmWBatch) {
    double xv[kEmWBatch], kv[kEmWBatch];
#pragma unroll
    for (int u = 0; u < kEmWBatch; ++u)
      if (s0 + u < e.n_bh) {
        const int64_t row = soff[s0 + u] + i;
        xv[u] = e.X[(size_t)row * e.ld + k];
        kv[u] = __ldg(e.kp + row);
      }
#pragma unroll
    for (int u = 0; u < kEmWBatch; ++u)
      if (s0 + u < e.n_bh) {
        const int64_t row = soff[s0 + u] + i;
        e.X[(size_t)row * e.ld + k] = xv[u] + sA[s0 + u] * kv[u] * l;
      }
  }
}

// The hook after a step, on the tensor pipe where it is dense (propagation.py:555-571, 620-665):
//   w = pair weights (k_em_w), es = R w, l = e- + e+ + 2 es (k_em_lep, e+- <- 0),
//   y = Tg gamma + Te l, gamma <- y.
void em_hook_forward(const EmParams& e, cudaStream_t st) {
  const size_t wsm = (size_t)e.n_bh * (sizeof(int64_t) + sizeof(double));
  if (e.ld % 2 == 0)
    k_em_w<2><<<dim3((unsigned)blocks_for(e.n_cr, 8), (unsigned)blocks_for(e.ncols, 64)), 256, wsm, st>>>(e);
  else
    k_em_w<1><<<dim3((unsigned)blocks_for(e.n_cr, 8), (unsigned)blocks_for(e.ncols, 32)), 256, wsm, st>>>(e);
  bgemm(st, e.R, e.w, e.es, e.n_em, e.ncols, e.n_cr, e.n_cr, e.ld, e.ld, 0, 0, 0, 1, false);
  k_em_lep<<<(unsigned)blocks_for((int64_t)e.n_em * e.ncols, 256), 256, 0, st>>>(e);
  double* gam = e.X + (size_t)e.g_off * e.ld;
  bgemm(st, e.Tg, gam, e.y, e.n_em, e.ncols, e.n_em, e.n_em, e.ld, e.ld, 0, 0, 0, 1, false);
  bgemm(st, e.Te, e.lep, e.y, e.n_em, e.ncols, e.n_em, e.n_em, e.ld, e.ld, 0, 0, 0, 1, true);
  cudaMemcpy2DAsync(gam, (size_t)e.ld * sizeof(double), e.y, (size_t)e.ld * sizeof(double),
                    (size_t)e.ncols * sizeof(double), (size_t)e.n_em, cudaMemcpyDeviceToDevice, st);
}

// Its transpose on lam (e.X): mu = Te^T lam_gamma, lam_gamma <- Tg^T lam_gamma,
// lam_e+- <- mu, lam_nuclei += cw (n_lep R^T mu) (k_em_wT).
void em_hook_adjoint(const EmParams& e, cudaStream_t st) {
  double* gam = e.X + (size_t)e.g_off * e.ld;
  bgemm(st, e.TeT, gam, e.es, e.n_em, e.ncols, e.n_em, e.n_em, e.ld, e.ld, 0, 0, 0, 1, false);
  bgemm(st, e.TgT, gam, e.y, e.n_em, e.ncols, e.n_em, e.n_em, e.ld, e.ld, 0, 0, 0, 1, false);
  cudaMemcpy2DAsync(gam, (size_t)e.ld * sizeof(double), e.y, (size_t)e.ld * sizeof(double),
                    (size_t)e.ncols * sizeof(double), (size_t)e.n_em, cudaMemcpyDeviceToDevice, st);
  k_em_lepT<<<(unsigned)blocks_for((int64_t)e.n_em * e.ncols, 256), 256, 0, st>>>(e);
  bgemm(st, e.RT, e.es, e.w, e.n_cr, e.ncols, e.n_em, e.n_em, e.ld, e.ld, 0, 0, 0, 1, false);
  const double nl = (double)((e.em_off >= 0) + (e.ep_off >= 0));
  if (nl != 1.0)
    k_em_scale_w<<<(unsigned)blocks_for((int64_t)e.n_cr * e.ncols, 256), 256, 0, st>>>(e, nl);
  const size_t wsm = (size_t)e.n_bh * (sizeof(int64_t) + sizeof(double));
  k_em_wT<<<dim3((unsigned)blocks_for(e.n_cr, 8), (unsigned)blocks_for(e.ncols, 32)), 256, wsm, st>>>(e);
}



// ---------------------------------------------------------------------------
// Bin-blocked adjoint sweep.  One backward step applies A^T twice (stage 1 to
// v1 = Phi2 lam', stage 2 to v2 = Phi1 mu - Phi2 lam'), with
//   A^T v = dl (M_off^T v + diag(kappa) D_off^T v + Lambda_off^T v).
// M_off^T v splits like the forward product:
//  * band part: for every mother species s, out_s = sum_N B_{N,s}^T v_N over
//    the band species N -- k_bandT on DMMA with the transposed tiles; the v_N
//    fragments stay in registers for all mother species, so no reduction
//    across species is needed (written to bT);
//  * bin-local part: mother rows gather from the daughters of the same bin --
//    k_slabT with the entries in bin-major, mother-grouped order.
// D_off^T v is k_fdT (species-major, transposed per-bin stencil).  k_slabT's
// epilogue combines the parts and applies the stage update of the adjoint
// step; it also writes the next v (v2 after stage 1; after stage 2, v1 of the
// previous step when its factors are recorded).
// ---------------------------------------------------------------------------
constexpr int kFdTMax = 6;          // entries of a column of the FD operator's off-diagonal block

struct AdjBlk {
  int64_t n;
  int d, nsp, ld, ncols, w, nb, spg;
  int64_t step;
  uint32_t flags;
  double h, dl;
  const double* v;          // the vector A^T is applied to (n x ld)
  double* bT;               // n x ld: band part of M_off^T v
  double* fdT;              // n x ld: D_off^T v
  const double* bandT;      // [W][band_stride] transposed band tiles
  int64_t band_stride;
  const double* slabT;      // [W][slabT_stride] bin-local entries by mother row, in quads (zero padding)
  int64_t slabT_stride;
  const int* slabT_qbase;   // [d + 1] first quad of each bin (even)
  const unsigned long long* slabT_q;  // per quad: byte offsets of the 4 daughters' rows in the v slab, 16 bits each
  const int4* slabT_pairs;  // mother-row pairs of k_slabT's warps: species A, B (-1: none), q0 << 16 | quads of A, of B
  const int* slabT_wrp;     // [d][kSlabTWarps + 1] first pair of each warp of a bin's CTA
  int slabT_maxq;           // quads of the largest bin
  int slabT_maxp;           // row pairs of a bin
  const int* fdT_cnt;       // per bin: entries of the transposed stencil, row offsets, values
  const int* fdT_off;
  const double* fdT_val;
  const double* fdT_dense;  // [d][kFdDenseW] transposed weights of offsets -kFdHalo..kFdHalo, or null
  const int* band_spec;
  const double* rf;         // recorded eD, phi1, phi2, kappa of this step (n each)
  const double* rf_prev;    // recorded factors of the previous step (phi2 used), or null
  const double* lam;        // dL/dx'
  double* mu;               // dL/da
  double* lam_out;          // dL/dx
  double* vout;             // stage 1: v2; stage 2: v1 of the previous step (if rf_prev)
  const double* P;          // recorded sensitivities of this step, or null
  const double* Q;
  double* gs;               // d x ld: photon-scale gradient, summed over the rows of each bin
  const CUtensorMap* tmap_v;  // k_slabT: tensor map of v for the TMA staging, or null (cp.async staging)
  int* err;                 // k_slabT: set when its staging wait gives up
  long long wait_tries;     // k_slabT: polls of the staging wait
  const int* inj_slot;
  double* gb_inj;
  const int64_t* lt_indptr; // Lambda_off^T, or null
  const int* lt_indices;
  const double* lt_vals;
};

// Y[rows[r]][cols[j]] = X[r][j]: the state in the caller's row and column order
// (a null map is the identity; Y is n x K)
__global__ void k_gather_cols(const double* __restrict__ X, int ld, int64_t n, int K, const int* __restrict__ cols,
                              const int* __restrict__ rows, double* __restrict__ Y) {
  const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int j = blockIdx.y * kColTile + (threadIdx.x & 31);
  if (r >= n || j >= K) return;
  const int64_t ro = rows ? rows[r] : r;
  Y[(size_t)ro * K + (cols ? cols[j] : j)] = X[(size_t)r * ld + j];
}

// lam[r][j] = S[rows[r]][cols[j]]: a state or seed given in the caller's row and
// column order, in solve order (S is n x K; a null map is the identity)
__global__ void k_pick_cols(const double* __restrict__ S, int64_t n, int K, const int* __restrict__ cols,
                            const int* __restrict__ rows, double* __restrict__ lam, int ld) {
  const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int j = blockIdx.y * kColTile + (threadIdx.x & 31);
  if (r >= n || j >= K) return;
  const int64_t ro = rows ? rows[r] : r;
  lam[(size_t)r * ld + j] = S[(size_t)ro * K + (cols ? cols[j] : j)];
}

// v1 = Phi2 lam' for the last step of a checkpoint segment
__global__ void k_adj_v1(const double* __restrict__ phi2, const double* __restrict__ lam, int64_t n, int ld,
                         int ncols, double* __restrict__ v) {
  const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int k = blockIdx.y * kColTile + (threadIdx.x & 31);
  if (r >= n || k >= ncols) return;
  const size_t i = (size_t)r * ld + k;
  v[i] = phi2[r] * lam[i];
}

// fdT = D_off^T v, species-major (the block of d x 32 states in shared memory).
__global__ void __launch_bounds__(256) k_fdT(AdjBlk q) {
  extern __shared__ double fsm[];
  const int sp = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int d = q.d, ld = q.ld;
  const int col = blockIdx.y * kColTile + lane;
  const double* __restrict__ v = q.v + (size_t)sp * d * ld + blockIdx.y * kColTile;
  for (int t = threadIdx.x; t < d * (kColTile / 2); t += blockDim.x) {
    const int e = t / (kColTile / 2), c = 2 * (t - e * (kColTile / 2));
    cp_async16(fsm + e * kColTile + c, v + (size_t)e * ld + c);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  for (int e = wid; e < d; e += blockDim.x >> 5) {
    const int cnt = q.fdT_cnt[e];
    double s = 0.0;
    for (int t = 0; t < cnt; ++t)
      s += q.fdT_val[e * kFdTMax + t] * fsm[(e + q.fdT_off[e * kFdTMax + t]) * kColTile + lane];
    q.fdT[((size_t)sp * d + e) * ld + col] = s;
  }
}

// fdT = D_off^T v, register-blocked like k_fd_dense (no kappa): the block's
// d x 32 states and the dense transposed weights in shared memory, a warp
// holds kFdChunk bins plus a kFdHalo halo per side in registers.  The terms
// are fused multiply-adds in ascending offset order from zero, so absent
// offsets (zero weights) leave each sum as k_fdT forms it.
__global__ void __launch_bounds__(256) k_fdT_dense(AdjBlk q) {
  extern __shared__ double fsm[];
  const int sp = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int d = q.d, ld = q.ld;
  const int col = blockIdx.y * kColTile + lane;
  double* vb = fsm;                        // d x 32
  double* wt = vb + (size_t)d * kColTile;  // d x kFdDenseW
  const double* __restrict__ v = q.v + (size_t)sp * d * ld + blockIdx.y * kColTile;
  for (int t = threadIdx.x; t < d * (kColTile / 2); t += blockDim.x) {
    const int e = t / (kColTile / 2), c = 2 * (t - e * (kColTile / 2));
    cp_async16(vb + e * kColTile + c, v + (size_t)e * ld + c);
  }
  for (int t = threadIdx.x; t < d * (kFdDenseW / 2); t += blockDim.x) cp_async16(wt + 2 * t, q.fdT_dense + 2 * t);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  double* __restrict__ out = q.fdT + (size_t)sp * d * ld + col;
  constexpr int U = kFdChunk + 2 * kFdHalo;
  for (int c0 = wid * kFdChunk; c0 < d; c0 += (blockDim.x >> 5) * kFdChunk) {
    double u[U];
#pragma unroll
    for (int i = 0; i < U; ++i) {
      const int e = c0 - kFdHalo + i;
      u[i] = (e >= 0 && e < d) ? vb[e * kColTile + lane] : 0.0;
    }
#pragma unroll
    for (int i = 0; i < kFdChunk; ++i) {
      const int e = c0 + i;
      if (e >= d) break;
      const double2* w2 = reinterpret_cast<const double2*>(wt + e * kFdDenseW);
      const double2 wa = w2[0], wb = w2[1], wc = w2[2], wd = w2[3];
      double sT = __fma_rn(wa.x, u[i], 0.0);
      sT = __fma_rn(wa.y, u[i + 1], sT);
      sT = __fma_rn(wb.x, u[i + 2], sT);
      sT = __fma_rn(wb.y, u[i + 3], sT);
      sT = __fma_rn(wc.x, u[i + 4], sT);
      sT = __fma_rn(wc.y, u[i + 5], sT);
      sT = __fma_rn(wd.x, u[i + 6], sT);
      out[(size_t)e * ld] = sT;
    }
  }
}

// bT = band part of M_off^T v.  CTA = (64-column block, mother-species group),
// 8 warps; warp = one 8-column tile.  The warp loads the v fragments of both
// band species once (k-tiles of 4 daughter bins, shifted by J - 2 so the band
// below each mother row tile starts at 0); per mother species the CTA copies
// its transposed tiles into shared memory (double-buffered cp.async) and the
// warp accumulates RT row tiles of 8 mother bins and writes them out.
template <int RT, int J>
__global__ void __launch_bounds__(256, 1) k_bandT(AdjBlk q) {
  extern __shared__ double sm[];
  constexpr int KS = J - 2;              // k-tile shift
  constexpr int KV = 2 * RT + KS;        // v fragments per band species
  constexpr int ABLK = 2 * RT * J * 32;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int c0 = blockIdx.x * 64 + wid * 8;
  const bool wact = c0 < q.ncols;
  const int g = blockIdx.y;
  const int s0 = g * q.spg, s1 = min(q.nsp, s0 + q.spg);
  const int d = q.d, ld = q.ld;
  const double* __restrict__ A = q.bandT + (size_t)q.w * q.band_stride;
  double* As = sm;
  auto issue = [&](int sp, int stage) {
    const double* src = A + (size_t)sp * ABLK;
    for (int c = threadIdx.x; c < ABLK / 2; c += blockDim.x) cp_async16(As + stage * ABLK + 2 * c, src + 2 * c);
    cp_async_commit();
  };
  const int kr = lane & 3;
  double vf[2][KV];
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    const bool on = wact && b < q.nb;
    const double* vs = q.v + (size_t)(on ? q.band_spec[b] : 0) * d * ld + c0 + (lane >> 2);
#pragma unroll
    for (int t = 0; t < KV; ++t) {
      const int e = 4 * (t - KS) + kr;
      vf[b][t] = (on && e >= 0 && e < d) ? vs[(size_t)e * ld] : 0.0;
    }
  }
  if (s0 < s1) issue(s0, 0);
  for (int sp = s0; sp < s1; ++sp) {
    const int stage = (sp - s0) & 1;
    if (sp + 1 < s1) {
      issue(sp + 1, stage ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* __restrict__ as = As + stage * ABLK + lane;
    double acc[RT][2];
#pragma unroll
    for (int mt = 0; mt < RT; ++mt) acc[mt][0] = acc[mt][1] = 0.0;
#pragma unroll
    for (int jj = 0; jj < J; ++jj)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int mt = 0; mt < RT; ++mt)
          dmma884(acc[mt][0], acc[mt][1], as[((b * RT + mt) * J + jj) * 32], vf[b][2 * mt + jj]);
    __syncthreads();
    if (wact) {
      double* __restrict__ out = q.bT + (size_t)sp * d * ld + c0 + kr * 2;
#pragma unroll
      for (int mt = 0; mt < RT; ++mt) {
        const int row = 8 * mt + (lane >> 2);
        if (row >= d) continue;
        double2 o;
        o.x = acc[mt][0];
        o.y = acc[mt][1];
        *reinterpret_cast<double2*>(out + (size_t)row * ld) = o;
      }
    }
  }
}

template <int RT, int J>
size_t bandT_smem_bytes() {
  return (size_t)2 * (2 * RT * J * 32) * sizeof(double);
}

// k_slabT's shared memory: the v slab of one bin (nsp x 16 columns), the bin's
// entry values (4 per quad), daughter-row byte offsets (4 x 16 bits per quad)
// and mother-row pairs.  Every block starts on a 16-byte boundary.
constexpr int kSlabTPre = 2;        // row pairs whose inputs a warp loads ahead
constexpr int kSlabTWarps = 12;     // two CTAs per SM (80 registers)
struct SlabTSmem {
  double* slab;  // rows padded to whole TMA boxes (as k_slab's)
  unsigned long long* bar;  // the TMA staging barrier (a 16-byte slot)
  double* vals;
  unsigned long long* sidx;
  int4* pairs;
  __host__ __device__ static size_t bytes(int nsp, int maxq, int maxp) {
    return (size_t)SlabSmem::rows(nsp) * kSlabCols * sizeof(double) + 16 +
           (size_t)maxq * (4 * sizeof(double) + sizeof(unsigned long long)) + (size_t)maxp * sizeof(int4);
  }
  __device__ SlabTSmem(double* base, int nsp, int maxq) {
    slab = base;
    bar = reinterpret_cast<unsigned long long*>(slab + (size_t)SlabSmem::rows(nsp) * kSlabCols);
    vals = slab + (size_t)SlabSmem::rows(nsp) * kSlabCols + 2;
    sidx = reinterpret_cast<unsigned long long*>(vals + (size_t)maxq * 4);
    pairs = reinterpret_cast<int4*>(sidx + maxq);
  }
};

// Bin-local part of M_off^T v and the adjoint stage update for every row of
// bin e.  CTA = (bin e, 16-column tile); a half-warp owns a mother row, its
// lane c owns column col0 + c.  The v slab of bin e arrives by TMA (boxes of a
// tensor map over v, as in k_slab), the bin's entry quads and row pairs by
// bulk copies, all on one bounded mbarrier wait (cp.async when TMA is off);
// each row is summed from shared
// memory (four accumulators, one per quad position).  The row's band term, FD
// term, lam' (stage 1) or mu (stage 2), P and Q, and its recorded factors are
// loaded kSlabTPre pairs ahead into registers.  Stage 1 reduces the
// photon-scale gradient of the bin's rows inside the CTA.
template <int STAGE>
__global__ void __launch_bounds__(kSlabTWarps * 32, 2) k_slabT(AdjBlk q) {
  extern __shared__ __align__(128) double sm[];  // TMA boxes land at 128-byte boundaries
  const int nsp = q.nsp, e = blockIdx.x, d = q.d, ld = q.ld;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int half = lane >> 4, c = lane & 15;
  const int col0 = blockIdx.y * kSlabCols, col = col0 + c;  // col < ld
  const bool active = col < q.ncols;
  SlabTSmem L(sm, nsp, q.slabT_maxq);
  const int qb = q.slabT_qbase[e], nqb = q.slabT_qbase[e + 1] - qb;
  const int pb0 = q.slabT_wrp[e * (kSlabTWarps + 1)], npb = q.slabT_wrp[e * (kSlabTWarps + 1) + kSlabTWarps] - pb0;
  const bool photohad = (q.flags & PB_PHOTOHAD) != 0, kap = (q.flags & PB_PARTIAL_DIFF) != 0;
  const double* mv = q.slabT + (size_t)q.w * q.slabT_stride + (size_t)qb * 4;
  if (q.tmap_v) {  // TMA: the v slab as tensor boxes, the entries and pairs as bulk copies, one barrier
    if (threadIdx.x == 0) mbar_init(L.bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      const int nb = SlabSmem::nbox(nsp), br = SlabSmem::box_rows(nsp);
      unsigned bytes = (unsigned)(nb * br * kSlabCols * sizeof(double)) + (unsigned)(npb * sizeof(int4));
      if (photohad) bytes += (unsigned)(nqb * (4 * sizeof(double) + sizeof(unsigned long long)));
      mbar_expect_tx(L.bar, bytes);
      for (int b = 0; b < nb; ++b) tma_load_3d(L.slab + (size_t)b * br * kSlabCols, q.tmap_v, col0, e, b * br, L.bar);
      if (photohad && nqb > 0) {
        bulk_load(L.vals, mv, (unsigned)(nqb * 4 * sizeof(double)), L.bar);
        bulk_load(L.sidx, q.slabT_q + qb, (unsigned)(nqb * sizeof(unsigned long long)), L.bar);
      }
      if (npb > 0) bulk_load(L.pairs, q.slabT_pairs + pb0, (unsigned)(npb * sizeof(int4)), L.bar);
    }
  } else {
    const double* vs = q.v + (size_t)e * ld + col0;
    for (int t = threadIdx.x; t < nsp * (kSlabCols / 2); t += blockDim.x) {
      const int sp = t / (kSlabCols / 2), cc = 2 * (t - sp * (kSlabCols / 2));
      cp_async16(L.slab + sp * kSlabCols + cc, vs + (size_t)sp * d * ld + cc);
    }
    if (photohad) {
      for (int t = threadIdx.x; t < 2 * nqb; t += blockDim.x) cp_async16(L.vals + 2 * t, mv + 2 * t);
      const unsigned long long* mq = q.slabT_q + qb;
      for (int t = threadIdx.x; t < nqb / 2; t += blockDim.x) cp_async16(L.sidx + 2 * t, mq + 2 * t);
    }
    for (int t = threadIdx.x; t < npb; t += blockDim.x) cp_async16(L.pairs + t, q.slabT_pairs + pb0 + t);
    cp_async_commit();
  }
  const int w0 = q.slabT_wrp[e * (kSlabTWarps + 1) + wid], w1 = q.slabT_wrp[e * (kSlabTWarps + 1) + wid + 1];
  const double* own_src = STAGE == 1 ? q.lam : q.mu;
  const bool want_pq = STAGE == 1 && q.gs;
  constexpr int PRE = kSlabTPre;
  // per pair slot: band term, FD term, own (lam' or mu), P, Q; kappa and the
  // row factors (stage 1: phi1, phi2; stage 2: eD, phi2 of the previous step)
  double rb[PRE], rfd[PRE], rown[PRE], rp[PRE], rq[PRE], rk[PRE], rf1[PRE], rf2[PRE];
  int rsl[PRE];
#define PB_SLABT_LOAD(U, PI, PR)                                                 \
  do {                                                                           \
    if ((PI) < w1) {                                                             \
      const int4 pr_ = (PR);                                                     \
      const int sp_ = half ? pr_.y : pr_.x;                                      \
      if (sp_ >= 0) {                                                            \
        const int r_ = sp_ * d + e;                                              \
        const size_t ix_ = (size_t)r_ * ld + col;                                \
        rb[U] = photohad ? q.bT[ix_] : 0.0;                                      \
        rfd[U] = kap ? q.fdT[ix_] : 0.0;                                         \
        rown[U] = own_src[ix_];                                                  \
        rp[U] = want_pq ? q.P[ix_] : 0.0;                                        \
        rq[U] = want_pq ? q.Q[ix_] : 0.0;                                        \
        rk[U] = kap ? q.rf[3 * q.n + r_] : 0.0;                                  \
        rf1[U] = STAGE == 1 ? q.rf[q.n + r_] : q.rf[r_];                         \
        rf2[U] = STAGE == 1 ? q.rf[2 * q.n + r_] : (q.rf_prev ? q.rf_prev[2 * q.n + r_] : 0.0); \
        rsl[U] = (STAGE == 1 && q.gb_inj) ? q.inj_slot[r_] : -1;                 \
      }                                                                          \
    }                                                                            \
  } while (0)
#pragma unroll
  for (int u = 0; u < PRE; ++u) PB_SLABT_LOAD(u, w0 + u, __ldg(q.slabT_pairs + w0 + u));
  if (q.tmap_v) {
    if (!mbar_wait_bounded(L.bar, 0, q.wait_tries)) {  // the copies did not land: report and leave
      if (threadIdx.x == 0) atomicExch(q.err, kErrStagingWait);
      mbar_wait_bounded(L.bar, 0, kWaitTries);
      return;
    }
  } else {
    cp_async_wait<0>();
  }
  __syncthreads();

  double gsa = 0.0;  // this lane's column of the photon-scale gradient over its rows
  const char* slb = reinterpret_cast<const char*>(L.slab + c);
  const double2* vq = reinterpret_cast<const double2*>(L.vals);
  for (int pb = w0; pb < w1; pb += PRE) {
#pragma unroll
    for (int u = 0; u < PRE; ++u) {
      const int pi = pb + u;
      if (pi >= w1) break;
      const int4 pr = L.pairs[pi - pb0];
      const int sp = half ? pr.y : pr.x;
      const int qq = half ? pr.w : pr.z;
      const int r = sp * d + e;
      double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
      if (sp >= 0 && photohad) {
        const int qa = qq >> 16, qz = qa + (qq & 0xffff);
#pragma unroll 2
        for (int k = qa; k < qz; ++k) {
          const double2 va = vq[2 * k], vb = vq[2 * k + 1];
          const unsigned long long m = L.sidx[k];
          const double x0 = *reinterpret_cast<const double*>(slb + ((unsigned)m & 0xffffu));
          const double x1 = *reinterpret_cast<const double*>(slb + ((unsigned)(m >> 16) & 0xffffu));
          const double x2 = *reinterpret_cast<const double*>(slb + ((unsigned)(m >> 32) & 0xffffu));
          const double x3 = *reinterpret_cast<const double*>(slb + (unsigned)(m >> 48));
          acc0 = __fma_rn(va.x, x0, acc0);
          acc1 = __fma_rn(va.y, x1, acc1);
          acc2 = __fma_rn(vb.x, x2, acc2);
          acc3 = __fma_rn(vb.y, x3, acc3);
        }
      }
      if (sp >= 0 && active) {
        double out = photohad ? ((acc0 + acc1) + (acc2 + acc3)) + rb[u] : 0.0;
        if (kap) out += rk[u] * rfd[u];
        if (q.lt_indptr) {
          double sL = 0.0;
          for (int64_t j = q.lt_indptr[r]; j < q.lt_indptr[r + 1]; ++j)
            sL += q.lt_vals[j] * q.v[(size_t)q.lt_indices[j] * ld + col];
          out += sL;
        }
        out *= q.dl;
        const size_t idx = (size_t)r * ld + col;
        if (STAGE == 1) {
          const double lam = rown[u];
          const double mu = lam + q.h * out;
          q.mu[idx] = mu;
          if (rsl[u] >= 0) q.gb_inj[(size_t)rsl[u] * ld + col] = q.h * rf1[u] * mu;
          if (want_pq) gsa += mu * rp[u] + lam * rq[u];
          q.vout[idx] = rf1[u] * mu - rf2[u] * lam;
        } else {
          const double lam = rf1[u] * rown[u] + q.h * out;
          q.lam_out[idx] = lam;
          if (q.rf_prev) q.vout[idx] = rf2[u] * lam;
        }
      }
      const int pn = pi + PRE;
      PB_SLABT_LOAD(u, pn, L.pairs[pn - pb0]);
    }
  }
#undef PB_SLABT_LOAD
  if (want_pq) {  // the half-warps' sums for each column, added to the bin's row of gs
    __syncthreads();
    double* red = L.slab;  // the slab is no longer read
    red[threadIdx.x] = gsa;
    __syncthreads();
    if (threadIdx.x < kSlabCols && col0 + (int)threadIdx.x < q.ncols) {
      double t = 0.0;
      for (int h = 0; h < 2 * kSlabTWarps; ++h) t += red[h * kSlabCols + threadIdx.x];
      q.gs[(size_t)e * ld + col0 + threadIdx.x] += t;
    }
  }
}

using BandTKernel = void (*)(AdjBlk);
struct BandTInstance {
  BandTKernel fn;
  size_t smem;
};
template <int RT>
BandTInstance bandT_kernel_j(int J) {
  switch (J) {
    case 5: return {k_bandT<RT, 5>, bandT_smem_bytes<RT, 5>()};
    case 9: return {k_bandT<RT, 9>, bandT_smem_bytes<RT, 9>()};
    case 13: return {k_bandT<RT, 13>, bandT_smem_bytes<RT, 13>()};
    case 17: return {k_bandT<RT, 17>, bandT_smem_bytes<RT, 17>()};
  }
  return {nullptr, 0};
}
BandTInstance bandT_kernel(int RT, int J) {
  switch (RT) {
    case 4: return bandT_kernel_j<4>(J);
    case 8: return bandT_kernel_j<8>(J);
    case 12: return bandT_kernel_j<12>(J);
    case 16: return bandT_kernel_j<16>(J);
  }
  return {nullptr, 0};
}

// transposed copies of the band tiles and the bin-local entries of every window
__global__ void k_transpose_blocks(const int* __restrict__ bslot, const int* __restrict__ bslotT,
                                   const int* __restrict__ sslot, const int* __restrict__ sslotT, int64_t R, int W,
                                   const double* __restrict__ band, double* __restrict__ bandT, int64_t bstride,
                                   const double* __restrict__ slab, int64_t sstride, double* __restrict__ slabT,
                                   int64_t tstride) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= R) return;
  const int b = bslot[j], bt = bslotT[j], s = sslot[j], st = sslotT[j];
  for (int w = 0; w < W; ++w) {
    if (b >= 0 && bt >= 0) bandT[(size_t)w * bstride + bt] = band[(size_t)w * bstride + b];
    if (s >= 0 && st >= 0) slabT[(size_t)w * tstride + st] = slab[(size_t)w * sstride + s];
  }
}

// ---------------------------------------------------------------------------
// Discrete adjoint of the ETD2 step.  Forward, with A = dl (M_off + D_off diag(kappa)
// + Lambda_off) frozen over the step:
//   a = E x + h Phi1 (A x + b),   x' = a + h Phi2 A (a - x).
// Backward, given lam' = dL/dx':
//   mu  = lam' + h A^T (Phi2 lam')                    (stage 1; dL/da)
//   lam = E mu + h A^T (Phi1 mu - Phi2 lam')          (stage 2; dL/dx)
//   dL/db = h Phi1 mu,
//   dL/dscale += mu . P + lam' . Q with the recorded P = d a / d scale and
//   Q = h d(Phi2)/d scale A(a - x) + h Phi2 (dA/d scale)(a - x).
// A^T = dl (M_off^T + diag(kappa) D_off^T + Lambda_off^T).
// ---------------------------------------------------------------------------
struct AdjParams {
  int64_t n;
  int64_t row0;             // first row of the launch (the tail of the bin-blocked sweep), else 0
  int ld;
  int ncols;
  int64_t step;
  uint32_t flags;
  double h, dl;
  int w;
  const int64_t* t_indptr;  // M_off^T pattern (rows = columns of M_off)
  const int* t_indices;
  const int* t_perm;        // entry of M_off behind each M_off^T entry
  const double* m_vals;     // window w values of M_off
  const int64_t* dt_indptr;
  const int* dt_indices;
  const double* dt_vals;
  const int64_t* lt_indptr;
  const int* lt_indices;
  const double* lt_vals;
  const double* rf;         // recorded eD, phi1, phi2, kappa of this step (n each)
  const double* P;          // recorded sigma vectors of this step or null
  const double* Q;
  const double* lam;        // dL/dx'
  double* mu;               // dL/da
  double* lam_out;          // dL/dx
  const int* inj_slot;
  double* gb_inj;           // n_inj x ld: dL/db of this step on the injected rows, or null
  double* gs;               // n x ld accumulator of the scale gradient, or null
};

template <int STAGE>
__device__ __forceinline__ double adj_v(const AdjParams& a, int c, int k) {
  const size_t i = (size_t)c * a.ld + k;
  if (STAGE == 1) return a.rf[2 * a.n + c] * a.lam[i];
  return a.rf[a.n + c] * a.mu[i] - a.rf[2 * a.n + c] * a.lam[i];
}

template <int STAGE>
__global__ void __launch_bounds__(256) k_adj(AdjParams a) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t r = a.row0 + (int64_t)blockIdx.x * (blockDim.x >> 5) + wid;
  if (r >= a.n) return;
  const int k = blockIdx.y * kColTile + lane;
  const bool active = k < a.ncols;
  const int kk = active ? k : 0;
  double sM = 0.0;
  if (a.flags & PB_PHOTOHAD) {
    const int64_t j0 = a.t_indptr[r], j1 = a.t_indptr[r + 1];
    for (int64_t base = j0; base < j1; base += 32) {
      const int64_t j = base + lane;
      const double mvl = (j < j1) ? a.m_vals[a.t_perm[j]] : 0.0;
      const int cl = (j < j1) ? a.t_indices[j] : 0;
      const int cnt = (int)min((int64_t)32, j1 - base);
      for (int q = 0; q < cnt; ++q) {
        const double mq = __shfl_sync(0xffffffffu, mvl, q);
        const int cq = __shfl_sync(0xffffffffu, cl, q);
        sM += mq * adj_v<STAGE>(a, cq, kk);
      }
    }
  }
  if (!active) return;
  double out = sM;
  if (a.flags & PB_PARTIAL_DIFF) {
    double sD = 0.0;
    for (int64_t j = a.dt_indptr[r]; j < a.dt_indptr[r + 1]; ++j) sD += a.dt_vals[j] * adj_v<STAGE>(a, a.dt_indices[j], k);
    out += a.rf[3 * a.n + r] * sD;
  }
  if ((a.flags & PB_DECAY) && a.lt_indptr) {
    double sL = 0.0;
    for (int64_t j = a.lt_indptr[r]; j < a.lt_indptr[r + 1]; ++j) sL += a.lt_vals[j] * adj_v<STAGE>(a, a.lt_indices[j], k);
    out += sL;
  }
  out *= a.dl;
  const size_t idx = (size_t)r * a.ld + k;
  if (STAGE == 1) {
    const double mu = a.lam[idx] + a.h * out;
    a.mu[idx] = mu;
    if (a.gb_inj) {
      const int slot = a.inj_slot[r];
      if (slot >= 0) a.gb_inj[(size_t)slot * a.ld + k] = a.h * a.rf[a.n + r] * mu;
    }
    if (a.gs) a.gs[idx] += mu * a.P[idx] + a.lam[idx] * a.Q[idx];
  } else {
    a.lam_out[idx] = a.rf[r] * a.mu[idx] + a.h * out;
  }
}

// transpose of the M_off pattern: row of every entry, sentinel keys past nnz
__global__ void k_entry_rows(const int64_t* __restrict__ indptr, int64_t n, int* __restrict__ row) {
  const int64_t r = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (r >= n) return;
  for (int64_t j = indptr[r] + (threadIdx.x & 31); j < indptr[r + 1]; j += 32) row[j] = (int)r;
}

__global__ void k_transpose_keys(const int* __restrict__ indices, const int64_t* __restrict__ indptr, int64_t n,
                                 int64_t R, int* __restrict__ keys, int* __restrict__ vals) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= R) return;
  const int64_t nnz = indptr[n];
  keys[j] = j < nnz ? indices[j] : (int)n;
  vals[j] = (int)j;
}

__global__ void k_transpose_finish(const int* __restrict__ skeys, const int* __restrict__ svals,
                                   const int* __restrict__ erow, int64_t n, int64_t R, int64_t* __restrict__ t_indptr,
                                   int* __restrict__ t_indices, int* __restrict__ t_perm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= n) {  // t_indptr[c] = first sorted position with key >= c
    int64_t lo = 0, hi = R;
    while (lo < hi) {
      const int64_t mid = (lo + hi) / 2;
      if (skeys[mid] < (int)i) lo = mid + 1; else hi = mid;
    }
    t_indptr[i] = lo;
  }
  if (i < R && skeys[i] < (int)n) {
    t_perm[i] = svals[i];
    t_indices[i] = erow[svals[i]];
  }
}

// dL/dcoeff[k][s] = finj_k sum_slot G[slot][s] dL/db_k[row(slot)][col(s)] (active steps)
__global__ void k_grad_coeff(const double* __restrict__ gb, const double* __restrict__ G,
                             const double* __restrict__ finj, const int* __restrict__ src_col,
                             const int* __restrict__ n_active, int64_t S, int n_src, int n_inj, int ld,
                             double* __restrict__ gcoeff) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S * n_src) return;
  const int64_t k = i / n_src;
  const int s = (int)(i % n_src), col = src_col[s];
  double acc = 0.0;
  if (col < n_active[k]) {
    const double* g = gb + (size_t)k * n_inj * ld;
    for (int q = 0; q < n_inj; ++q) acc += G[(size_t)q * n_src + s] * g[(size_t)q * ld + col];
    acc *= finj[k];
  }
  gcoeff[i] = acc;
}

// dL/dG[slot][s] = sum_k finj_k coeff[k][s] dL/db_k[row(slot)][col(s)] (active steps)
__global__ void k_grad_grids(const double* __restrict__ gb, const double* __restrict__ coeff,
                             const double* __restrict__ finj, const int* __restrict__ src_col,
                             const int* __restrict__ n_active, int64_t S, int n_src, int n_inj, int ld,
                             double* __restrict__ gG) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)n_inj * n_src) return;
  const int q = (int)(i / n_src), s = (int)(i % n_src), col = src_col[s];
  double acc = 0.0;
  for (int64_t k = 0; k < S; ++k)
    if (col < n_active[k]) acc += finj[k] * coeff[(size_t)k * n_src + s] * gb[((size_t)k * n_inj + q) * ld + col];
  gG[i] = acc;
}

__global__ void k_grad_scale(const double* __restrict__ gs, int64_t n, int ld, int K, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  double acc = 0.0;
  for (int64_t r = 0; r < n; ++r) acc += gs[(size_t)r * ld + k];
  out[k] = acc;
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
template <class T>
int upload(pb_context* c, DBuf& b, const T* src, size_t count) {
  cudaError_t e = b.ensure(count * sizeof(T));
  if (e != cudaSuccess) return fail(c, PB_ERR_CUDA, "cudaMalloc(%zu) failed: %s", count * sizeof(T), cudaGetErrorString(e));
  if (count) {
    e = cudaMemcpyAsync(b.p, src, count * sizeof(T), cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return fail(c, PB_ERR_CUDA, "cudaMemcpyAsync H2D failed: %s", cudaGetErrorString(e));
  }
  return PB_OK;
}

int set_device(pb_context* c) {
  PB_CUDA(c, cudaSetDevice(c->device));
  return PB_OK;
}

FieldDesc field_desc(const pb_context* c, double scale) {
  FieldDesc f;
  memset(&f, 0, sizeof(f));  // padding bytes take part in the graph key
  f.n = c->n_comp;
  for (int i = 0; i < 8; ++i) {
    f.kind[i] = i < c->n_comp ? c->comp_kind[i] : 0;
    for (int q = 0; q < 3; ++q) f.p[i][q] = i < c->n_comp ? c->comp_par[i][q] : 0.0;
  }
  f.scale = scale;
  if (c->tab_nz > 0) {
    f.tz = c->tab_z.as<double>();
    f.tle = c->tab_le.as<double>();
    f.tv = c->tab_v.as<double>();
    f.tnz = c->tab_nz;
    f.tne = c->tab_ne;
  }
  return f;
}

// Buffers the forward solve reads or writes (the two captured graphs point into these).
std::vector<DBuf*> solve_buffers(pb_context* c) {
  return {&c->cpl_indptr, &c->cpl_indices, &c->cpl_row, &c->cpl_is_diag, &c->short_rows, &c->long_rows, &c->kernel,
          &c->eph, &c->d_indptr, &c->d_indices, &c->d_vals, &c->d_diag, &c->adia_E, &c->pair_scale, &c->pair_bin,
          &c->xi, &c->phi_xi2, &c->pair_pg, &c->l_diag, &c->l_indptr, &c->l_indices, &c->l_vals, &c->inj_slot,
          &c->inj_G, &c->src_ptr, &c->PT, &c->zwin, &c->rs, &c->kp, &c->keep, &c->pos, &c->dest, &c->m_indptr,
          &c->m_indices, &c->m_vals, &c->m_diag, &c->s_h, &c->s_dldz, &c->s_hc, &c->s_finj, &c->s_win, &c->s_coeff,
          &c->X, &c->A, &c->F, &c->rowf, &c->scan_tmp, &c->seg_cb, &c->seg_ce, &c->seg_lr, &c->lr_seg0, &c->lr_nseg,
          &c->seg_mb, &c->seg_me, &c->partial, &c->counter, &c->dt_indptr, &c->dt_indices, &c->dt_vals,
          &c->lt_indptr, &c->lt_indices, &c->lt_vals, &c->inj_rows, &c->src_col_d, &c->ckpt,
          &c->em_bh_off, &c->em_bh_A, &c->em_invE, &c->em_dE, &c->em_Tg, &c->em_Te, &c->em_R, &c->em_wbuf,
          &c->em_es, &c->em_lep, &c->em_y, &c->em_TgT, &c->em_TeT, &c->em_RT,
          &c->band_slot, &c->band_spec, &c->slab_spec, &c->band_vals, &c->band_part, &c->slab_rp,
          &c->slab_sidx, &c->slab_slot, &c->slab_vals, &c->slab_quart, &c->slab_wrp, &c->slab_rowslot, &c->slab_fac, &c->fd_cnt, &c->fd_off, &c->fd_val, &c->fd_dense, &c->fdT_dense, &c->fdbuf,
          &c->bandT_slot, &c->slabT_rp, &c->slabT_offs, &c->slabT_slot, &c->fdT_cnt, &c->fdT_off, &c->fdT_val,
          &c->slabT_pairs, &c->slabT_wrp, &c->tmaps, &c->d_err, &c->tab_z, &c->tab_le, &c->tab_v};
}

// Every device buffer: the solve's and the adjoint's scratch.
std::vector<DBuf*> all_buffers(pb_context* c) {
  std::vector<DBuf*> b = solve_buffers(c);
  for (DBuf* x : {&c->nact, &c->lam, &c->lam2, &c->mu, &c->rec_rf, &c->rec_P, &c->rec_Q, &c->rec_sx, &c->dsig, &c->gb_inj,
                  &c->gs, &c->g_out, &c->erow, &c->tkeys, &c->tvals, &c->skeys, &c->svals, &c->t_indptr,
                  &c->t_indices, &c->t_perm, &c->sort_tmp, &c->fdkp, &c->bandT_vals, &c->slabT_vals, &c->vbuf,
                  &c->vbuf2, &c->bTbuf, &c->fdTbuf, &c->outcols, &c->tmapsT})
    b.push_back(x);
  return b;
}

// Stable CSR transpose (entries of a transposed row keep increasing column order).
void csr_transpose(int64_t n, int64_t nnz, const int64_t* ip, const int32_t* ix, const double* v,
                   std::vector<int64_t>& tip, std::vector<int32_t>& tix, std::vector<double>& tv) {
  tip.assign((size_t)n + 1, 0);
  for (int64_t j = 0; j < nnz; ++j) tip[(size_t)ix[j] + 1]++;
  for (int64_t i = 0; i < n; ++i) tip[i + 1] += tip[i];
  std::vector<int64_t> fill(tip.begin(), tip.end() - 1);
  tix.assign((size_t)std::max<int64_t>(nnz, 1), 0);
  tv.assign((size_t)std::max<int64_t>(nnz, 1), 0.0);
  for (int64_t r = 0; r < n; ++r)
    for (int64_t j = ip[r]; j < ip[r + 1]; ++j) {
      const int64_t t = fill[ix[j]]++;
      tix[t] = (int32_t)r;
      tv[t] = v[j];
    }
}


// Step parameters of a solve on the context's device buffers.
void fill_step_params(pb_context* c, StepParams& p, int K, int ld, uint32_t flags, bool pair, bool inj, int64_t S,
                      int ctiles) {
  const int64_t n = c->n;
  const int64_t mstride = std::max<int64_t>(c->R, 1);
  p.n = n;
  p.ld = ld;
  p.flags = flags;
  p.wait_tries = c->staging_wait_tries;
  if (!pair) p.flags &= ~PB_PAIRPROD;
  if (!inj) p.flags &= ~PB_INJECTION;
  p.h = c->s_h.as<double>();
  p.dldz = c->s_dldz.as<double>();
  p.hc = c->s_hc.as<double>();
  p.finj = c->s_finj.as<double>();
  p.win = c->s_win.as<int>();
  p.m_indptr = c->m_indptr.as<int64_t>();
  p.m_indices = c->m_indices.as<int>();
  p.m_vals = c->m_vals.as<double>();
  p.m_wstride = mstride;
  p.m_diag = c->m_diag.as<double>();
  p.d_indptr = c->d_indptr.as<int64_t>();
  p.d_indices = c->d_indices.as<int>();
  p.d_vals = c->d_vals.as<double>();
  p.d_diag = c->d_diag.as<double>();
  p.E = c->adia_E.as<double>();
  p.kp = pair ? c->kp.as<double>() : nullptr;
  if ((flags & PB_DECAY) && c->have_decay) {
    p.l_indptr = c->l_indptr.as<int64_t>();
    p.l_indices = c->l_indices.as<int>();
    p.l_vals = c->l_vals.as<double>();
    p.l_diag = c->l_diag.as<double>();
  }
  if (inj) {
    p.inj_slot = c->inj_slot.as<int>();
    p.G = c->inj_G.as<double>();
    p.n_src = c->n_src;
    p.src_ptr = c->src_ptr.as<int>();
    p.coeff = c->s_coeff.as<double>();
  }
  p.a = c->A.as<double>();
  p.f = c->F.as<double>();
  p.n_steps = S;
  p.eD = c->rowf.as<double>();
  p.phi1 = p.eD + 2 * n;
  p.phi2 = p.eD + 4 * n;
  p.kap = p.eD + 6 * n;
  p.rows = c->short_rows.as<int>();
  p.nrows = (int)c->h_short_rows.size();
  p.nsb = (int)blocks_for(p.nrows, K == 1 ? 256 : 8);   // thread per row (K = 1) or warp per row
  p.seg_lr = c->seg_lr.as<int>();
  p.seg_mb = c->seg_mb.as<int64_t>();
  p.seg_me = c->seg_me.as<int64_t>();
  p.nseg = c->n_seg;
  p.lr_row = c->long_rows.as<int>();
  p.lr_seg0 = c->lr_seg0.as<int>();
  p.lr_nseg = c->lr_nseg.as<int>();
  p.partial = c->partial.as<double>();
  p.counter = c->counter.as<int>();
  p.ctiles = ctiles;
  p.d = c->lay_d;
  p.nsp = c->lay_nsp;
  p.slab_spec = c->slab_spec.as<int>();
  p.n_slab_spec = c->n_slab_spec;
  p.slab_qbase = c->slab_rp.as<int>();
  p.slab_q = c->slab_sidx.as<unsigned long long>();
  p.slab_quart = c->slab_quart.as<int4>();
  p.slab_wrp = c->slab_wrp.as<int>();
  p.slab_vals = c->slab_vals.as<double>();
  p.slab_stride = c->slab_nent;
  p.slab_maxq = c->slab_maxbin;
  p.slab_maxp = (c->n_slab_spec + kSlabRows - 1) / kSlabRows;
  p.slab_rowslot = c->blocked_ok ? c->slab_rowslot.as<int>() : nullptr;
  p.slab_fac = c->slab_fac.as<double>();
  p.slab_nslots = c->slab_nslots;
  p.fd_cnt = c->fd_cnt.as<int>();
  p.fd_off = c->fd_off.as<int>();
  p.fd_val = c->fd_val.as<double>();
  p.fd_dense = c->fd_dense.as<double>();
  p.fdbuf = c->fdbuf.as<double>();
  p.band_spec = c->band_spec.as<int>();
  p.nb = c->band_nb;
  p.band_vals = c->band_vals.as<double>();
  p.band_stride = c->band_stride;
  p.band_part = c->band_part.as<double>();
}

// cuTensorMapEncodeTiled, reached through the runtime (no link against the driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn tensor_map_encoder() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  });
  return fn;
}

// Tensor maps of X and A as (column, bin, species) for k_slab's TMA staging
// (box = 16 columns x 1 bin x box_rows species) and for k_band_tma's (box =
// 64 columns x d bins x 1 species).  Leaves tma_ok false (cp.async staging)
// when TMA is switched off, the encoder is missing or a map is refused, and
// tma_band_ok false when only the band maps are refused.
int ensure_tmaps(pb_context* c, bool blocked, int ld) {
  const bool want = blocked && c->tma_mode == 1 && ld % kSlabCols == 0;
  if (want && c->tma_ok && c->tma_key[0] == c->X.p && c->tma_key[1] == c->A.p &&
      c->tma_key[2] == reinterpret_cast<const void*>((intptr_t)ld))
    return PB_OK;
  c->tma_ok = false;
  c->tma_band_ok = false;
  if (!want) return PB_OK;
  const EncodeTiledFn enc = tensor_map_encoder();
  if (!enc) return PB_OK;
  const int d = c->lay_d, nsp = c->lay_nsp;
  CUtensorMap maps[4];
  bool band_ok = d <= 256;
  for (int k = 0; k < 4; ++k) {
    const bool band = k >= 2;
    if (band && !band_ok) break;
    const cuuint64_t dims[3] = {(cuuint64_t)ld, (cuuint64_t)d, (cuuint64_t)nsp};
    const cuuint64_t strides[2] = {(cuuint64_t)ld * sizeof(double), (cuuint64_t)d * ld * sizeof(double)};
    const cuuint32_t box[3] = {band ? 64u : (cuuint32_t)kSlabCols, band ? (cuuint32_t)d : 1u,
                               band ? 1u : (cuuint32_t)SlabSmem::box_rows(nsp)};
    const cuuint32_t es[3] = {1u, 1u, 1u};
    if (enc(&maps[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, k % 2 == 0 ? c->X.p : c->A.p, dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      if (!band) return PB_OK;
      band_ok = false;
    }
  }
  PB_CUDA(c, c->tmaps.ensure(sizeof(maps)));
  PB_CUDA(c, cudaMemcpy(c->tmaps.p, maps, sizeof(maps), cudaMemcpyHostToDevice));
  c->tma_key[0] = c->X.p;
  c->tma_key[1] = c->A.p;
  c->tma_key[2] = reinterpret_cast<const void*>((intptr_t)ld);
  c->tma_ok = true;
  c->tma_band_ok = band_ok;
  return PB_OK;
}

// Tensor maps of the adjoint sweep's v buffers (vbuf: stage 1, vbuf2: stage 2)
// for k_slabT's TMA staging, shaped as k_slab's.  Leaves tmaT_ok false
// (cp.async staging) when TMA is switched off or a map is refused.
int ensure_tmapsT(pb_context* c, int ld) {
  const bool want = c->tma_mode == 1 && ld % kSlabCols == 0;
  if (want && c->tmaT_ok && c->tmaT_key[0] == c->vbuf.p && c->tmaT_key[1] == c->vbuf2.p &&
      c->tmaT_key[2] == reinterpret_cast<const void*>((intptr_t)ld))
    return PB_OK;
  c->tmaT_ok = false;
  if (!want) return PB_OK;
  const EncodeTiledFn enc = tensor_map_encoder();
  if (!enc) return PB_OK;
  const int d = c->lay_d, nsp = c->lay_nsp;
  CUtensorMap maps[2];
  for (int k = 0; k < 2; ++k) {
    const cuuint64_t dims[3] = {(cuuint64_t)ld, (cuuint64_t)d, (cuuint64_t)nsp};
    const cuuint64_t strides[2] = {(cuuint64_t)ld * sizeof(double), (cuuint64_t)d * ld * sizeof(double)};
    const cuuint32_t box[3] = {(cuuint32_t)kSlabCols, 1u, (cuuint32_t)SlabSmem::box_rows(nsp)};
    const cuuint32_t es[3] = {1u, 1u, 1u};
    if (enc(&maps[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, k == 0 ? c->vbuf.p : c->vbuf2.p, dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return PB_OK;
  }
  PB_CUDA(c, c->tmapsT.ensure(sizeof(maps)));
  PB_CUDA(c, cudaMemcpy(c->tmapsT.p, maps, sizeof(maps), cudaMemcpyHostToDevice));
  c->tmaT_key[0] = c->vbuf.p;
  c->tmaT_key[1] = c->vbuf2.p;
  c->tmaT_key[2] = reinterpret_cast<const void*>((intptr_t)ld);
  c->tmaT_ok = true;
  return PB_OK;
}

// Reports a bounded wait that gave up inside a kernel of the last enqueued work.
int check_wait_flag(pb_context* c, const char* who) {
  int herr = 0;
  PB_CUDA(c, cudaMemcpy(&herr, c->d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (herr) return fail(c, PB_ERR_DEVICE, "%s: a CTA gave up waiting for its staging copies (code %d: 1 bin-local rows, 2 band tiles)", who, herr);
  return PB_OK;
}

// The k_slab staging of a stage: the tensor map of its source, or null.
const CUtensorMap* stage_tmap(const pb_context* c, int stage) {
  return c->tma_ok ? reinterpret_cast<const CUtensorMap*>(c->tmaps.p) + (stage == 1 ? 0 : 1) : nullptr;
}
// k_band_tma's map of a stage's source, or null (the cp.async k_band runs).
const CUtensorMap* stage_tmap_band(const pb_context* c, int stage) {
  return (c->tma_ok && c->tma_band_ok && c->band_tma_fits) ? reinterpret_cast<const CUtensorMap*>(c->tmaps.p) + (stage == 1 ? 2 : 3)
                                                          : nullptr;
}

// Whether a solve with K columns runs the bin-blocked kernels.
bool use_blocked(const pb_context* c, int K) {
  const int64_t ld = ((K + kColTile - 1) / kColTile) * kColTile;
  return c->blocked_ok && c->fd_tab_ok && c->batched_mode == 1 && K > 1 && c->n * ld < ((int64_t)1 << 31);
}

// One stage of the bin-blocked path: k_band on the second stream, k_fd then
// k_slab on the launching stream, then k_band_finish (and the next step's row
// factors of the bin-local rows after stage 2).
// k_band's grid for the active columns: column blocks of 8 nw columns and
// mother-species groups (sets p.spg, p.ngroups).  With nw = 8 the groups fill
// at least one wave of the SMs (a CTA per SM); with nw = 4 they stay within one
// wave, so that each SM holds at most one k_band CTA beside its k_slab CTA.
int band_grid(const pb_context* c, StepParams& p, int nw) {
  const int cblocks = (int)blocks_for(p.ncols, 8 * nw);
  const int per = cblocks * std::max(c->band_npairs, 1);
  int G;
  if (nw == 4) {
    G = std::max(1, std::min({c->num_sms / per, kMaxBandGroups, p.nsp}));
  } else {
    // One CTA per SM.  At least one wave of CTAs (measured best up to
    // K = 512); with many column blocks the launch takes ceil(CTAs / SMs)
    // waves of CTAs that each walk ceil(nsp / G) mother species, so G is
    // raised to the one with the fewest waves x species (the smaller on ties,
    // at most 16 beyond one wave's worth: the partial sums grow with G x
    // columns).  At K = 2048 this takes G from 5 to 9 and k_band from 818 to
    // 469 us per launch.
    const int gmax = std::min({kMaxBandGroups, p.nsp, std::max(16, c->num_sms / per)});
    int gw = 1;
    int64_t best = -1;
    for (int g = 1; g <= gmax; ++g) {
      const int64_t waves = ((int64_t)per * g + c->num_sms - 1) / c->num_sms;
      const int64_t cost = waves * ((p.nsp + g - 1) / g);
      if (best < 0 || cost < best) {
        best = cost;
        gw = g;
      }
    }
    const int fill = (c->num_sms + per - 1) / per;
    G = std::max(1, std::min({std::max(fill, gw), kMaxBandGroups, p.nsp}));
  }
  p.spg = (p.nsp + G - 1) / G;
  p.ngroups = (p.nsp + p.spg - 1) / p.spg;
  return cblocks;
}

template <int STAGE>
int64_t launch_blocked_stage(pb_context* c, StepParams& p, cudaStream_t st) {
  const bool photohad = (p.flags & PB_PHOTOHAD) != 0;
  const bool kap = (p.flags & PB_PARTIAL_DIFF) != 0;
  int64_t launches = 0;
  p.ngroups = 0;
  p.spg = 1;
  if (photohad && p.nb > 0) {
    const BandInstance bi = (c->band_warps == 8 && p.tmap_band) ? band_kernel_tma(c->band_RT, c->band_J)
                                                                : band_kernel(c->band_RT, c->band_J, c->band_warps);
    const int cblocks = band_grid(c, p, bi.warps);
    cudaEventRecord(c->ev_fork, st);
    cudaStreamWaitEvent(c->stream2, c->ev_fork, 0);
    bi.fn<<<dim3(cblocks, p.ngroups, c->band_npairs), bi.warps * 32, bi.smem, c->stream2>>>(p);
    cudaEventRecord(c->ev_join, c->stream2);
    ++launches;
  }
  const unsigned tiles = (unsigned)blocks_for(p.ncols, kColTile);
  if (kap) {
    const size_t fsmem = (size_t)p.d * (kColTile + kFdDenseW + 2) * sizeof(double);
    if (c->fd_dense_ok && p.fdkp) k_fd_dense<true><<<dim3(p.nsp, tiles), 256, fsmem, st>>>(p);
    else if (c->fd_dense_ok) k_fd_dense<false><<<dim3(p.nsp, tiles), 256, fsmem, st>>>(p);
    else k_fd<<<dim3(p.nsp, tiles), 256, (size_t)p.d * (kColTile + 2) * sizeof(double), st>>>(p);
    ++launches;
  }
  const dim3 sg(p.d, (unsigned)blocks_for(p.ncols, kSlabCols));
  slab_kernel(STAGE, p.rec_P != nullptr, c->slab_pre)<<<sg, kSlabWarps * 32, c->slab_smem, st>>>(p);
  ++launches;
  if (STAGE == 2 && p.step + 1 < p.n_steps) {
    k_slab_prep<<<blocks_for((int64_t)p.n_slab_spec * p.d, 256), 256, 0, st>>>(p);
    ++launches;
  }
  if (c->n_tail > 0) {  // tail rows (another grid): the general row kernel, a warp per row
    if (c->tail_wait) {  // the previous step's EM hook (on its own stream) writes the tail rows
      cudaStreamWaitEvent(st, c->ev_hook_done, 0);
      c->tail_wait = false;
    }
    StepParams q = p;
    q.rows = c->tail_rows.as<int>();
    q.nrows = c->n_tail;
    q.nsb = (int)blocks_for(q.nrows, 8);
    q.nseg = 0;
    k_step_multi<STAGE><<<dim3((unsigned)q.nsb, tiles), 256, 0, st>>>(q);
    ++launches;
  }
  if (p.ngroups > 0) cudaStreamWaitEvent(st, c->ev_join, 0);
  if (p.nb > 0) {
    k_band_finish<STAGE><<<dim3(blocks_for((int64_t)p.nb * p.d, 8), tiles), 256, 0, st>>>(p);
    ++launches;
  }
  return launches;
}

// One stage of the bin-blocked adjoint sweep: k_bandT on the second stream,
// k_fdT on the launching stream, then k_slabT.
template <int STAGE>
void launch_adj_blocked(pb_context* c, AdjBlk& q, cudaStream_t st) {
  const bool photohad = (q.flags & PB_PHOTOHAD) != 0, kap = (q.flags & PB_PARTIAL_DIFF) != 0;
  const unsigned tiles = (unsigned)blocks_for(q.ncols, kColTile);
  bool forked = false;
  if (photohad && q.nb > 0) {
    const int cblocks = (int)blocks_for(q.ncols, 64);
    const int G = std::max(1, std::min({(c->num_sms + cblocks - 1) / cblocks, kMaxBandGroups, q.nsp}));
    q.spg = (q.nsp + G - 1) / G;
    const int ngroups = (q.nsp + q.spg - 1) / q.spg;
    cudaEventRecord(c->ev_fork, st);
    cudaStreamWaitEvent(c->stream2, c->ev_fork, 0);
    const BandTInstance bi = bandT_kernel(c->band_RT, c->band_J);
    bi.fn<<<dim3(cblocks, ngroups), 256, bi.smem, c->stream2>>>(q);
    cudaEventRecord(c->ev_join, c->stream2);
    forked = true;
  }
  if (kap && c->fdT_dense_ok)
    k_fdT_dense<<<dim3(q.nsp, tiles), 256, (size_t)q.d * (kColTile + kFdDenseW) * sizeof(double), st>>>(q);
  else if (kap)
    k_fdT<<<dim3(q.nsp, tiles), 256, (size_t)q.d * kColTile * sizeof(double), st>>>(q);
  if (forked) cudaStreamWaitEvent(st, c->ev_join, 0);
  k_slabT<STAGE><<<dim3(q.d, (unsigned)blocks_for(q.ncols, kSlabCols)), kSlabTWarps * 32, c->slabT_smem, st>>>(q);
}

// The EM hook's operands for window w on the n x ld buffer X (a state, or the adjoint's lam).
EmParams em_params(const pb_context* c, int w, int ld, int ncols, double* X) {
  EmParams e;
  e.n = c->n;
  e.ld = ld;
  e.ncols = ncols;
  e.n_em = c->em_n;
  e.n_cr = c->em_ncr;
  e.n_bh = c->em_nbh;
  e.g_off = c->em_g;
  e.em_off = c->em_m;
  e.ep_off = c->em_p;
  e.bh_off = c->em_bh_off.as<int64_t>();
  e.bh_A = c->em_bh_A.as<double>();
  e.invE = c->em_invE.as<double>();
  e.dE = c->em_dE.as<double>();
  e.kp = c->kp.as<double>() + (size_t)w * c->n;
  e.dl_step = c->em_dl[w];
  e.Tg = c->em_Tg.as<double>() + (size_t)w * c->em_n * c->em_n;
  e.Te = c->em_Te.as<double>() + (size_t)w * c->em_n * c->em_n;
  e.R = c->em_R.as<double>() + (size_t)w * c->em_n * c->em_ncr;
  e.X = X;
  e.w = c->em_wbuf.as<double>();
  e.es = c->em_es.as<double>();
  e.lep = c->em_lep.as<double>();
  e.y = c->em_y.as<double>();
  e.TgT = c->em_TgT.as<double>() + (size_t)w * c->em_n * c->em_n;
  e.TeT = c->em_TeT.as<double>() + (size_t)w * c->em_n * c->em_n;
  e.RT = c->em_RT.as<double>() + (size_t)w * c->em_n * c->em_ncr;
  return e;
}


// Enqueue the ETD2 steps [k0, k1) on `st`.  Columns [0, n_active[k]) are
// advanced at step k; a step without active columns is skipped (every column
// is still exactly zero).  With `ckpt`, the state before every step k with
// k % every == 0 is copied to checkpoint k / every.  Returns the kernel count.
int64_t launch_steps(pb_context* c, StepParams& p, int K, const int32_t* n_active, int64_t k0, int64_t k1,
                     cudaStream_t st, double* ckpt, int every) {
  const int64_t n = c->n;
  double* X = c->X.as<double>();
  const size_t sbytes = (size_t)n * p.ld * sizeof(double);
  int64_t launches = 0;
  bool prepared = false;
  const bool em = c->have_em && (p.flags & PB_EM_CASCADE);
  // With the EM rows as the tail of the bin-blocked layout, a step's EM hook
  // (it reads the nuclei and writes only the EM rows) runs on stream3 beside
  // the next step's first stage; that stage's tail kernel, and everything
  // after it on the launching stream, waits for it.
  bool hook_pending = false;
  auto join_hook = [&]() {
    if (hook_pending) cudaStreamWaitEvent(st, c->ev_hook_done, 0);
    hook_pending = false;
    c->tail_wait = false;
  };
  for (int64_t k = k0; k < k1; ++k) {
    if (ckpt && every > 0 && k % every == 0) {
      join_hook();
      cudaMemcpyAsync(ckpt + (size_t)(k / every) * n * p.ld, X, sbytes, cudaMemcpyDeviceToDevice, st);
    }
    p.step = k;
    p.step_w = c->h_win[k];
    p.ncols = n_active[k];
    if (p.ncols == 0) continue;
    if (!prepared) {  // row factors of the first active step; later steps get them from stage 2
      k_prep<<<blocks_for(n, 256), 256, 0, st>>>(p);
      ++launches;
      prepared = true;
    }
    const bool blocked = use_blocked(c, K) && (!p.rec_P || p.fdkp || !(p.flags & PB_PAIRPROD));
    const bool overlap = em && blocked && c->n_tail > 0;
    if (!overlap) join_hook();
    c->tail_wait = hook_pending;
    for (int stage = 1; stage <= 2; ++stage) {
      p.src = stage == 1 ? X : c->A.as<double>();
      p.x = X;
      p.xout = X;
      p.tmap_src = blocked ? stage_tmap(c, stage) : nullptr;
      p.tmap_band = blocked ? stage_tmap_band(c, stage) : nullptr;
      p.err = c->d_err.as<int>();
      if (blocked) {
        launches += stage == 1 ? launch_blocked_stage<1>(c, p, st) : launch_blocked_stage<2>(c, p, st);
        continue;
      }
      const unsigned tiles = K == 1 ? 1u : blocks_for(p.ncols, kColTile);
      dim3 grid((unsigned)p.nsb + blocks_for(p.nseg, 8), tiles);
      if (K == 1) {
        if (stage == 1) k_step_plain<1><<<grid, 256, 0, st>>>(p); else k_step_plain<2><<<grid, 256, 0, st>>>(p);
      } else {
        if (stage == 1) k_step_multi<1><<<grid, 256, 0, st>>>(p); else k_step_multi<2><<<grid, 256, 0, st>>>(p);
      }
      ++launches;
    }
    if (c->tail_wait) join_hook();  // no tail launch consumed the wait
    hook_pending = false;
    if (em) {
      const EmParams e = em_params(c, c->h_win[k], p.ld, p.ncols, X);
      if (overlap) {
        cudaEventRecord(c->ev_hook_fork, st);
        cudaStreamWaitEvent(c->stream3, c->ev_hook_fork, 0);
        em_hook_forward(e, c->stream3);
        cudaEventRecord(c->ev_hook_done, c->stream3);
        hook_pending = true;
      } else {
        em_hook_forward(e, st);
      }
      launches += 5;
    }
  }
  join_hook();
  return launches;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

int pb_abi_version(void) { return kAbiVersion; }

const char* pb_global_error(void) { return g_error.c_str(); }

const char* pb_last_error(const pb_context* ctx) { return ctx ? ctx->err.c_str() : g_error.c_str(); }

int pb_create(int device, pb_context** out) {
  if (!out) return fail(nullptr, PB_ERR_ARG, "pb_create: out is NULL");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(nullptr, PB_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
  if (device < 0 || device >= ndev) return fail(nullptr, PB_ERR_ARG, "device %d out of range [0,%d)", device, ndev);
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(nullptr, PB_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  if (prop.major < 10)
    return fail(nullptr, PB_ERR_CUDA, "device %d is sm_%d%d; this build targets sm_100a", device, prop.major, prop.minor);
  pb_context* c = new pb_context();
  c->device = device;
  c->num_sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaEventCreate(&c->ev2) != cudaSuccess || cudaEventCreate(&c->ev3) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream3, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_hook_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_hook_done, cudaEventDisableTiming) != cudaSuccess) {
    delete c;
    return fail(nullptr, PB_ERR_CUDA, "stream/event creation failed");
  }
  e = cudaFuncSetAttribute(k_fold_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (kFoldBM + kFoldBN) * (kMaxPhoton + 4) * (int)sizeof(double));
  if (e != cudaSuccess) {
    pb_destroy(c);
    return fail(nullptr, PB_ERR_CUDA, "cudaFuncSetAttribute(k_fold_gemm): %s", cudaGetErrorString(e));
  }
  *out = c;
  return PB_OK;
}

void pb_destroy(pb_context* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->stream2) cudaStreamSynchronize(c->stream2);
  if (c->stream3) cudaStreamSynchronize(c->stream3);
  for (DBuf* b : all_buffers(c)) b->release();
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->graph_exec2) cudaGraphExecDestroy(c->graph_exec2);
  cudaEventDestroy(c->ev0);
  cudaEventDestroy(c->ev1);
  cudaEventDestroy(c->ev2);
  cudaEventDestroy(c->ev3);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->stream2) cudaStreamDestroy(c->stream2);
  if (c->ev_hook_fork) cudaEventDestroy(c->ev_hook_fork);
  if (c->ev_hook_done) cudaEventDestroy(c->ev_hook_done);
  if (c->stream3) cudaStreamDestroy(c->stream3);
  cudaStreamDestroy(c->stream);
  delete c;
}

int pb_set_coupling(pb_context* c, int64_t n, int64_t R, const int64_t* indptr, const int32_t* indices) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (n <= 0 || R < 0 || !indptr || (R > 0 && !indices)) return fail(c, PB_ERR_ARG, "pb_set_coupling: bad arguments");
  if (n >= (int64_t)1 << 31 || R >= (int64_t)1 << 31) return fail(c, PB_ERR_ARG, "pb_set_coupling: sizes exceed int32 indexing");
  if (indptr[0] != 0 || indptr[n] != R) return fail(c, PB_ERR_ARG, "pb_set_coupling: indptr must run from 0 to n_entries");
  for (int64_t i = 0; i < n; ++i)
    if (indptr[i + 1] < indptr[i]) return fail(c, PB_ERR_ARG, "pb_set_coupling: indptr not monotone at row %lld", (long long)i);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = indptr[i]; j < indptr[i + 1]; ++j) {
      if (indices[j] < 0 || indices[j] >= n) return fail(c, PB_ERR_ARG, "pb_set_coupling: column %d out of range", indices[j]);
      if (j > indptr[i] && indices[j] <= indices[j - 1]) return fail(c, PB_ERR_ARG, "pb_set_coupling: columns not strictly increasing in row %lld", (long long)i);
    }
  int rc = set_device(c);
  if (rc) return rc;
  c->n = n;
  c->R = R;
  c->h_cpl_indptr.assign(indptr, indptr + n + 1);
  c->h_cpl_indices.assign(indices, indices + R);
  c->blocked_ok = false;
  c->lay_d = c->lay_nsp = 0;
  c->lay_nu = n;
  c->n_tail = 0;
  c->have_row_map = false;
  if ((rc = upload(c, c->cpl_indptr, indptr, (size_t)n + 1))) return rc;
  if ((rc = upload(c, c->cpl_indices, indices, (size_t)R))) return rc;
  PB_CUDA(c, c->cpl_row.ensure((size_t)std::max<int64_t>(R, 1) * sizeof(int)));
  PB_CUDA(c, c->cpl_is_diag.ensure((size_t)std::max<int64_t>(R, 1) * sizeof(int)));
  if (R > 0)
    k_coupling_rows<<<blocks_for(n, 8), 256, 0, c->stream>>>(c->cpl_indptr.as<int64_t>(), n,
                                                             c->cpl_indices.as<int>(), c->cpl_row.as<int>(),
                                                             c->cpl_is_diag.as<int>());
  PB_CUDA(c, cudaGetLastError());
  c->h_short_rows.clear();
  c->h_long_rows.clear();
  for (int64_t i = 0; i < n; ++i) (indptr[i + 1] - indptr[i] > kLongRow ? c->h_long_rows : c->h_short_rows).push_back((int)i);
  std::vector<int64_t> scb, sce;
  std::vector<int32_t> slr, l0, ln;
  for (size_t lr = 0; lr < c->h_long_rows.size(); ++lr) {
    const int r = c->h_long_rows[lr];
    l0.push_back((int32_t)scb.size());
    for (int64_t j = indptr[r]; j < indptr[r + 1]; j += kSegLen) {
      scb.push_back(j);
      sce.push_back(std::min<int64_t>(j + kSegLen, indptr[r + 1]));
      slr.push_back((int32_t)lr);
    }
    ln.push_back((int32_t)scb.size() - l0.back());
  }
  c->n_seg = (int32_t)scb.size();
  if ((rc = upload(c, c->short_rows, c->h_short_rows.data(), c->h_short_rows.size()))) return rc;
  if ((rc = upload(c, c->long_rows, c->h_long_rows.data(), c->h_long_rows.size()))) return rc;
  if ((rc = upload(c, c->seg_cb, scb.data(), scb.size()))) return rc;
  if ((rc = upload(c, c->seg_ce, sce.data(), sce.size()))) return rc;
  if ((rc = upload(c, c->seg_lr, slr.data(), slr.size()))) return rc;
  if ((rc = upload(c, c->lr_seg0, l0.data(), l0.size()))) return rc;
  if ((rc = upload(c, c->lr_nseg, ln.data(), ln.size()))) return rc;
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->have_coupling = true;
  c->have_kernel = false;
  c->have_fd = c->have_losses = c->have_decay = c->have_em = false;
  c->em_W = 0;
  c->n_src = 0;
  c->have_solution = false;
  return PB_OK;
}

int pb_set_fold_kernel(pb_context* c, int64_t R, int32_t dph, const double* K) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_coupling) return fail(c, PB_ERR_STATE, "pb_set_fold_kernel: set the coupling pattern first");
  if (R != c->R) return fail(c, PB_ERR_ARG, "pb_set_fold_kernel: %lld rows, coupling has %lld entries", (long long)R, (long long)c->R);
  if (dph <= 0 || dph > kMaxPhoton) return fail(c, PB_ERR_ARG, "pb_set_fold_kernel: photon bins must be in [1, %d]", kMaxPhoton);
  if (R > 0 && !K) return fail(c, PB_ERR_ARG, "pb_set_fold_kernel: kernel is NULL");
  if (c->have_photon_grid && dph != c->dph) return fail(c, PB_ERR_ARG, "pb_set_fold_kernel: photon axis %d != photon grid %d", dph, c->dph);
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = upload(c, c->kernel, K, (size_t)R * dph))) return rc;
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->dph = dph;
  c->have_kernel = true;
  return PB_OK;
}

int pb_build_fold_kernel(pb_context* c, const pb_kernel_spec* k) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!k) return fail(c, PB_ERR_ARG, "pb_build_fold_kernel: spec is NULL");
  if (!c->have_coupling) return fail(c, PB_ERR_STATE, "pb_build_fold_kernel: set the coupling pattern first");
  const int d = k->d, dph = k->dph;
  if (d < 1 || c->lay_nu % d != 0)
    return fail(c, PB_ERR_ARG, "pb_build_fold_kernel: d = %d does not divide the %lld block states", d, (long long)c->lay_nu);
  if (c->h_cpl_indptr[c->lay_nu] != c->R)
    return fail(c, PB_ERR_ARG, "pb_build_fold_kernel: coupling entries in the tail rows");
  for (int64_t j = 0; j < c->R; ++j)
    if (c->h_cpl_indices[j] >= c->lay_nu) return fail(c, PB_ERR_ARG, "pb_build_fold_kernel: coupling entries in the tail columns");
  if (dph <= 0 || dph > kMaxPhoton) return fail(c, PB_ERR_ARG, "pb_build_fold_kernel: photon bins must be in [1, %d]", kMaxPhoton);
  if (c->have_photon_grid && dph != c->dph) return fail(c, PB_ERR_ARG, "pb_build_fold_kernel: photon axis %d != photon grid %d", dph, c->dph);
  if (!k->f_mo || !k->dE || k->n_resp < 0 || k->n_ddr < 0 || k->n_sep < 0 || k->n_channels < 1 || !k->channels ||
      (c->R > 0 && !k->entry_channel) || (k->n_resp > 0 && !k->resp) || (k->n_ddr > 0 && !k->ddr) ||
      (k->n_sep > 0 && (!k->sep_a || !k->sep_b)))
    return fail(c, PB_ERR_ARG, "pb_build_fold_kernel: bad arguments");
  for (int q = 0; q < k->n_channels; ++q) {
    const int kind = k->channels[4 * q], p1 = k->channels[4 * q + 1], p2 = k->channels[4 * q + 2];
    const int n1 = kind == 0 ? k->n_resp : kind == 1 ? k->n_ddr : kind == 2 ? k->n_sep : -1;
    if (n1 < 0) return fail(c, PB_ERR_ARG, "pb_build_fold_kernel: channel %d has unknown kind %d", q, kind);
    if (p1 < (kind == 0 ? -1 : 0) || p1 >= n1 || p2 < -1 || p2 >= k->n_resp)
      return fail(c, PB_ERR_ARG, "pb_build_fold_kernel: channel %d indexes outside its tables", q);
  }
  for (int64_t e = 0; e < c->R; ++e)
    if (k->entry_channel[e] < 0 || k->entry_channel[e] >= k->n_channels)
      return fail(c, PB_ERR_ARG, "pb_build_fold_kernel: entry %lld has channel %d", (long long)e, k->entry_channel[e]);
  int rc = set_device(c);
  if (rc) return rc;
  const size_t na = (size_t)d + dph - 1, nb = 2 * (size_t)d - 1;
  DBuf fm, de, rs, dd, sa, sb, ch, ec;
  auto cleanup = [&]() { for (DBuf* b : {&fm, &de, &rs, &dd, &sa, &sb, &ch, &ec}) b->release(); };
  const double zero = 0.0;
  const int32_t izero = 0;
  if ((rc = upload(c, fm, k->f_mo, (size_t)d)) || (rc = upload(c, de, k->dE, (size_t)d)) ||
      (rc = upload(c, rs, k->n_resp ? k->resp : &zero, k->n_resp ? (size_t)k->n_resp * na : 1)) ||
      (rc = upload(c, dd, k->n_ddr ? k->ddr : &zero, k->n_ddr ? (size_t)k->n_ddr * na * nb : 1)) ||
      (rc = upload(c, sa, k->n_sep ? k->sep_a : &zero, k->n_sep ? (size_t)k->n_sep * na : 1)) ||
      (rc = upload(c, sb, k->n_sep ? k->sep_b : &zero, k->n_sep ? (size_t)k->n_sep * nb : 1)) ||
      (rc = upload(c, ch, k->channels, (size_t)4 * k->n_channels)) ||
      (rc = upload(c, ec, c->R ? k->entry_channel : &izero, c->R ? (size_t)c->R : 1))) {
    cleanup();
    return rc;
  }
  if (c->kernel.ensure((size_t)std::max<int64_t>(c->R, 1) * dph * sizeof(double)) != cudaSuccess) {
    cleanup();
    return fail(c, PB_ERR_CUDA, "pb_build_fold_kernel: allocation of the %lld x %d kernel failed", (long long)c->R, dph);
  }
  const int64_t total = c->R * (int64_t)dph;
  if (total > 0)
    k_build_kernel<<<blocks_for(total, 256), 256, 0, c->stream>>>(
        c->cpl_row.as<int>(), c->cpl_indices.as<int>(), ec.as<int>(), ch.as<int>(), fm.as<double>(), de.as<double>(),
        rs.as<double>(), dd.as<double>(), sa.as<double>(), sb.as<double>(), d, dph, total, c->kernel.as<double>());
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cleanup();
  if (e != cudaSuccess) return fail(c, PB_ERR_CUDA, "pb_build_fold_kernel: %s", cudaGetErrorString(e));
  c->dph = dph;
  c->have_kernel = true;
  return PB_OK;
}

int pb_get_fold_kernel(pb_context* c, int64_t R, int32_t dph, double* K) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_kernel) return fail(c, PB_ERR_STATE, "pb_get_fold_kernel: no fold kernel on the device");
  if (R != c->R || dph != c->dph || (R > 0 && !K))
    return fail(c, PB_ERR_ARG, "pb_get_fold_kernel: the kernel is %lld x %d", (long long)c->R, c->dph);
  if (R == 0) return PB_OK;
  int rc = set_device(c);
  if (rc) return rc;
  PB_CUDA(c, cudaMemcpyAsync(K, c->kernel.p, (size_t)R * dph * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  return PB_OK;
}

int pb_set_photon_grid(pb_context* c, int32_t dph, const double* e) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (dph <= 0 || dph > kMaxPhoton || !e) return fail(c, PB_ERR_ARG, "pb_set_photon_grid: bad arguments");
  if (c->have_kernel && dph != c->dph) return fail(c, PB_ERR_ARG, "pb_set_photon_grid: %d bins, fold kernel has %d", dph, c->dph);
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = upload(c, c->eph, e, (size_t)dph))) return rc;
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->dph = dph;
  c->have_photon_grid = true;
  return PB_OK;
}

int pb_set_photon_field(pb_context* c, int32_t n_comp, const int32_t* kinds, const double* params) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (n_comp < 1 || n_comp > 8 || !kinds || !params) return fail(c, PB_ERR_ARG, "pb_set_photon_field: 1..8 components required");
  for (int i = 0; i < n_comp; ++i) {
    if (kinds[i] < 0 || kinds[i] > 3) return fail(c, PB_ERR_ARG, "pb_set_photon_field: unknown kind %d", kinds[i]);
    if (kinds[i] == 3 && c->tab_nz == 0)
      return fail(c, PB_ERR_STATE, "pb_set_photon_field: a tabulated component needs pb_set_photon_table first");
    if ((kinds[i] == 0 || kinds[i] == 2) && !(params[3 * i + 1] > 0.0))
      return fail(c, PB_ERR_ARG, "pb_set_photon_field: temperature must be positive");
    c->comp_kind[i] = kinds[i];
    for (int q = 0; q < 3; ++q) c->comp_par[i][q] = params[3 * i + q];
  }
  c->n_comp = n_comp;
  c->have_field = true;
  return PB_OK;
}

int pb_set_photon_table(pb_context* c, int32_t nz, int32_t ne, const double* z, const double* log10_e,
                        const double* log10_density) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (nz < 2 || ne < 2 || !z || !log10_e || !log10_density)
    return fail(c, PB_ERR_ARG, "pb_set_photon_table: need at least 2 x 2 points and all three arrays");
  for (int i = 1; i < nz; ++i)
    if (!(z[i] > z[i - 1])) return fail(c, PB_ERR_ARG, "pb_set_photon_table: redshifts must increase");
  for (int j = 1; j < ne; ++j)
    if (!(log10_e[j] > log10_e[j - 1])) return fail(c, PB_ERR_ARG, "pb_set_photon_table: energies must increase");
  for (int64_t k = 0; k < (int64_t)nz * ne; ++k)
    if (!std::isfinite(log10_density[k])) return fail(c, PB_ERR_ARG, "pb_set_photon_table: non-finite density entry %lld", (long long)k);
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = upload(c, c->tab_z, z, (size_t)nz)) || (rc = upload(c, c->tab_le, log10_e, (size_t)ne)) ||
      (rc = upload(c, c->tab_v, log10_density, (size_t)nz * ne)))
    return rc;
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->tab_nz = nz;
  c->tab_ne = ne;
  return PB_OK;
}

// Per-bin FD stencil of the bin-blocked kernels: the off-diagonal entries of
// the FD operator's row e, which must be the same (offsets and values) in
// every species block; padded to kFdMax terms with zero weights on the row
// itself.  Sets fd_tab_ok.
static int build_fd_table(pb_context* c) {
  c->fd_tab_ok = false;
  c->fdT_ok = false;
  const int d = c->lay_d;
  if (!c->have_fd || d <= 0 || c->h_d_indptr.size() != (size_t)c->n + 1) return PB_OK;
  const int nsp = (int)(c->lay_nu / d);
  {  // the species blocks' stencils stay inside the blocks
    const std::vector<int64_t>& ip0 = c->h_d_indptr;
    for (int64_t j = 0; j < ip0[c->lay_nu]; ++j)
      if (c->h_d_indices[j] >= c->lay_nu) return PB_OK;
  }
  const std::vector<int64_t>& ip = c->h_d_indptr;
  const std::vector<int32_t>& ix = c->h_d_indices;
  const std::vector<double>& dv = c->h_d_vals;
  std::vector<int32_t> cnt(d, 0), off((size_t)d * kFdMax, 0);
  std::vector<double> val((size_t)d * kFdMax, 0.0);
  for (int e = 0; e < d; ++e) {
    const int64_t n0 = ip[e + 1] - ip[e];
    if (n0 > kFdMax) return PB_OK;
    cnt[e] = (int32_t)n0;
    for (int64_t t = 0; t < n0; ++t) {
      off[(size_t)e * kFdMax + t] = ix[ip[e] + t] - e;
      val[(size_t)e * kFdMax + t] = dv[ip[e] + t];
    }
    for (int sp = 1; sp < nsp; ++sp) {
      const int64_t r = (int64_t)sp * d + e;
      if (ip[r + 1] - ip[r] != n0) return PB_OK;
      for (int64_t t = 0; t < n0; ++t)
        if (ix[ip[r] + t] - r != off[(size_t)e * kFdMax + t] || dv[ip[r] + t] != val[(size_t)e * kFdMax + t])
          return PB_OK;
    }
  }
  // the transposed stencil: column e of the block receives from rows e + off
  std::vector<int32_t> tcnt(d, 0), toff((size_t)d * kFdTMax, 0);
  std::vector<double> tval((size_t)d * kFdTMax, 0.0);
  bool t_ok = true;
  for (int e = 0; e < d; ++e)      // row e, in row order, so each column's list is in row order
    for (int t = 0; t < cnt[e]; ++t) {
      const int cidx = e + off[(size_t)e * kFdMax + t];
      if (tcnt[cidx] >= kFdTMax) { t_ok = false; continue; }
      toff[(size_t)cidx * kFdTMax + tcnt[cidx]] = e - cidx;
      tval[(size_t)cidx * kFdTMax + tcnt[cidx]] = val[(size_t)e * kFdMax + t];
      ++tcnt[cidx];
    }
  // dense form for k_fd_dense: weights of offsets -kFdHalo..kFdHalo per bin (zeros
  // where the stencil has no term), usable when the terms are in ascending
  // offset order within the halo
  std::vector<double> dense((size_t)d * kFdDenseW, 0.0);
  bool dense_ok = true;
  for (int e = 0; e < d && dense_ok; ++e)
    for (int t = 0; t < cnt[e]; ++t) {
      const int o = off[(size_t)e * kFdMax + t];
      if (o < -kFdHalo || o > kFdHalo || o == 0 || (t > 0 && o <= off[(size_t)e * kFdMax + t - 1])) {
        dense_ok = false;
        break;
      }
      dense[(size_t)e * kFdDenseW + o + kFdHalo] = val[(size_t)e * kFdMax + t];
    }
  // k_fd_dense's shared memory stays within the default 48 KB dynamic limit
  dense_ok = dense_ok && (size_t)d * (kColTile + kFdDenseW + 2) * sizeof(double) <= 48 * 1024;
  int rc;
  c->fd_dense_ok = false;
  if (dense_ok) {
    if ((rc = upload(c, c->fd_dense, dense.data(), dense.size()))) return rc;
    c->fd_dense_ok = true;
  }
  if ((rc = upload(c, c->fd_cnt, cnt.data(), cnt.size()))) return rc;
  if ((rc = upload(c, c->fd_off, off.data(), off.size()))) return rc;
  if ((rc = upload(c, c->fd_val, val.data(), val.size()))) return rc;
  // dense form of the transposed stencil for k_fdT_dense (column lists are in
  // row order, i.e. ascending offsets)
  std::vector<double> tdense((size_t)d * kFdDenseW, 0.0);
  bool tdense_ok = t_ok && (size_t)d * (kColTile + kFdDenseW) * sizeof(double) <= 48 * 1024;
  for (int e = 0; e < d && tdense_ok; ++e)
    for (int t = 0; t < tcnt[e]; ++t) {
      const int o = toff[(size_t)e * kFdTMax + t];
      if (o < -kFdHalo || o > kFdHalo || o == 0 || (t > 0 && o <= toff[(size_t)e * kFdTMax + t - 1])) {
        tdense_ok = false;
        break;
      }
      tdense[(size_t)e * kFdDenseW + o + kFdHalo] = tval[(size_t)e * kFdTMax + t];
    }
  c->fdT_dense_ok = false;
  if (tdense_ok) {
    if ((rc = upload(c, c->fdT_dense, tdense.data(), tdense.size()))) return rc;
    c->fdT_dense_ok = true;
  }
  if (t_ok) {
    if ((rc = upload(c, c->fdT_cnt, tcnt.data(), tcnt.size()))) return rc;
    if ((rc = upload(c, c->fdT_off, toff.data(), toff.size()))) return rc;
    if ((rc = upload(c, c->fdT_val, tval.data(), tval.size()))) return rc;
  }
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->fd_tab_ok = true;
  c->fdT_ok = t_ok;
  return PB_OK;
}

int pb_set_fd_operator(pb_context* c, int64_t nnz, const int64_t* indptr, const int32_t* indices,
                       const double* values, const double* diag) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_coupling) return fail(c, PB_ERR_STATE, "pb_set_fd_operator: set the coupling pattern first");
  if (nnz < 0 || !indptr || !diag || (nnz > 0 && (!indices || !values))) return fail(c, PB_ERR_ARG, "pb_set_fd_operator: bad arguments");
  if (indptr[0] != 0 || indptr[c->n] != nnz) return fail(c, PB_ERR_ARG, "pb_set_fd_operator: indptr must run from 0 to nnz");
  for (int64_t j = 0; j < nnz; ++j)
    if (indices[j] < 0 || indices[j] >= c->n) return fail(c, PB_ERR_ARG, "pb_set_fd_operator: column out of range");
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = upload(c, c->d_indptr, indptr, (size_t)c->n + 1))) return rc;
  if ((rc = upload(c, c->d_indices, indices, (size_t)nnz))) return rc;
  if ((rc = upload(c, c->d_vals, values, (size_t)nnz))) return rc;
  if ((rc = upload(c, c->d_diag, diag, (size_t)c->n))) return rc;
  {
    std::vector<int64_t> tip;
    std::vector<int32_t> tix;
    std::vector<double> tv;
    csr_transpose(c->n, nnz, indptr, indices, values, tip, tix, tv);
    if ((rc = upload(c, c->dt_indptr, tip.data(), tip.size()))) return rc;
    if ((rc = upload(c, c->dt_indices, tix.data(), tix.size()))) return rc;
    if ((rc = upload(c, c->dt_vals, tv.data(), tv.size()))) return rc;
    PB_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->nnzD = nnz;
  c->have_fd = true;
  c->h_d_indptr.assign(indptr, indptr + c->n + 1);
  c->h_d_indices.assign(indices, indices + nnz);
  c->h_d_vals.assign(values, values + nnz);
  return build_fd_table(c);
}

int pb_set_losses(pb_context* c, const double* adia_energy, const double* pair_scale, const int32_t* pair_bin,
                  int32_t n_cr_bins, int32_t n_xi, const double* xi, const double* phi_xi2, const double* pg) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_coupling) return fail(c, PB_ERR_STATE, "pb_set_losses: set the coupling pattern first");
  if (!adia_energy || !pair_scale || !pair_bin || n_cr_bins <= 0 || n_xi < 2 || !xi || !phi_xi2 || !pg)
    return fail(c, PB_ERR_ARG, "pb_set_losses: bad arguments");
  for (int64_t r = 0; r < c->n; ++r)
    if (pair_bin[r] < -1 || pair_bin[r] >= n_cr_bins) return fail(c, PB_ERR_ARG, "pb_set_losses: pair_bin out of range");
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = upload(c, c->adia_E, adia_energy, (size_t)c->n))) return rc;
  if ((rc = upload(c, c->pair_scale, pair_scale, (size_t)c->n))) return rc;
  if ((rc = upload(c, c->pair_bin, pair_bin, (size_t)c->n))) return rc;
  if ((rc = upload(c, c->xi, xi, (size_t)n_xi))) return rc;
  if ((rc = upload(c, c->phi_xi2, phi_xi2, (size_t)n_xi))) return rc;
  if ((rc = upload(c, c->pair_pg, pg, (size_t)n_cr_bins * n_xi))) return rc;
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->n_cr_bins = n_cr_bins;
  c->n_xi = n_xi;
  c->have_losses = true;
  return PB_OK;
}

int pb_set_decay(pb_context* c, const double* diag, int64_t nnz, const int64_t* indptr, const int32_t* indices,
                 const double* values) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_coupling) return fail(c, PB_ERR_STATE, "pb_set_decay: set the coupling pattern first");
  if (nnz < 0 || (nnz > 0 && (!indptr || !indices || !values))) return fail(c, PB_ERR_ARG, "pb_set_decay: bad arguments");
  int rc = set_device(c);
  if (rc) return rc;
  std::vector<double> zero;
  if (!diag) zero.assign((size_t)c->n, 0.0);
  if ((rc = upload(c, c->l_diag, diag ? diag : zero.data(), (size_t)c->n))) return rc;
  std::vector<int64_t> zp;
  if (nnz == 0 || !indptr) {
    zp.assign((size_t)c->n + 1, 0);
    indptr = zp.data();
  } else {
    if (indptr[0] != 0 || indptr[c->n] != nnz) return fail(c, PB_ERR_ARG, "pb_set_decay: indptr must run from 0 to nnz");
    for (int64_t j = 0; j < nnz; ++j)
      if (indices[j] < 0 || indices[j] >= c->n) return fail(c, PB_ERR_ARG, "pb_set_decay: column out of range");
  }
  if ((rc = upload(c, c->l_indptr, indptr, (size_t)c->n + 1))) return rc;
  if ((rc = upload(c, c->l_indices, indices, (size_t)nnz))) return rc;
  if ((rc = upload(c, c->l_vals, values, (size_t)nnz))) return rc;
  {
    std::vector<int64_t> tip;
    std::vector<int32_t> tix;
    std::vector<double> tv;
    csr_transpose(c->n, nnz, indptr, indices, values, tip, tix, tv);
    if ((rc = upload(c, c->lt_indptr, tip.data(), tip.size()))) return rc;
    if ((rc = upload(c, c->lt_indices, tix.data(), tix.size()))) return rc;
    if ((rc = upload(c, c->lt_vals, tv.data(), tv.size()))) return rc;
    PB_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->nnzL = nnz;
  c->have_decay = true;
  return PB_OK;
}

int pb_set_injection(pb_context* c, int32_t n_src, int32_t n_rows, const int32_t* rows, const double* grids,
                     int32_t n_cols, const int32_t* src_col) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_coupling) return fail(c, PB_ERR_STATE, "pb_set_injection: set the coupling pattern first");
  if (n_src < 0 || n_rows < 0 || n_cols < 1 || (n_src > 0 && (!src_col || (n_rows > 0 && (!rows || !grids)))))
    return fail(c, PB_ERR_ARG, "pb_set_injection: bad arguments");
  std::vector<int32_t> slot((size_t)c->n, -1);
  for (int i = 0; i < n_rows; ++i) {
    if (rows[i] < 0 || rows[i] >= c->n) return fail(c, PB_ERR_ARG, "pb_set_injection: row out of range");
    if (slot[rows[i]] >= 0) return fail(c, PB_ERR_ARG, "pb_set_injection: duplicated row %d", rows[i]);
    slot[rows[i]] = i;
  }
  std::vector<int32_t> ptr((size_t)n_cols + 1, 0);
  for (int s = 0; s < n_src; ++s) {
    if (src_col[s] < 0 || src_col[s] >= n_cols) return fail(c, PB_ERR_ARG, "pb_set_injection: src_col out of range");
    if (s > 0 && src_col[s] < src_col[s - 1]) return fail(c, PB_ERR_ARG, "pb_set_injection: src_col must be non-decreasing");
    ptr[src_col[s] + 1]++;
  }
  for (int k = 0; k < n_cols; ++k) ptr[k + 1] += ptr[k];
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = upload(c, c->inj_slot, slot.data(), slot.size()))) return rc;
  if ((rc = upload(c, c->inj_G, grids, (size_t)n_rows * n_src))) return rc;
  if ((rc = upload(c, c->src_ptr, ptr.data(), ptr.size()))) return rc;
  if ((rc = upload(c, c->inj_rows, rows, (size_t)n_rows))) return rc;
  if ((rc = upload(c, c->src_col_d, src_col, (size_t)n_src))) return rc;
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->n_src = n_src;
  c->n_inj_rows = n_rows;
  c->n_src_cols = n_cols;
  return PB_OK;
}

int pb_set_row_map(pb_context* c, const int32_t* caller_row) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_coupling) return fail(c, PB_ERR_STATE, "pb_set_row_map: set the coupling pattern first");
  if (!caller_row) {
    c->have_row_map = false;
    return PB_OK;
  }
  std::vector<char> seen((size_t)c->n, 0);
  for (int64_t i = 0; i < c->n; ++i) {
    const int32_t r = caller_row[i];
    if (r < 0 || r >= c->n || seen[r]) return fail(c, PB_ERR_ARG, "pb_set_row_map: not a permutation (row %lld)", (long long)i);
    seen[r] = 1;
  }
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = upload(c, c->row_map, caller_row, (size_t)c->n))) return rc;
  c->have_row_map = true;
  return PB_OK;
}

int pb_set_layout(pb_context* c, int32_t d) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  return pb_set_layout_rows(c, d, c->n);
}

int pb_set_layout_rows(pb_context* c, int32_t d, int64_t n_blocks) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_coupling) return fail(c, PB_ERR_STATE, "pb_set_layout: set the coupling pattern first");
  if (n_blocks <= 0 || n_blocks > c->n)
    return fail(c, PB_ERR_ARG, "pb_set_layout_rows: %lld block rows outside [1, %lld]", (long long)n_blocks, (long long)c->n);
  if (d <= 0 || n_blocks % d != 0)
    return fail(c, PB_ERR_ARG, "pb_set_layout: %lld states are not blocks of %d bins", (long long)n_blocks, d);
  int rc = set_device(c);
  if (rc) return rc;
  const int64_t n = c->n, R = c->R;
  const int nsp = (int)(n_blocks / d);
  const std::vector<int64_t>& ip = c->h_cpl_indptr;
  const std::vector<int32_t>& ix = c->h_cpl_indices;
  // the tail: rows past the species blocks, stepped by the general row kernel
  c->lay_nu = n_blocks;
  c->n_tail = (int32_t)(n - n_blocks);
  if (c->n_tail > 0) {
    std::vector<int32_t> tr((size_t)c->n_tail);
    for (int32_t i = 0; i < c->n_tail; ++i) tr[i] = (int32_t)(n_blocks + i);
    if ((rc = upload(c, c->tail_rows, tr.data(), tr.size()))) return rc;
  }
  // the bin-blocked kernels need the coupling block-diagonal over (blocks, tail)
  bool split_ok = true;
  for (int64_t r = 0; r < n && split_ok; ++r)
    for (int64_t j = ip[r]; j < ip[r + 1]; ++j)
      if ((r < n_blocks) != (ix[j] < n_blocks)) { split_ok = false; break; }
  // band species: rows with an off-diagonal entry that leaves the row's bin
  std::vector<int32_t> bspec, sspec;
  int lo = 1 << 30, hi = -(1 << 30);
  for (int sp = 0; sp < nsp; ++sp) {
    bool band = false;
    for (int64_t r = (int64_t)sp * d; r < (int64_t)(sp + 1) * d && !band; ++r)
      for (int64_t j = ip[r]; j < ip[r + 1]; ++j)
        if (ix[j] != r && ix[j] % d != r % d) { band = true; break; }
    (band ? bspec : sspec).push_back(sp);
  }
  for (int32_t sp : bspec)
    for (int64_t r = (int64_t)sp * d; r < (int64_t)(sp + 1) * d; ++r)
      for (int64_t j = ip[r]; j < ip[r + 1]; ++j) {
        if (ix[j] == r) continue;
        const int off = ix[j] % d - (int)(r % d);
        lo = std::min(lo, off);
        hi = std::max(hi, off);
      }
  {  // bin-local species by coupling entries, longest rows first (k_slab's warps take rows strided)
    std::vector<int64_t> cnt(nsp, 0);
    for (int32_t sp : sspec)
      for (int64_t r = (int64_t)sp * d; r < (int64_t)(sp + 1) * d; ++r) cnt[sp] += ip[r + 1] - ip[r];
    std::stable_sort(sspec.begin(), sspec.end(), [&](int32_t a, int32_t b) { return cnt[a] > cnt[b]; });
  }
  c->blocked_ok = false;
  c->band_tma_fits = false;
  c->lay_d = d;
  c->lay_nsp = nsp;
  if ((rc = build_fd_table(c))) return rc;
  const int nb = (int)bspec.size(), nss = (int)sspec.size();
  const int npairs = (nb + 1) / 2;
  const int RTr = (d + 7) / 8;
  const int Jr = bspec.empty() ? 1 : (7 + hi) / 4 + 1;
  int RT = 0, J = 0;
  for (int v : kBandRT) if (!RT && v >= RTr) RT = v;
  for (int v : kBandJ) if (!J && v >= Jr) J = v;
  // bin-local rows, per bin: rows ordered by entry quads (longest first) and
  // grouped in quartets, a quarter-warp of k_slab per row; quartets spread
  // over k_slab's warps longest-processing-time first.  Each row's entries in
  // CSR order in quads of 4; zero values pad the row's last quad and the row
  // up to the longest row of its quartet.  The quads of a quartet's four rows
  // interleave (row g's quad t at q0 + 4 t + g), so that the four rows' entry
  // loads fall into distinct shared-memory banks; every bin and quartet starts
  // on a multiple of 4 quads.
  int64_t band_nnz = 0, slab_nnz = 0;
  std::vector<int32_t> qbase((size_t)d + 1, 0), wrp((size_t)d * (kSlabWarps + 1), 0), squart;
  std::vector<unsigned long long> squad;
  std::vector<int32_t> sslot((size_t)std::max<int64_t>(R, 1), -1), rowslot((size_t)n, -1);
  int32_t maxbin = 0;
  // 16-bit slab byte offsets and 16-bit species (0xffff marks an empty quartet row)
  bool quads_fit = (size_t)nsp * kSlabCols * sizeof(double) <= (1 << 16) && nsp < 0xffff;
  {
    std::vector<int32_t> nq(nss), order(nss);
    std::vector<std::vector<int32_t>> wl(kSlabWarps);
    std::vector<int64_t> load(kSlabWarps);
    for (int e = 0; e < d; ++e) {
      qbase[e] = (int32_t)squad.size();
      for (int i = 0; i < nss; ++i) {
        const int64_t r = (int64_t)sspec[i] * d + e;
        int64_t cnt = 0;
        for (int64_t j = ip[r]; j < ip[r + 1]; ++j) cnt += ix[j] != r;
        nq[i] = (int32_t)((cnt + 3) / 4);
        order[i] = i;
      }
      std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return nq[a] > nq[b]; });
      for (auto& v : wl) v.clear();
      std::fill(load.begin(), load.end(), 0);
      for (int k = 0; k < nss; k += kSlabRows) {  // quartet k / 4 = rows order[k .. k + 3], the longest first
        const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        wl[w].push_back(k);
        load[w] += nq[order[k]] + 1;
      }
      for (int w = 0; w < kSlabWarps; ++w) {
        wrp[(size_t)e * (kSlabWarps + 1) + w] = (int32_t)(squart.size() / 4);
        for (int k : wl[w]) {
          const int nqmax = nq[order[k]];
          const int64_t q0 = (int64_t)squad.size() - qbase[e];
          const size_t qa = squad.size();
          squad.resize(qa + (size_t)kSlabRows * nqmax, 0);
          int32_t sp4[kSlabRows] = {0xffff, 0xffff, 0xffff, 0xffff};
          for (int g = 0; g < kSlabRows; ++g) {
            if (k + g >= nss) continue;
            const int i = order[k + g];
            const int64_t r = (int64_t)sspec[i] * d + e;
            int t = 0, pad_sp = sspec[i];
            for (int64_t j = ip[r]; j < ip[r + 1]; ++j) {
              if (ix[j] == r) continue;
              if (t == 0) pad_sp = ix[j] / d;
              const size_t q = qa + (size_t)kSlabRows * (t / 4) + g;
              squad[q] |= (unsigned long long)((ix[j] / d) * kSlabCols * sizeof(double)) << (16 * (t % 4));
              sslot[j] = (int32_t)(q * 4 + t % 4);
              ++slab_nnz;
              ++t;
            }
            for (; t < 4 * nqmax; ++t) {  // zero values on a mother row of the slab
              const size_t q = qa + (size_t)kSlabRows * (t / 4) + g;
              squad[q] |= (unsigned long long)(pad_sp * kSlabCols * sizeof(double)) << (16 * (t % 4));
            }
            sp4[g] = sspec[i];
            rowslot[r] = (int32_t)(squart.size() + g);  // quartet index * 4 + row
          }
          if (q0 >= (1 << 30)) quads_fit = false;
          const int32_t qd[4] = {(int32_t)((uint32_t)sp4[0] | ((uint32_t)sp4[1] << 16)),
                                 (int32_t)((uint32_t)sp4[2] | ((uint32_t)sp4[3] << 16)), (int32_t)q0, nqmax};
          squart.insert(squart.end(), qd, qd + 4);
        }
      }
      wrp[(size_t)e * (kSlabWarps + 1) + kSlabWarps] = (int32_t)(squart.size() / 4);
      maxbin = std::max<int32_t>(maxbin, (int32_t)(squad.size() - qbase[e]));
    }
    qbase[d] = (int32_t)squad.size();
    if (squad.empty()) squad.assign(4, 0);
    if (squart.empty()) squart.assign(4, 0);
  }
  const size_t max_smem = 227 * 1024;
  const size_t ssm = SlabSmem::bytes(nsp, maxbin, (nss + kSlabRows - 1) / kSlabRows);
  const BandInstance bi = (RT && J) ? band_kernel(RT, J) : BandInstance{nullptr, 0, 0};
  const BandInstance bi4 = (RT && J) ? band_kernel(RT, J, 4) : BandInstance{nullptr, 0, 0};
  const bool ok = split_ok && quads_fit && ssm <= max_smem && bi.fn && bi.smem <= max_smem && (bspec.empty() || lo >= 0) &&
                  (size_t)d * (kColTile + 2) * sizeof(double) <= max_smem &&
                  (int64_t)nsp * 2 * npairs * RT * J * 32 < ((int64_t)1 << 31) && squad.size() < ((size_t)1 << 29);
  if (!ok) return PB_OK;  // the general row kernels stay in use
  // band tiles: [species][band pair][2][RT / 2][J][32][2] DMMA A fragments per window
  std::vector<int32_t> bslot((size_t)std::max<int64_t>(R, 1), -1);
  for (int b = 0; b < nb; ++b)
    for (int e = 0; e < d; ++e) {
      const int64_t r = (int64_t)bspec[b] * d + e;
      const int rt = e / 8;
      for (int64_t j = ip[r]; j < ip[r + 1]; ++j) {
        if (ix[j] == r) continue;
        const int sp = ix[j] / d, e2 = ix[j] % d;
        const int jj = e2 / 4 - 2 * rt;
        // row tiles in pairs: lane l holds the fragments of tiles 2p and 2p + 1 side by side
        const size_t tile = ((size_t)sp * 2 * npairs + b) * (RT / 2) + rt / 2;
        bslot[j] = (int32_t)(((tile * J + jj) * 32 + (e % 8) * 4 + (e2 % 4)) * 2 + (rt & 1));
        ++band_nnz;
      }
    }
  if ((rc = upload(c, c->band_slot, bslot.data(), bslot.size()))) return rc;
  if ((rc = upload(c, c->band_spec, bspec.data(), bspec.size()))) return rc;
  if ((rc = upload(c, c->slab_spec, sspec.data(), sspec.size()))) return rc;
  if ((rc = upload(c, c->slab_rp, qbase.data(), qbase.size()))) return rc;
  if ((rc = upload(c, c->slab_sidx, squad.data(), squad.size()))) return rc;
  if ((rc = upload(c, c->slab_quart, squart.data(), squart.size()))) return rc;
  if ((rc = upload(c, c->slab_wrp, wrp.data(), wrp.size()))) return rc;
  if ((rc = upload(c, c->slab_rowslot, rowslot.data(), rowslot.size()))) return rc;
  c->slab_nslots = (int64_t)squart.size();
  PB_CUDA(c, c->slab_fac.ensure((size_t)2 * 3 * c->slab_nslots * sizeof(double)));
  PB_CUDA(c, cudaMemsetAsync(c->slab_fac.p, 0, (size_t)2 * 3 * c->slab_nslots * sizeof(double), c->stream));
  if ((rc = upload(c, c->slab_slot, sslot.data(), sslot.size()))) return rc;
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  std::vector<const void*> slab_fns;
  for (int pre : {1, 2, 3})
    for (int st = 1; st <= 2; ++st)
      for (bool rec : {false, true}) slab_fns.push_back((const void*)slab_kernel(st, rec, pre));
  for (const void* fn : slab_fns) {
    // the attribute belongs to the kernel, not the context: the largest limit,
    // so that a smaller layout on another context never lowers it under ours
    PB_CUDA(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem));
    PB_CUDA(c, cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
  }
  PB_CUDA(c, cudaFuncSetAttribute(bi.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bi.smem));
  PB_CUDA(c, cudaFuncSetAttribute(bi4.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bi4.smem));
  {
    const BandInstance bt = band_kernel_tma(RT, J);
    c->band_tma_fits = bt.fn && bt.smem <= max_smem;
    if (c->band_tma_fits) PB_CUDA(c, cudaFuncSetAttribute(bt.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bt.smem));
  }
  c->band_nb = nb;
  c->band_npairs = npairs;
  c->band_RT = RT;
  c->band_J = J;
  c->band_stride = (int64_t)nsp * 2 * npairs * RT * J * 32;
  c->n_slab_spec = nss;
  c->slab_nent = (int64_t)squad.size() * 4;
  c->slab_maxbin = maxbin;
  c->slab_smem = ssm;
  c->band_smem = bi.smem;
  c->band_nnz = band_nnz;
  c->slab_nnz = slab_nnz;
  c->blocked_ok = true;
  // ---- transposed structures of the adjoint sweep (at most one band pair)
  c->blockedT_ok = false;
  if (npairs > 1) return PB_OK;
  std::vector<int32_t> btslot((size_t)std::max<int64_t>(R, 1), -1);
  for (int b = 0; b < nb; ++b)
    for (int e = 0; e < d; ++e) {
      const int64_t r = (int64_t)bspec[b] * d + e;
      for (int64_t j = ip[r]; j < ip[r + 1]; ++j) {
        if (ix[j] == r) continue;
        const int sp = ix[j] / d, e2 = ix[j] % d;   // mother species and bin
        const int mt = e2 / 8, jj = e / 4 - 2 * mt + (J - 2);
        if (jj < 0 || jj >= J) return PB_OK;
        const size_t tile = ((size_t)sp * 2 + b) * RT + mt;
        btslot[j] = (int32_t)((tile * J + jj) * 32 + (e2 % 8) * 4 + (e % 4));
      }
    }
  // transposed bin-local rows (mothers), per bin: every species is a row; its
  // daughter entries in the order (daughter species in k_slab's species order,
  // CSR order), in quads of 4 (daughter slab byte offsets, zero values pad the
  // last quad); rows paired for k_slabT's half-warps and the pairs spread over
  // its warps longest-processing-time first; every bin starts on an even quad.
  std::vector<std::vector<std::pair<int32_t, int64_t>>> bym(nsp);
  std::vector<int32_t> tqbase((size_t)d + 1, 0), twrp((size_t)d * (kSlabTWarps + 1), 0), tpairs;
  std::vector<unsigned long long> tquad;
  std::vector<int32_t> tslot((size_t)std::max<int64_t>(R, 1), -1);
  int32_t tmax = 0;
  bool tq_fit = (size_t)nsp * kSlabCols * sizeof(double) <= (1 << 16);
  {
    std::vector<int32_t> nqm(nsp), order(nsp);
    std::vector<std::vector<int32_t>> wl(kSlabTWarps);
    std::vector<int64_t> load(kSlabTWarps);
    for (int e = 0; e < d; ++e) {
      for (auto& v : bym) v.clear();
      for (int i = 0; i < nss; ++i) {
        const int64_t r = (int64_t)sspec[i] * d + e;
        for (int64_t j = ip[r]; j < ip[r + 1]; ++j)
          if (ix[j] != r) bym[ix[j] / d].push_back({sspec[i], j});
      }
      tqbase[e] = (int32_t)tquad.size();
      for (int m = 0; m < nsp; ++m) {
        nqm[m] = (int32_t)((bym[m].size() + 3) / 4);
        order[m] = m;
      }
      std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return nqm[a] > nqm[b]; });
      for (auto& v : wl) v.clear();
      std::fill(load.begin(), load.end(), 0);
      for (int k = 0; k < nsp; k += 2) {
        const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        wl[w].push_back(k);
        load[w] += nqm[order[k]] + 1;
      }
      for (int w = 0; w < kSlabTWarps; ++w) {
        twrp[(size_t)e * (kSlabTWarps + 1) + w] = (int32_t)(tpairs.size() / 4);
        for (int k : wl[w]) {
          int32_t pr[4] = {-1, -1, 0, 0};
          for (int hf = 0; hf < 2; ++hf) {
            if (k + hf >= nsp) continue;
            const int m = order[k + hf];
            const int64_t q0 = (int64_t)tquad.size() - tqbase[e];
            int t = 0;
            const unsigned long long pad = bym[m].empty() ? 0ull : (unsigned long long)bym[m][0].first * kSlabCols * sizeof(double);
            for (auto& dj : bym[m]) {
              if (t % 4 == 0) tquad.push_back(0);
              tquad.back() |= ((unsigned long long)dj.first * kSlabCols * sizeof(double)) << (16 * (t % 4));
              tslot[dj.second] = (int32_t)((tquad.size() - 1) * 4 + t % 4);
              ++t;
            }
            for (; t % 4; ++t) tquad.back() |= pad << (16 * (t % 4));
            if (q0 >= (1 << 15) || nqm[m] >= (1 << 16)) tq_fit = false;
            pr[hf] = m;
            pr[2 + hf] = (int32_t)((q0 << 16) | nqm[m]);
          }
          tpairs.insert(tpairs.end(), pr, pr + 4);
        }
      }
      twrp[(size_t)e * (kSlabTWarps + 1) + kSlabTWarps] = (int32_t)(tpairs.size() / 4);
      if ((tquad.size() - tqbase[e]) % 2) tquad.push_back(0);
      tmax = std::max<int32_t>(tmax, (int32_t)(tquad.size() - tqbase[e]));
    }
    tqbase[d] = (int32_t)tquad.size();
    if (tquad.empty()) tquad.assign(2, 0);
  }
  if (!tq_fit) return PB_OK;
  // at least one double per thread: stage 1 reduces the gradient over the slab's space
  const size_t tsm = std::max(SlabTSmem::bytes(nsp, tmax, (nsp + 1) / 2), (size_t)kSlabTWarps * 32 * sizeof(double));
  const BandTInstance bti = bandT_kernel(RT, J);
  if (tsm > max_smem || !bti.fn || bti.smem > max_smem || (size_t)d * kColTile * sizeof(double) > max_smem) return PB_OK;
  if ((rc = upload(c, c->bandT_slot, btslot.data(), btslot.size()))) return rc;
  if ((rc = upload(c, c->slabT_rp, tqbase.data(), tqbase.size()))) return rc;
  if ((rc = upload(c, c->slabT_offs, tquad.data(), tquad.size()))) return rc;
  if ((rc = upload(c, c->slabT_pairs, tpairs.data(), tpairs.size()))) return rc;
  if ((rc = upload(c, c->slabT_wrp, twrp.data(), twrp.size()))) return rc;
  if ((rc = upload(c, c->slabT_slot, tslot.data(), tslot.size()))) return rc;
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  for (const void* fn : {(const void*)k_slabT<1>, (const void*)k_slabT<2>}) {
    PB_CUDA(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));  // per kernel
    PB_CUDA(c, cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
  }
  PB_CUDA(c, cudaFuncSetAttribute(bti.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bti.smem));
  c->slabT_nent = (int64_t)tquad.size() * 4;
  c->slabT_maxbin = tmax;
  c->slabT_smem = tsm;
  c->bandT_smem = bti.smem;
  c->blockedT_ok = true;
  return PB_OK;
}

int pb_profile_stage(pb_context* c, int64_t step, int32_t stage, int32_t reps, double* ms) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!ms || reps < 1 || (stage != 1 && stage != 2)) return fail(c, PB_ERR_ARG, "pb_profile_stage: bad arguments");
  if (!c->have_solution) return fail(c, PB_ERR_STATE, "pb_profile_stage: run pb_solve first");
  const int K = c->last_K;
  if (!use_blocked(c, K)) return fail(c, PB_ERR_STATE, "pb_profile_stage: the last solve did not run the bin-blocked kernels");
  if (step < 0 || step >= c->last_S || c->h_nact[step] == 0) return fail(c, PB_ERR_ARG, "pb_profile_stage: step without active columns");
  int rc = set_device(c);
  if (rc) return rc;
  const int ld = ((K + kColTile - 1) / kColTile) * kColTile;
  const uint32_t flags = c->last_flags;
  const bool pair = (flags & PB_PAIRPROD) && (flags & PB_PARTIAL_DIFF);
  const bool inj = (flags & PB_INJECTION) && c->n_src > 0;
  StepParams p;
  memset(&p, 0, sizeof(p));
  fill_step_params(c, p, K, ld, flags, pair, inj, c->last_S, ld / kColTile);
  p.step = step;
  p.step_w = c->h_win[step];
  p.ncols = c->h_nact[step];
  p.src = stage == 1 ? c->X.as<double>() : c->A.as<double>();
  p.x = c->X.as<double>();
  p.xout = c->X.as<double>();
  p.tmap_src = stage_tmap(c, stage);
  p.tmap_band = stage_tmap_band(c, stage);
  PB_CUDA(c, c->d_err.ensure(sizeof(int)));
  p.err = c->d_err.as<int>();
  cudaStream_t st = c->stream;
  const bool photohad = (flags & PB_PHOTOHAD) != 0, kap = (flags & PB_PARTIAL_DIFF) != 0;
  const unsigned tiles = (unsigned)blocks_for(p.ncols, kColTile);
  const BandInstance bi = (c->band_warps == 8 && p.tmap_band) ? band_kernel_tma(c->band_RT, c->band_J)
                                                              : band_kernel(c->band_RT, c->band_J, c->band_warps);
  const int cblocks = band_grid(c, p, bi.warps);
  if (!(photohad && p.nb > 0)) p.ngroups = 0;
  for (int kk = 0; kk < 4; ++kk) ms[kk] = 0.0;
  for (int kk = 0; kk < 4; ++kk) {
    const bool runs = kk == 0 ? kap : kk == 1 ? true : kk == 2 ? p.ngroups > 0 : p.nb > 0;
    if (!runs) continue;
    for (int r = -1; r < reps; ++r) {  // one untimed launch first
      PB_CUDA(c, cudaEventRecord(c->ev0, st));
      if (kk == 0) {
        if (c->fd_dense_ok)
          k_fd_dense<false><<<dim3(p.nsp, tiles), 256, (size_t)p.d * (kColTile + kFdDenseW + 2) * sizeof(double), st>>>(p);
        else k_fd<<<dim3(p.nsp, tiles), 256, (size_t)p.d * (kColTile + 2) * sizeof(double), st>>>(p);
      }
      if (kk == 1) {
        const dim3 sg(p.d, (unsigned)blocks_for(p.ncols, kSlabCols));
        slab_kernel(stage, false, c->slab_pre)<<<sg, kSlabWarps * 32, c->slab_smem, st>>>(p);
      }
      if (kk == 2) bi.fn<<<dim3(cblocks, p.ngroups, c->band_npairs), bi.warps * 32, bi.smem, st>>>(p);
      if (kk == 3) {
        const unsigned gb = (unsigned)blocks_for((int64_t)p.nb * p.d, 8);
        if (stage == 1) k_band_finish<1><<<dim3(gb, tiles), 256, 0, st>>>(p);
        else k_band_finish<2><<<dim3(gb, tiles), 256, 0, st>>>(p);
      }
      PB_CUDA(c, cudaGetLastError());
      PB_CUDA(c, cudaEventRecord(c->ev1, st));
      PB_CUDA(c, cudaEventSynchronize(c->ev1));
      float t = 0.f;
      PB_CUDA(c, cudaEventElapsedTime(&t, c->ev0, c->ev1));
      if (r >= 0) ms[kk] += t / reps;
    }
  }
  return PB_OK;
}

// FP64 tensor-pipe throughput probe: independent DMMA m8n8k4 chains in registers.
__global__ void k_fp64_probe(double* out, int iters) {
  double a = 1.0 + threadIdx.x * 1e-9, b = 1.0 - threadIdx.x * 1e-9;
  double cc[8][2];
#pragma unroll
  for (int i = 0; i < 8; ++i) cc[i][0] = cc[i][1] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) dmma884(cc[i][0], cc[i][1], a, b);
  }
  double sum = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) sum += cc[i][0] + cc[i][1];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = sum;
}

int pb_fp64_peak(pb_context* c, double* tflops) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!tflops) return fail(c, PB_ERR_ARG, "pb_fp64_peak: tflops is NULL");
  int rc = set_device(c);
  if (rc) return rc;
  const int blocks = 4 * c->num_sms, threads = 256, iters = 4096;
  DBuf out;
  PB_CUDA(c, out.ensure((size_t)blocks * threads * sizeof(double)));
  cudaStream_t st = c->stream;
  k_fp64_probe<<<blocks, threads, 0, st>>>(out.as<double>(), 16);
  PB_CUDA(c, cudaEventRecord(c->ev0, st));
  k_fp64_probe<<<blocks, threads, 0, st>>>(out.as<double>(), iters);
  PB_CUDA(c, cudaEventRecord(c->ev1, st));
  PB_CUDA(c, cudaEventSynchronize(c->ev1));
  float t = 0.f;
  PB_CUDA(c, cudaEventElapsedTime(&t, c->ev0, c->ev1));
  out.release();
  const double flop = 2.0 * 256 * 8 * (double)iters * ((double)blocks * threads / 32);
  *tflops = flop / (t * 1e-3) / 1e12;
  return PB_OK;
}

int pb_set_option(pb_context* c, int32_t key, int64_t value) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  switch (key) {
    case PB_OPT_BATCHED_KERNELS:
      if (value != 0 && value != 1) return fail(c, PB_ERR_ARG, "pb_set_option: batched kernels must be 0 or 1");
      c->batched_mode = (int32_t)value;
      return PB_OK;
    case PB_OPT_TMA_STAGING:
      if (value != 0 && value != 1) return fail(c, PB_ERR_ARG, "pb_set_option: TMA staging must be 0 or 1");
      c->tma_mode = (int32_t)value;
      return PB_OK;
    case PB_OPT_BAND_WARPS:
      if (value != 4 && value != 8) return fail(c, PB_ERR_ARG, "pb_set_option: band warps must be 4 or 8");
      c->band_warps = (int32_t)value;
      return PB_OK;
    case PB_OPT_SLAB_PREFETCH:
      if (value < 1 || value > 3) return fail(c, PB_ERR_ARG, "pb_set_option: slab prefetch must be 1, 2 or 3");
      c->slab_pre = (int32_t)value;
      return PB_OK;
    case PB_OPT_STAGING_WAIT_TRIES:
      if (value < 0) c->staging_wait_tries = kWaitTries;
      else if (value > kWaitTries) return fail(c, PB_ERR_ARG, "pb_set_option: staging wait above %lld polls", kWaitTries);
      else c->staging_wait_tries = (long long)value;
      return PB_OK;
  }
  return fail(c, PB_ERR_ARG, "pb_set_option: unknown key %d", key);
}

int pb_get_info(pb_context* c, int32_t key, int64_t* value) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!value) return fail(c, PB_ERR_ARG, "pb_get_info: value is NULL");
  switch (key) {
    case PB_OPT_BATCHED_KERNELS: *value = c->batched_mode; return PB_OK;
    case PB_OPT_TMA_STAGING: *value = c->tma_mode; return PB_OK;
    case PB_OPT_STAGING_WAIT_TRIES: *value = c->staging_wait_tries; return PB_OK;
    case PB_OPT_BAND_WARPS: *value = c->band_warps; return PB_OK;
    case PB_OPT_SLAB_PREFETCH: *value = c->slab_pre; return PB_OK;
    case PB_INFO_LAST_TMA: *value = c->last_tma ? 1 : 0; return PB_OK;
    case PB_INFO_BLOCKED_LAYOUT: *value = (c->blocked_ok && c->fd_tab_ok) ? 1 : 0; return PB_OK;
    case PB_INFO_LAST_BLOCKED: *value = c->last_blocked ? 1 : 0; return PB_OK;
    case PB_INFO_BAND_SPECIES: *value = c->band_nb; return PB_OK;
    case PB_INFO_BAND_ENTRIES: *value = c->band_nnz; return PB_OK;
    case PB_INFO_SLAB_ENTRIES: *value = c->slab_nnz; return PB_OK;
    case PB_INFO_SLAB_ROWS: *value = (int64_t)c->n_slab_spec * c->lay_d; return PB_OK;
    case PB_INFO_FD_DENSE: *value = c->fd_dense_ok ? 1 : 0; return PB_OK;
  }
  return fail(c, PB_ERR_ARG, "pb_get_info: unknown key %d", key);
}

int pb_set_em(pb_context* c, int32_t n_em, int64_t gamma_off, int64_t em_off, int64_t ep_off, int32_t n_cr,
              int32_t n_bh, const int64_t* bh_off, const double* bh_A, const double* inv_E, const double* dE) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_coupling) return fail(c, PB_ERR_STATE, "pb_set_em: set the coupling pattern first");
  if (n_em < 1 || n_em > kMaxEmBins || n_cr < 1 || n_cr > kMaxEmBins || n_bh < 0 || n_bh > kMaxBhSpecies ||
      (n_bh > 0 && (!bh_off || !bh_A)) || !inv_E || !dE)
    return fail(c, PB_ERR_ARG, "pb_set_em: bad arguments (bins must be in [1, %d], at most %d nuclei)", kMaxEmBins,
                kMaxBhSpecies);
  if (gamma_off < 0 || gamma_off + n_em > c->n) return fail(c, PB_ERR_ARG, "pb_set_em: gamma block out of range");
  for (int64_t off : {em_off, ep_off})
    if (off >= 0 && off + n_em > c->n) return fail(c, PB_ERR_ARG, "pb_set_em: lepton block out of range");
  for (int s = 0; s < n_bh; ++s)
    if (bh_off[s] < 0 || bh_off[s] + n_cr > c->n) return fail(c, PB_ERR_ARG, "pb_set_em: nucleus block out of range");
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = upload(c, c->em_bh_off, bh_off, (size_t)n_bh))) return rc;
  if ((rc = upload(c, c->em_bh_A, bh_A, (size_t)n_bh))) return rc;
  if ((rc = upload(c, c->em_invE, inv_E, (size_t)n_cr))) return rc;
  if ((rc = upload(c, c->em_dE, dE, (size_t)n_cr))) return rc;
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->em_n = n_em;
  c->em_ncr = n_cr;
  c->em_nbh = n_bh;
  c->em_g = gamma_off;
  c->em_m = em_off;
  c->em_p = ep_off;
  c->have_em = true;
  c->em_W = 0;
  return PB_OK;
}

int pb_set_em_windows(pb_context* c, int32_t n_windows, const double* Tg, const double* Te, const double* R,
                      const double* dl_step) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_em) return fail(c, PB_ERR_STATE, "pb_set_em_windows: call pb_set_em first");
  if (n_windows < 1 || !Tg || !Te || !R || !dl_step) return fail(c, PB_ERR_ARG, "pb_set_em_windows: bad arguments");
  int rc = set_device(c);
  if (rc) return rc;
  const size_t nn = (size_t)c->em_n * c->em_n, nr = (size_t)c->em_n * c->em_ncr;
  if ((rc = upload(c, c->em_Tg, Tg, nn * n_windows))) return rc;
  if ((rc = upload(c, c->em_Te, Te, nn * n_windows))) return rc;
  if ((rc = upload(c, c->em_R, R, nr * n_windows))) return rc;
  {  // transposes for the adjoint's GEMMs
    std::vector<double> tg(nn * n_windows), te(nn * n_windows), rt(nr * n_windows);
    const int m = c->em_n, q = c->em_ncr;
    for (int32_t w = 0; w < n_windows; ++w)
      for (int i = 0; i < m; ++i) {
        for (int j = 0; j < m; ++j) {
          tg[w * nn + (size_t)j * m + i] = Tg[w * nn + (size_t)i * m + j];
          te[w * nn + (size_t)j * m + i] = Te[w * nn + (size_t)i * m + j];
        }
        for (int j = 0; j < q; ++j) rt[w * nr + (size_t)j * m + i] = R[w * nr + (size_t)i * q + j];
      }
    if ((rc = upload(c, c->em_TgT, tg.data(), tg.size()))) return rc;
    if ((rc = upload(c, c->em_TeT, te.data(), te.size()))) return rc;
    if ((rc = upload(c, c->em_RT, rt.data(), rt.size()))) return rc;
  }
  PB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->em_dl.assign(dl_step, dl_step + n_windows);
  c->em_W = n_windows;
  return PB_OK;
}


// Kinetic EM-cascade transfer (em_transfer.cuh): field-free kernels, the
// contractions with the photon stacks, the per-redshift matrices and the
// scattering iteration on the device; (T_gamma, T_electron) per redshift back
// to the host.  The small per-electron loss grid, the trapezoid weights and
// the loss-shift indices are set up here, as the reference computes them.
int pb_em_transfer(pb_context* c, const pb_em_transfer_args* a) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!a) return fail(c, PB_ERR_ARG, "pb_em_transfer: args is NULL");
  if (!c->have_field) return fail(c, PB_ERR_STATE, "pb_em_transfer: set the photon field first");
  const int n = a->n, nz = a->n_z, ne = a->n_eps, no = a->n_eps_o, nmu = a->n_mu, nE1 = a->n_E1;
  if (n < 2 || n > 1024 || nz < 1 || ne < 2 || no < 2 || nmu < 2 || nE1 < 2 || !a->E || !a->z || !a->dl_step ||
      !a->eps || !a->eps_o || !a->mu || !a->T_gamma || !a->T_electron || a->max_scatter < 1 || !(a->tol > 0))
    return fail(c, PB_ERR_ARG, "pb_em_transfer: bad arguments");
  // grid sizes within the launch limits of the kernels below (GEMM rows / 64 and
  // the batch of redshifts are grid dimensions)
  if ((int64_t)n * nE1 > 4000000 || ne > 100000 || no > 100000 || nmu > 100000 || nz > 65535)
    return fail(c, PB_ERR_ARG, "pb_em_transfer: grid sizes beyond the supported limits");
  for (int i = 1; i < n; ++i)
    if (!(a->E[i] > a->E[i - 1])) return fail(c, PB_ERR_ARG, "pb_em_transfer: E must increase");
  int rc = set_device(c);
  if (rc) return rc;
  cudaStream_t st = c->stream;
  if (!(a->m_electron > 0) || !(a->r_electron > 0) || !(a->c_cm > 0))
    return fail(c, PB_ERR_ARG, "pb_em_transfer: unit constants must be positive");
  const double me = a->m_electron;
  const double sigma_t = 8.0 / 3.0 * M_PI * (a->r_electron * a->r_electron);
  const EmConst K{me, 0.75 * sigma_t * a->c_cm, sigma_t};
  // host set-up (small): trapezoid weights, per-electron loss grid, dE, loss shift
  auto tw = [](const double* x, int m, std::vector<double>& w) {
    w.assign((size_t)m, 0.0);
    for (int i = 1; i + 1 < m; ++i) w[i] = (x[i + 1] - x[i - 1]) / 2.0;
    w[0] = (x[1] - x[0]) / 2.0;
    w[m - 1] = (x[m - 1] - x[m - 2]) / 2.0;
  };
  std::vector<double> w_eps, w_o, dE((size_t)n), E1((size_t)n * nE1), w1((size_t)n * nE1), epsw_eps((size_t)ne);
  tw(a->eps, ne, w_eps);
  tw(a->eps_o, no, w_o);
  for (int k = 0; k < ne; ++k) epsw_eps[k] = w_eps[k] * a->eps[k];
  for (int i = 0; i < n; ++i)  // numpy.gradient: central inside, one-sided at the ends
    dE[i] = i == 0 ? a->E[1] - a->E[0] : i == n - 1 ? a->E[n - 1] - a->E[n - 2] : (a->E[i + 1] - a->E[i - 1]) / 2.0;
  double emin = a->eps[0];
  for (int k = 1; k < ne; ++k) emin = std::min(emin, a->eps[k]);
  const double lo = log10(emin);
  for (int j = 0; j < n; ++j) {  // numpy.logspace(lo, log10(0.9999 E_j), nE1)
    const double hi = log10(0.9999 * a->E[j]);
    const double step = (hi - lo) / (nE1 - 1);
    for (int m = 0; m < nE1; ++m) E1[(size_t)j * nE1 + m] = pow(10.0, m == nE1 - 1 ? hi : m * step + lo);
    std::vector<double> w;
    tw(&E1[(size_t)j * nE1], nE1, w);
    std::copy(w.begin(), w.end(), w1.begin() + (size_t)j * nE1);
  }
  std::vector<int> bidx((size_t)n * n, -1);
  std::vector<double> frac((size_t)n * n, 0.0);
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j) {
      const double Eep = a->E[j] - a->E[k];
      if (!(Eep > a->E[0])) continue;
      int b = (int)(std::lower_bound(a->E, a->E + n, Eep) - a->E) - 1;
      b = std::min(std::max(b, 0), n - 2);
      const double f = (a->E[b + 1] - Eep) / (a->E[b + 1] - a->E[b]);
      bidx[(size_t)k * n + j] = b;
      frac[(size_t)k * n + j] = std::min(std::max(f, 0.0), 1.0);
    }
  const size_t nn = (size_t)n * n, zn = (size_t)nz * n, znn = (size_t)nz * nn;
  DBuf dE_d, E_d, z_d, dl_d, eps_d, weps_d, epso_d, wo_d, mu_d, E1_d, w1_d, b_d, f_d, N, No, Ae, Ap, Bl, Kt, raw,
      rawdN, rawt, emis, pair, P, Sg, cold, De, Mic, loss, Pe, epsm, G, e, esc, fin, T1, ec, eh, Gh, Gc, done, Te;
  std::vector<DBuf*> all{&dE_d, &E_d, &z_d, &dl_d, &eps_d, &weps_d, &epso_d, &wo_d, &mu_d, &E1_d, &w1_d, &b_d, &f_d,
                         &N, &No, &Ae, &Ap, &Bl, &Kt, &raw, &rawdN, &rawt, &emis, &pair, &P, &Sg, &cold, &De,
                         &Mic, &loss, &Pe, &epsm, &G, &e, &esc, &fin, &T1, &ec, &eh, &Gh, &Gc, &done, &Te};
  auto cleanup = [&]() { for (DBuf* b : all) b->release(); };
  auto fail_cuda = [&](cudaError_t err, const char* what) {
    cleanup();
    return fail(c, PB_ERR_CUDA, "pb_em_transfer: %s: %s", what, cudaGetErrorString(err));
  };
  if ((rc = upload(c, dE_d, dE.data(), dE.size())) || (rc = upload(c, E_d, a->E, (size_t)n)) ||
      (rc = upload(c, z_d, a->z, (size_t)nz)) || (rc = upload(c, dl_d, a->dl_step, (size_t)nz)) ||
      (rc = upload(c, eps_d, a->eps, (size_t)ne)) || (rc = upload(c, weps_d, w_eps.data(), w_eps.size())) ||
      (rc = upload(c, epso_d, a->eps_o, (size_t)no)) || (rc = upload(c, wo_d, w_o.data(), w_o.size())) ||
      (rc = upload(c, mu_d, a->mu, (size_t)nmu)) || (rc = upload(c, E1_d, E1.data(), E1.size())) ||
      (rc = upload(c, w1_d, w1.data(), w1.size())) || (rc = upload(c, b_d, bidx.data(), bidx.size())) ||
      (rc = upload(c, f_d, frac.data(), frac.size()))) {
    cleanup();
    return rc;
  }
  struct Want { DBuf* b; size_t bytes; };
  for (const Want& w : {Want{&N, (size_t)ne * nz * 8}, Want{&No, (size_t)no * nz * 8}, Want{&Ae, nn * ne * 8},
                        Want{&Ap, nn * ne * 8}, Want{&Bl, (size_t)n * nE1 * ne * 8}, Want{&Kt, (size_t)n * no * 8},
                        Want{&raw, nn * nz * 8}, Want{&rawdN, (size_t)n * nE1 * nz * 8}, Want{&rawt, zn * 8},
                        Want{&emis, znn * 8}, Want{&pair, znn * 8}, Want{&P, znn * 8}, Want{&Sg, znn * 8},
                        Want{&cold, zn}, Want{&De, znn * 8}, Want{&Mic, znn * 8}, Want{&loss, zn * 8},
                        Want{&Pe, zn * 8}, Want{&epsm, (size_t)nz * 8}, Want{&G, znn * 8}, Want{&e, znn * 8},
                        Want{&esc, znn * 8}, Want{&fin, znn * 8}, Want{&T1, znn * 8}, Want{&ec, znn * 8},
                        Want{&eh, znn * 8}, Want{&Gh, znn * 8}, Want{&Gc, znn * 8}, Want{&done, (size_t)nz * 4},
                        Want{&Te, znn * 8}}) {
    const cudaError_t err = w.b->ensure(w.bytes);
    if (err != cudaSuccess) return fail_cuda(err, "allocation");
  }
  const FieldDesc f = field_desc(c, a->photon_scale);
  const int T = 256;
  auto nb = [&](int64_t work) { return (unsigned)blocks_for(work, T); };
  // 1. photon stacks; 2. field-free kernels
  k_em_stack<<<nb((int64_t)ne * nz), T, 0, st>>>(f, eps_d.as<double>(), ne, z_d.as<double>(), nz, N.as<double>());
  k_em_stack<<<nb((int64_t)no * nz), T, 0, st>>>(f, epso_d.as<double>(), no, z_d.as<double>(), nz, No.as<double>());
  k_em_ic<<<nb((int64_t)nn * ne), T, 0, st>>>(K, E_d.as<double>(), n, eps_d.as<double>(), weps_d.as<double>(), ne,
                                               Ae.as<double>());
  k_em_pair<<<nb((int64_t)nn * ne), T, 0, st>>>(K, E_d.as<double>(), n, eps_d.as<double>(), weps_d.as<double>(), ne,
                                                 Ap.as<double>());
  k_em_icloss<<<nb((int64_t)n * nE1 * ne), T, 0, st>>>(K, E_d.as<double>(), E1_d.as<double>(), n, nE1,
                                                       eps_d.as<double>(), weps_d.as<double>(), ne, Bl.as<double>());
  k_em_tau<<<nb((int64_t)n * no), T, 0, st>>>(K, E_d.as<double>(), n, epso_d.as<double>(), wo_d.as<double>(), no,
                                              mu_d.as<double>(), nmu, Kt.as<double>());
  // 3. contractions (FP64 tensor-core GEMMs) and the per-column prefactors
  std::vector<double> pe((size_t)n), pp((size_t)n);
  for (int j = 0; j < n; ++j) {
    const double g = a->E[j] / me;
    pe[j] = g > 1.0 ? K.pref_ic / (g * g) : 0.0;
    pp[j] = K.pref_ic / (g * g * g);
  }
  DBuf pe_d, pp_d;
  all.push_back(&pe_d);
  all.push_back(&pp_d);
  if ((rc = upload(c, pe_d, pe.data(), pe.size())) || (rc = upload(c, pp_d, pp.data(), pp.size()))) {
    cleanup();
    return rc;
  }
  const unsigned gz = nb((int64_t)znn);
  bgemm(st, Ae.as<double>(), N.as<double>(), raw.as<double>(), (int)nn, nz, ne, ne, nz, nz, 0, 0, 0, 1, false);
  k_em_scatter_contraction<<<gz, T, 0, st>>>(raw.as<double>(), n, nz, pe_d.as<double>(), emis.as<double>());
  bgemm(st, Ap.as<double>(), N.as<double>(), raw.as<double>(), (int)nn, nz, ne, ne, nz, nz, 0, 0, 0, 1, false);
  k_em_scatter_contraction<<<gz, T, 0, st>>>(raw.as<double>(), n, nz, pp_d.as<double>(), pair.as<double>());
  bgemm(st, Bl.as<double>(), N.as<double>(), rawdN.as<double>(), n * nE1, nz, ne, ne, nz, nz, 0, 0, 0, 1, false);
  bgemm(st, Kt.as<double>(), No.as<double>(), rawt.as<double>(), n, nz, no, no, nz, nz, 0, 0, 0, 1, false);
  // eps_mean[z] = (w eps) N / (w N), on the host from the stack (nz x ne values)
  std::vector<double> Nh((size_t)ne * nz), em((size_t)nz);
  cudaError_t err = cudaMemcpyAsync(Nh.data(), N.p, Nh.size() * 8, cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err != cudaSuccess) return fail_cuda(err, "photon stack");
  for (int z = 0; z < nz; ++z) {
    double a1 = 0.0, b1 = 0.0;
    for (int k = 0; k < ne; ++k) {
      a1 += epsw_eps[k] * Nh[(size_t)k * nz + z];
      b1 += w_eps[k] * Nh[(size_t)k * nz + z];
    }
    em[z] = a1 / b1;
  }
  if ((rc = upload(c, epsm, em.data(), em.size()))) {
    cleanup();
    return rc;
  }
  // 4. per-redshift matrices
  std::vector<double> pl = pe;
  DBuf pl_d;
  all.push_back(&pl_d);
  if ((rc = upload(c, pl_d, pl.data(), pl.size()))) {
    cleanup();
    return rc;
  }
  k_em_loss<<<nb((int64_t)zn), T, 0, st>>>(rawdN.as<double>(), n, nE1, nz, pl_d.as<double>(), E1_d.as<double>(),
                                           w1_d.as<double>(), epsm.as<double>(), loss.as<double>());
  k_em_columns<<<nb((int64_t)zn), T, 0, st>>>(pair.as<double>(), emis.as<double>(), E_d.as<double>(),
                                              dE_d.as<double>(), n, nz, a->cool_floor_frac, P.as<double>(),
                                              Sg.as<double>(), cold.as<unsigned char>());
  k_em_shift<<<gz, T, 0, st>>>(Sg.as<double>(), E_d.as<double>(), dE_d.as<double>(), b_d.as<int>(), f_d.as<double>(),
                               n, nz, De.as<double>());
  k_em_cooled<<<nb((int64_t)zn), T, 0, st>>>(emis.as<double>(), loss.as<double>(), E_d.as<double>(), n, nz,
                                             Mic.as<double>());
  k_em_normalise<<<nb((int64_t)zn), T, 0, st>>>(Mic.as<double>(), E_d.as<double>(), n, nz);
  k_em_escape<<<nb((int64_t)zn), T, 0, st>>>(rawt.as<double>(), dl_d.as<double>(), n, nz, Pe.as<double>());
  // 5. the scattering iteration, checked on the host every 8 passes (a
  // redshift that has converged keeps its frozen result)
  std::vector<double> Ein((size_t)n);
  for (int i = 0; i < n; ++i) Ein[i] = a->E[i] * dE[i];
  DBuf Ein_d;
  all.push_back(&Ein_d);
  if ((rc = upload(c, Ein_d, Ein.data(), Ein.size()))) {
    cleanup();
    return rc;
  }
  k_em_iter_init<<<gz, T, 0, st>>>(n, nz, G.as<double>(), e.as<double>(), esc.as<double>(), fin.as<double>());
  err = cudaMemsetAsync(done.p, 0, (size_t)nz * 4, st);
  if (err != cudaSuccess) return fail_cuda(err, "init");
  const long long snn = (long long)nn;
  int passes = 0;
  std::vector<int> hd((size_t)nz);
  while (passes < a->max_scatter) {
    const int batch = std::min(8, a->max_scatter - passes);
    for (int q = 0; q < batch; ++q) {
      k_em_iter_a<<<gz, T, 0, st>>>(Pe.as<double>(), dE_d.as<double>(), n, nz, G.as<double>(), esc.as<double>(),
                                    T1.as<double>());
      bgemm(st, P.as<double>(), T1.as<double>(), e.as<double>(), n, n, n, n, n, n, snn, snn, snn, nz, true);
      k_em_iter_b<<<gz, T, 0, st>>>(e.as<double>(), cold.as<unsigned char>(), dE_d.as<double>(), n, nz,
                                    ec.as<double>(), eh.as<double>());
      bgemm(st, Mic.as<double>(), ec.as<double>(), Gc.as<double>(), n, n, n, n, n, n, snn, snn, snn, nz, false);
      bgemm(st, Sg.as<double>(), eh.as<double>(), Gh.as<double>(), n, n, n, n, n, n, snn, snn, snn, nz, false);
      bgemm(st, De.as<double>(), eh.as<double>(), e.as<double>(), n, n, n, n, n, n, snn, snn, snn, nz, false);
      k_em_iter_c<<<gz, T, 0, st>>>(Pe.as<double>(), n, nz, Gh.as<double>(), Gc.as<double>(), G.as<double>(),
                                    esc.as<double>());
      k_em_iter_conv<<<nz, 256, 0, st>>>(Ein_d.as<double>(), Pe.as<double>(), n, a->tol, G.as<double>(),
                                         e.as<double>(), esc.as<double>(), fin.as<double>(), done.as<int>());
    }
    passes += batch;
    err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaMemcpyAsync(hd.data(), done.p, (size_t)nz * 4, cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err != cudaSuccess) return fail_cuda(err, "iteration");
    if (std::all_of(hd.begin(), hd.end(), [](int v) { return v != 0; })) break;
  }
  k_em_finish<<<gz, T, 0, st>>>(done.as<int>(), esc.as<double>(), Mic.as<double>(), dE_d.as<double>(), n, nz,
                                fin.as<double>(), T1.as<double>());
  bgemm(st, fin.as<double>(), T1.as<double>(), Te.as<double>(), n, n, n, n, n, n, snn, snn, snn, nz, false);
  err = cudaGetLastError();
  if (err == cudaSuccess) err = cudaMemcpyAsync(a->T_gamma, fin.p, znn * 8, cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaMemcpyAsync(a->T_electron, Te.p, znn * 8, cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err != cudaSuccess) return fail_cuda(err, "results");
  if (a->iterations) *a->iterations = passes;
  cleanup();
  return PB_OK;
}


// Bethe-Heitler e+- pair shape per redshift on the device (em_transfer.cuh).
int pb_bh_shape(pb_context* c, const pb_bh_shape_args* a) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!a) return fail(c, PB_ERR_ARG, "pb_bh_shape: args is NULL");
  if (!c->have_field) return fail(c, PB_ERR_STATE, "pb_bh_shape: set the photon field first");
  const int ne = a->n_e, np = a->n_p, nk = a->n_eps, nz = a->n_z;
  if (ne < 2 || np < 1 || nk < 2 || nz < 1 || ne > 4096 || np > 4096 || nk > 4096 || nz > 65535 || !a->E_e ||
      !a->E_p || !a->eps || !a->z || !a->R || !(a->m_electron > 0) || !(a->m_proton > 0))
    return fail(c, PB_ERR_ARG, "pb_bh_shape: bad arguments");
  int rc = set_device(c);
  if (rc) return rc;
  cudaStream_t st = c->stream;
  DBuf Ee, Ep, eps, zs, K, neps, col, R;
  auto cleanup = [&]() { for (DBuf* b : {&Ee, &Ep, &eps, &zs, &K, &neps, &col, &R}) b->release(); };
  if ((rc = upload(c, Ee, a->E_e, (size_t)ne)) || (rc = upload(c, Ep, a->E_p, (size_t)np)) ||
      (rc = upload(c, eps, a->eps, (size_t)nk)) || (rc = upload(c, zs, a->z, (size_t)nz))) {
    cleanup();
    return rc;
  }
  const size_t zne = (size_t)nz * ne * np;
  for (auto w : {std::make_pair(&K, (size_t)ne * np * nk * 8), std::make_pair(&neps, (size_t)nk * nz * 8),
                 std::make_pair(&col, zne * 8), std::make_pair(&R, zne * 8)}) {
    const cudaError_t e = w.first->ensure(w.second);
    if (e != cudaSuccess) {
      cleanup();
      return fail(c, PB_ERR_CUDA, "pb_bh_shape: allocation: %s", cudaGetErrorString(e));
    }
  }
  const FieldDesc f = field_desc(c, a->photon_scale);
  k_em_stack<<<blocks_for((int64_t)nk * nz, 256), 256, 0, st>>>(f, eps.as<double>(), nk, zs.as<double>(), nz,
                                                                neps.as<double>());
  k_bh_kernel<<<blocks_for((int64_t)ne * np * nk, 128), 128, 0, st>>>(a->m_electron, a->m_proton, Ee.as<double>(), ne,
                                                                      Ep.as<double>(), np, eps.as<double>(), nk,
                                                                      K.as<double>());
  k_bh_col<<<blocks_for((int64_t)zne, 256), 256, 0, st>>>(K.as<double>(), Ee.as<double>(), ne, Ep.as<double>(), np,
                                                          eps.as<double>(), neps.as<double>(), nk, nz, a->e_p_min,
                                                          col.as<double>());
  k_bh_norm<<<blocks_for((int64_t)nz * np, 256), 256, 0, st>>>(col.as<double>(), Ee.as<double>(), ne,
                                                               Ep.as<double>(), np, nz, R.as<double>());
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(a->R, R.p, zne * 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cleanup();
  if (e != cudaSuccess) return fail(c, PB_ERR_CUDA, "pb_bh_shape: %s", cudaGetErrorString(e));
  return PB_OK;
}

int pb_solve(pb_context* c, const pb_solve_args* a) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!a) return fail(c, PB_ERR_ARG, "pb_solve: args is NULL");
  if (!c->have_coupling || !c->have_photon_grid || !c->have_field || !c->have_fd || !c->have_losses)
    return fail(c, PB_ERR_STATE, "pb_solve: coupling, photon grid, photon field, FD operator and losses must be set");
  const uint32_t flags = a->flags;
  if ((flags & PB_PHOTOHAD) && !c->have_kernel) return fail(c, PB_ERR_STATE, "pb_solve: fold kernel not set");
  if ((flags & PB_DECAY) && !c->have_decay) return fail(c, PB_ERR_STATE, "pb_solve: decay operator not set");
  const int64_t S = a->n_steps;
  const int W = a->n_windows;
  const int K = a->n_cols;
  if (S < 0 || W < 1 || K < 1 || !a->state) return fail(c, PB_ERR_ARG, "pb_solve: bad sizes");
  if (S > 0 && (!a->z_window || !a->window || !a->h || !a->dldz || !a->hc || !a->finj || !a->n_active))
    return fail(c, PB_ERR_ARG, "pb_solve: schedule arrays missing");
  const bool inj = (flags & PB_INJECTION) && c->n_src > 0;
  if ((flags & PB_EM_CASCADE) && (!c->have_em || c->em_W != W))
    return fail(c, PB_ERR_STATE, "pb_solve: EM cascade requested but pb_set_em / pb_set_em_windows (%d windows) missing", W);
  if (inj && c->n_src_cols != K) return fail(c, PB_ERR_ARG, "pb_solve: injection was set for %d columns, solve has %d", c->n_src_cols, K);
  if (inj && S > 0 && !a->coeff) return fail(c, PB_ERR_ARG, "pb_solve: coeff missing");
  for (int64_t k = 0; k < S; ++k) {
    if (a->window[k] < 0 || a->window[k] >= W) return fail(c, PB_ERR_ARG, "pb_solve: window index out of range at step %lld", (long long)k);
    if (a->n_active[k] < 0 || a->n_active[k] > K) return fail(c, PB_ERR_ARG, "pb_solve: n_active out of range");
  }
  if ((int64_t)W * c->n >= ((int64_t)1 << 40)) return fail(c, PB_ERR_ARG, "pb_solve: too many windows");
  c->h_win.assign(a->window, a->window + S);
  c->h_nact.assign(a->n_active, a->n_active + S);
  int rc = set_device(c);
  if (rc) return rc;
  const int64_t n = c->n;
  const int ld = K == 1 ? 1 : ((K + kColTile - 1) / kColTile) * kColTile;
  cudaStream_t st = c->stream;

  // ---- per-solve uploads -------------------------------------------------
  if ((rc = upload(c, c->zwin, a->z_window, (size_t)W))) return rc;
  if (S > 0) {
    if ((rc = upload(c, c->s_h, a->h, (size_t)S))) return rc;
    if ((rc = upload(c, c->s_dldz, a->dldz, (size_t)S))) return rc;
    if ((rc = upload(c, c->s_hc, a->hc, (size_t)S))) return rc;
    if ((rc = upload(c, c->s_finj, a->finj, (size_t)S))) return rc;
    if ((rc = upload(c, c->s_win, a->window, (size_t)S))) return rc;
    if (inj && (rc = upload(c, c->s_coeff, a->coeff, (size_t)S * c->n_src))) return rc;
  }
  PB_CUDA(c, c->PT.ensure((size_t)W * c->dph * sizeof(double)));
  PB_CUDA(c, c->rs.ensure((size_t)W * c->n_cr_bins * sizeof(double)));
  PB_CUDA(c, c->kp.ensure((size_t)W * n * sizeof(double)));
  PB_CUDA(c, c->m_indptr.ensure(((size_t)n + 1) * sizeof(int64_t)));
  PB_CUDA(c, c->m_diag.ensure((size_t)W * n * sizeof(double)));
  const int64_t R = c->R;
  const int64_t mstride = std::max<int64_t>(R, 1);
  PB_CUDA(c, c->m_vals.ensure((size_t)W * mstride * sizeof(double)));
  PB_CUDA(c, c->m_indices.ensure((size_t)mstride * sizeof(int)));
  PB_CUDA(c, c->keep.ensure(((size_t)R + 1) * sizeof(int)));
  PB_CUDA(c, c->pos.ensure(((size_t)R + 1) * sizeof(int)));
  PB_CUDA(c, c->dest.ensure((size_t)mstride * 2 * sizeof(int)));
  const size_t sbytes = (size_t)n * ld * sizeof(double);
  PB_CUDA(c, c->X.ensure(sbytes));
  PB_CUDA(c, c->A.ensure(sbytes));
  PB_CUDA(c, c->F.ensure(sbytes));
  if ((flags & PB_EM_CASCADE) && c->have_em) {
    PB_CUDA(c, c->em_wbuf.ensure((size_t)c->em_ncr * ld * sizeof(double)));
    for (DBuf* b : {&c->em_es, &c->em_lep, &c->em_y}) PB_CUDA(c, b->ensure((size_t)c->em_n * ld * sizeof(double)));
  }
  PB_CUDA(c, c->rowf.ensure((size_t)8 * n * sizeof(double)));
  const int ctiles = ld / (K == 1 ? 1 : kColTile);
  const int nlong_rows = (int)c->h_long_rows.size();
  PB_CUDA(c, c->seg_mb.ensure((size_t)std::max(c->n_seg, 1) * sizeof(int64_t)));
  PB_CUDA(c, c->seg_me.ensure((size_t)std::max(c->n_seg, 1) * sizeof(int64_t)));
  PB_CUDA(c, c->partial.ensure((size_t)std::max(c->n_seg, 1) * ld * sizeof(double)));
  PB_CUDA(c, c->counter.ensure((size_t)std::max(nlong_rows, 1) * ctiles * sizeof(int)));
  if (a->ckpt_every < 0) return fail(c, PB_ERR_ARG, "pb_solve: ckpt_every must be >= 0");
  if (a->out_cols)
    for (int j = 0; j < K; ++j)
      if (a->out_cols[j] < 0 || a->out_cols[j] >= K) return fail(c, PB_ERR_ARG, "pb_solve: out_cols[%d] out of range", j);
  if (a->ckpt_every > 0)
    PB_CUDA(c, c->ckpt.ensure((size_t)((S + a->ckpt_every - 1) / a->ckpt_every + 1) * n * ld * sizeof(double)));
  const bool blocked = use_blocked(c, K);
  if (blocked) {
    PB_CUDA(c, c->slab_vals.ensure((size_t)W * std::max<int64_t>(c->slab_nent, 1) * sizeof(double)));
    PB_CUDA(c, c->fdbuf.ensure(sbytes));
    PB_CUDA(c, c->band_vals.ensure((size_t)W * std::max<int64_t>(c->band_stride, 1) * sizeof(double)));
    PB_CUDA(c, c->band_part.ensure((size_t)kMaxBandGroups * std::max(c->band_nb, 1) * c->lay_d * ld * sizeof(double)));
  }
  c->last_blocked = blocked;
  PB_CUDA(c, c->d_err.ensure(sizeof(int)));
  if ((rc = ensure_tmaps(c, blocked, ld))) return rc;
  c->last_tma = blocked && c->tma_ok;
  PB_CUDA(c, cudaMemsetAsync(c->d_err.p, 0, sizeof(int), st));
  size_t scan_need = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_need, (int*)nullptr, (int*)nullptr, (int)(R + 1));
  PB_CUDA(c, c->scan_tmp.ensure(scan_need));

  double* X = c->X.as<double>();
  const int* rmap = c->have_row_map ? c->row_map.as<int>() : nullptr;
  if (a->init_state && rmap) {  // the caller's rows: one copy to scratch, then a gather into solve order
    PB_CUDA(c, cudaMemcpyAsync(c->F.p, a->state, (size_t)n * K * sizeof(double),
                               a->state_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    if (K > 1 && ld > K) PB_CUDA(c, cudaMemsetAsync(X, 0, sbytes, st));
    k_pick_cols<<<dim3(blocks_for(n, 8), blocks_for(K, kColTile)), 256, 0, st>>>(c->F.as<double>(), n, K, nullptr,
                                                                               rmap, X, ld);
    PB_CUDA(c, cudaGetLastError());
  } else if (a->init_state) {
    if (a->state_on_device) {
      PB_CUDA(c, cudaMemcpy2DAsync(X, ld * sizeof(double), a->state, K * sizeof(double), K * sizeof(double), n,
                                   cudaMemcpyDeviceToDevice, st));
    } else {
      PB_CUDA(c, cudaMemcpy2DAsync(X, ld * sizeof(double), a->state, K * sizeof(double), K * sizeof(double), n,
                                   cudaMemcpyHostToDevice, st));
    }
  } else {
    PB_CUDA(c, cudaMemsetAsync(X, 0, sbytes, st));
  }
  const FieldDesc fd = field_desc(c, a->photon_scale);
  int64_t launches = 0;
  // Everything from here to the end of the last step is enqueued by `enqueue`:
  // directly, or under stream capture into a CUDA graph that is replayed while
  // the solve's shape and buffers stay the same.
  StepParams p;
  memset(&p, 0, sizeof(p));
  auto enqueue = [&](int64_t& launches) -> int {

  // ---- photon matrix and pair-loss vectors for every window ---------------
  k_photon_matrix<<<blocks_for((int64_t)W * c->dph, 256), 256, 0, st>>>(fd, c->eph.as<double>(), c->dph,
                                                                          c->zwin.as<double>(), W, c->PT.as<double>());
  ++launches;
  const bool pair = (flags & PB_PAIRPROD) && (flags & PB_PARTIAL_DIFF);
  if (pair || (flags & PB_EM_CASCADE)) {  // the EM hook reads kappa_pair whatever the loss flags
    k_pair_rate<<<dim3(c->n_cr_bins, W), 128, 0, st>>>(fd, c->pair_pg.as<double>(), c->xi.as<double>(),
                                                       c->phi_xi2.as<double>(), c->n_xi, c->n_cr_bins,
                                                       c->zwin.as<double>(), c->rs.as<double>());
    k_pair_expand<<<blocks_for((int64_t)W * n, 256), 256, 0, st>>>(c->rs.as<double>(), c->pair_scale.as<double>(),
                                                                   c->pair_bin.as<int>(), c->n_cr_bins, n, W,
                                                                   c->kp.as<double>());
    launches += 2;
  }
  // ---- operator pattern and fold -----------------------------------------
  int* dest = c->dest.as<int>();
  int* diag_row = dest + mstride;
  PB_CUDA(c, cudaMemsetAsync(c->m_diag.p, 0, (size_t)W * n * sizeof(double), st));
  if (blocked && c->band_stride > 0)
    PB_CUDA(c, cudaMemsetAsync(c->band_vals.p, 0, (size_t)W * c->band_stride * sizeof(double), st));
  if (blocked && c->slab_nent > 0)
    PB_CUDA(c, cudaMemsetAsync(c->slab_vals.p, 0, (size_t)W * c->slab_nent * sizeof(double), st));
  if ((flags & PB_PHOTOHAD) && R > 0) {
    k_fold_first<<<blocks_for(R + 1, 8), 256, 0, st>>>(c->kernel.as<double>(), R, c->dph, c->PT.as<double>(),
                                                       c->cpl_is_diag.as<int>(), c->keep.as<int>());
    size_t tb = c->scan_tmp.bytes;
    PB_CUDA(c, cub::DeviceScan::ExclusiveSum(c->scan_tmp.p, tb, c->keep.as<int>(), c->pos.as<int>(), (int)(R + 1), st));
    k_compact<<<blocks_for(R, 256), 256, 0, st>>>(c->keep.as<int>(), c->pos.as<int>(), c->cpl_indices.as<int>(),
                                                  c->cpl_is_diag.as<int>(), c->cpl_row.as<int>(), R, dest, diag_row,
                                                  c->m_indices.as<int>());
    k_m_indptr<<<blocks_for(n + 1, 256), 256, 0, st>>>(c->cpl_indptr.as<int64_t>(), c->pos.as<int>(), n,
                                                       c->m_indptr.as<int64_t>());
    if (c->n_seg > 0) {
      k_seg_map<<<blocks_for(c->n_seg, 256), 256, 0, st>>>(c->seg_cb.as<int64_t>(), c->seg_ce.as<int64_t>(),
                                                           c->pos.as<int>(), c->n_seg, c->seg_mb.as<int64_t>(),
                                                           c->seg_me.as<int64_t>());
      ++launches;
    }
    const int kpad = (c->dph + 3) / 4 * 4;
    const size_t smem = (size_t)(kFoldBM + kFoldBN) * (kpad + 4) * sizeof(double);
    k_fold_gemm<<<dim3(blocks_for(R, kFoldBM), blocks_for(W, kFoldBN)), 256, smem, st>>>(
        c->kernel.as<double>(), R, c->dph, kpad, c->PT.as<double>(), W, dest, diag_row, c->m_vals.as<double>(),
        mstride, c->m_diag.as<double>(), n, blocked ? c->band_slot.as<int>() : nullptr,
        blocked ? c->band_vals.as<double>() : nullptr, c->band_stride, blocked ? c->slab_slot.as<int>() : nullptr,
        blocked ? c->slab_vals.as<double>() : nullptr, c->slab_nent);
    launches += 5;
  } else {
    PB_CUDA(c, cudaMemsetAsync(c->m_indptr.p, 0, ((size_t)n + 1) * sizeof(int64_t), st));
    if (c->n_seg > 0) {
      PB_CUDA(c, cudaMemsetAsync(c->seg_mb.p, 0, (size_t)c->n_seg * sizeof(int64_t), st));
      PB_CUDA(c, cudaMemsetAsync(c->seg_me.p, 0, (size_t)c->n_seg * sizeof(int64_t), st));
    }
  }
  PB_CUDA(c, cudaMemsetAsync(c->counter.p, 0, (size_t)std::max(nlong_rows, 1) * ctiles * sizeof(int), st));
  PB_CUDA(c, cudaGetLastError());

  // ---- ETD2 step parameters -----------------------------------------------
  fill_step_params(c, p, K, ld, flags, pair, inj, S, ctiles);
    return PB_OK;
  };
  auto enqueue_steps = [&](int64_t& launches) -> int {
  const int CK = a->ckpt_every;
  launches += launch_steps(c, p, K, a->n_active, 0, S, st, CK > 0 ? c->ckpt.as<double>() : nullptr, CK);
  PB_CUDA(c, cudaGetLastError());
    return PB_OK;
  };

  std::vector<uint64_t> key;
  {
    auto put = [&](uint64_t v) { key.push_back(v); };
    put((uint64_t)S); put((uint64_t)W); put((uint64_t)K); put((uint64_t)ld); put(flags); put(inj); put(R);
    put((uint64_t)c->n_seg); put((uint64_t)c->h_short_rows.size()); put((uint64_t)c->n_cr_bins);
    put((uint64_t)a->ckpt_every);
    put((uint64_t)blocked);
    put((uint64_t)(blocked && c->tma_ok));
    put((uint64_t)c->staging_wait_tries);
    put((uint64_t)c->band_warps);
    put((uint64_t)c->slab_pre);
    put((uint64_t)c->band_RT); put((uint64_t)c->band_J); put((uint64_t)c->band_nb); put((uint64_t)c->lay_d);
    put((uint64_t)c->slab_nent);
    put((uint64_t)c->em_W);
    for (double v : c->em_dl) { uint64_t b; memcpy(&b, &v, 8); put(b); }
    const unsigned char* fb = reinterpret_cast<const unsigned char*>(&fd);
    for (size_t i = 0; i < sizeof(fd); i += 8) { uint64_t w = 0; memcpy(&w, fb + i, std::min<size_t>(8, sizeof(fd) - i)); put(w); }
    for (const DBuf* b : solve_buffers(c)) put((uint64_t)(uintptr_t)b->p);  // adjoint scratch is not in the graphs
    for (int64_t k = 0; k < S; ++k) put((uint64_t)a->n_active[k]);
  }
  // Two graphs -- the per-solve operator set-up and the step loop -- with the
  // timing events recorded on the stream between them.
  static const bool no_graph = getenv("PRINCE_B200_NO_GRAPH") != nullptr;
  if (no_graph) {
    PB_CUDA(c, cudaEventRecord(c->ev0, st));
    if ((rc = enqueue(launches))) return rc;
    PB_CUDA(c, cudaEventRecord(c->ev2, st));
    if ((rc = enqueue_steps(launches))) return rc;
    PB_CUDA(c, cudaEventRecord(c->ev3, st));
  } else {
    if (!c->graph_exec || !c->graph_exec2 || c->graph_key != key) {
      for (cudaGraphExec_t* ge : {&c->graph_exec, &c->graph_exec2})
        if (*ge) {
          cudaGraphExecDestroy(*ge);
          *ge = nullptr;
        }
      int64_t l1 = 0, l2 = 0;
      for (int part = 0; part < 2; ++part) {
        PB_CUDA(c, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int rc2 = part == 0 ? enqueue(l1) : enqueue_steps(l2);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc2) {
          if (g) cudaGraphDestroy(g);
          return rc2;
        }
        PB_CUDA(c, e);
        const cudaError_t ei = cudaGraphInstantiate(part == 0 ? &c->graph_exec : &c->graph_exec2, g, 0);
        cudaGraphDestroy(g);
        PB_CUDA(c, ei);
      }
      c->graph_key = key;
      c->graph_launches = l1 + l2;
    }
    PB_CUDA(c, cudaEventRecord(c->ev0, st));
    PB_CUDA(c, cudaGraphLaunch(c->graph_exec, st));
    PB_CUDA(c, cudaEventRecord(c->ev2, st));
    PB_CUDA(c, cudaGraphLaunch(c->graph_exec2, st));
    PB_CUDA(c, cudaEventRecord(c->ev3, st));
    launches = c->graph_launches;
  }
  const cudaMemcpyKind out_kind = a->state_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const bool ocols = a->out_cols && K > 1;
  if (ocols || rmap) {  // rows and columns in the caller's order, gathered on the device, then one copy
    if (ocols && (rc = upload(c, c->outcols, a->out_cols, (size_t)K))) return rc;
    double* Y = c->F.as<double>();  // F(x) scratch of the steps, n x ld >= n x K
    k_gather_cols<<<dim3(blocks_for(n, 8), blocks_for(K, kColTile)), 256, 0, st>>>(
        X, ld, n, K, ocols ? c->outcols.as<int>() : nullptr, rmap, Y);
    PB_CUDA(c, cudaGetLastError());
    PB_CUDA(c, cudaMemcpyAsync(a->state, Y, (size_t)n * K * sizeof(double), out_kind, st));
  } else {
    PB_CUDA(c, cudaMemcpy2DAsync(a->state, K * sizeof(double), X, ld * sizeof(double), K * sizeof(double), n,
                                 out_kind, st));
  }
  PB_CUDA(c, cudaEventRecord(c->ev1, st));
  PB_CUDA(c, cudaStreamSynchronize(st));
  if ((rc = check_wait_flag(c, "pb_solve"))) return rc;
  PB_CUDA(c, cudaEventElapsedTime(&c->last_solve_ms, c->ev0, c->ev1));
  PB_CUDA(c, cudaEventElapsedTime(&c->last_device_ms, c->ev0, c->ev3));
  PB_CUDA(c, cudaEventElapsedTime(&c->last_steps_ms, c->ev2, c->ev3));
  c->last_launches = launches;
  c->last_W = W;
  c->have_solution = true;
  c->last_ckpt = a->ckpt_every;
  c->last_S = S;
  c->last_K = K;
  c->last_flags = flags;
  c->last_scale = a->photon_scale;
  return PB_OK;
}

// The tile parameters of the bin-blocked stage, searched on the live operator:
// every (band-tile CTA warps, k_slab prefetch depth, k_slab staging) candidate
// runs the caller's (short) solve `reps` times and is scored by its fastest
// step loop (CUDA events around the step graph); the fastest candidate stays
// set on the context.  Only the batched bin-blocked path has choices.
int pb_autotune(pb_context* c, const pb_solve_args* a, int32_t reps, int32_t max_out, pb_tune_choice* out,
                int32_t* n_out) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!a || reps < 1 || max_out < 0 || (max_out > 0 && !out) || !n_out)
    return fail(c, PB_ERR_ARG, "pb_autotune: bad arguments");
  *n_out = 0;
  if (!use_blocked(c, a->n_cols)) return fail(c, PB_ERR_STATE, "pb_autotune: the solve does not run the bin-blocked kernels");
  const int32_t keep_bw = c->band_warps, keep_pre = c->slab_pre, keep_tma = c->tma_mode;
  std::vector<pb_tune_choice> cand;
  for (int tma : {1, 0})
    for (int bw : {8, 4})
      for (int pre : {2, 1, 3}) cand.push_back(pb_tune_choice{bw, pre, tma, 0.0});
  int best = -1;
  for (size_t i = 0; i < cand.size(); ++i) {
    c->band_warps = cand[i].band_warps;
    c->slab_pre = cand[i].slab_prefetch;
    c->tma_mode = cand[i].tma_staging;
    double t = 1e300;
    for (int r = 0; r < reps + 1; ++r) {  // the first run captures the candidate's graph
      const int rc = pb_solve(c, a);
      if (rc) {
        c->band_warps = keep_bw;
        c->slab_pre = keep_pre;
        c->tma_mode = keep_tma;
        return rc;
      }
      if (r > 0) t = std::min(t, (double)c->last_steps_ms);
    }
    if (cand[i].tma_staging == 1 && !c->last_tma) t = 1e300;  // tensor maps unavailable: not a candidate
    cand[i].steps_ms = t;
    if (best < 0 || t < cand[best].steps_ms) best = (int)i;
  }
  c->band_warps = cand[best].band_warps;
  c->slab_pre = cand[best].slab_prefetch;
  c->tma_mode = cand[best].tma_staging;
  // best first, then the rest in search order
  std::vector<pb_tune_choice> ordered{cand[best]};
  for (size_t i = 0; i < cand.size(); ++i)
    if ((int)i != best) ordered.push_back(cand[i]);
  const int n = std::min<int>(max_out, (int)ordered.size());
  for (int i = 0; i < n; ++i) out[i] = ordered[i];
  *n_out = n;
  return PB_OK;
}

int pb_adjoint(pb_context* c, const pb_solve_args* a, const double* seed, int32_t seed_on_device,
               double* grad_grids, double* grad_coeff, double* grad_scale) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!a || !seed) return fail(c, PB_ERR_ARG, "pb_adjoint: args and seed are required");
  if (!c->have_solution || c->last_ckpt <= 0)
    return fail(c, PB_ERR_STATE, "pb_adjoint: run pb_solve with ckpt_every > 0 first");
  if (a->n_steps != c->last_S || a->n_cols != c->last_K || a->flags != c->last_flags ||
      a->ckpt_every != c->last_ckpt || a->n_windows != c->last_W || a->photon_scale != c->last_scale)
    return fail(c, PB_ERR_ARG, "pb_adjoint: arguments differ from the checkpointed solve");
  const bool em = (a->flags & PB_EM_CASCADE) && c->have_em;
  if (em && grad_scale)
    return fail(c, PB_ERR_ARG, "pb_adjoint: no photon-scale gradient through the EM cascade transfer "
                               "(pass grad_scale = NULL with PB_EM_CASCADE)");
  const int64_t S = a->n_steps, n = c->n, R = c->R;
  const int K = a->n_cols, CK = a->ckpt_every;
  const int ld = K == 1 ? 1 : ((K + kColTile - 1) / kColTile) * kColTile;
  const uint32_t flags = a->flags;
  const bool inj = (flags & PB_INJECTION) && c->n_src > 0;
  const bool pair = (flags & PB_PAIRPROD) && (flags & PB_PARTIAL_DIFF);
  const bool want_scale = grad_scale != nullptr;
  const bool want_inj = inj && (grad_grids || grad_coeff);
  if (want_scale && !(a->photon_scale > 0.0)) return fail(c, PB_ERR_ARG, "pb_adjoint: photon scale must be positive");
  int rc = set_device(c);
  if (rc) return rc;
  cudaStream_t st = c->stream;
  PB_CUDA(c, c->d_err.ensure(sizeof(int)));
  PB_CUDA(c, cudaMemsetAsync(c->d_err.p, 0, sizeof(int), st));
  const int64_t mstride = std::max<int64_t>(R, 1);
  const size_t sb = (size_t)n * ld * sizeof(double);

  // ---- transposed M_off pattern (stable radix sort of the entries by column) --
  PB_CUDA(c, c->erow.ensure((size_t)mstride * sizeof(int)));
  PB_CUDA(c, c->tkeys.ensure((size_t)mstride * sizeof(int)));
  PB_CUDA(c, c->tvals.ensure((size_t)mstride * sizeof(int)));
  PB_CUDA(c, c->skeys.ensure((size_t)mstride * sizeof(int)));
  PB_CUDA(c, c->svals.ensure((size_t)mstride * sizeof(int)));
  PB_CUDA(c, c->t_indptr.ensure(((size_t)n + 1) * sizeof(int64_t)));
  PB_CUDA(c, c->t_indices.ensure((size_t)mstride * sizeof(int)));
  PB_CUDA(c, c->t_perm.ensure((size_t)mstride * sizeof(int)));
  int end_bit = 1;
  while (((int64_t)1 << end_bit) <= n) ++end_bit;
  size_t sort_need = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sort_need, (int*)nullptr, (int*)nullptr, (int*)nullptr, (int*)nullptr,
                                  (int)mstride, 0, end_bit);
  PB_CUDA(c, c->sort_tmp.ensure(sort_need));
  if (R > 0) {
    k_entry_rows<<<blocks_for(n, 8), 256, 0, st>>>(c->m_indptr.as<int64_t>(), n, c->erow.as<int>());
    k_transpose_keys<<<blocks_for(R, 256), 256, 0, st>>>(c->m_indices.as<int>(), c->m_indptr.as<int64_t>(), n, R,
                                                         c->tkeys.as<int>(), c->tvals.as<int>());
    size_t tb = c->sort_tmp.bytes;
    PB_CUDA(c, cub::DeviceRadixSort::SortPairs(c->sort_tmp.p, tb, c->tkeys.as<int>(), c->skeys.as<int>(),
                                               c->tvals.as<int>(), c->svals.as<int>(), (int)R, 0, end_bit, st));
    k_transpose_finish<<<blocks_for(std::max<int64_t>(R, n + 1), 256), 256, 0, st>>>(
        c->skeys.as<int>(), c->svals.as<int>(), c->erow.as<int>(), n, R, c->t_indptr.as<int64_t>(),
        c->t_indices.as<int>(), c->t_perm.as<int>());
  } else {
    PB_CUDA(c, cudaMemsetAsync(c->t_indptr.p, 0, ((size_t)n + 1) * sizeof(int64_t), st));
  }
  PB_CUDA(c, cudaGetLastError());

  // ---- work buffers ----------------------------------------------------------
  PB_CUDA(c, c->lam.ensure(sb));
  PB_CUDA(c, c->lam2.ensure(sb));
  PB_CUDA(c, c->mu.ensure(sb));
  PB_CUDA(c, c->rec_rf.ensure((size_t)CK * 4 * n * sizeof(double)));
  PB_CUDA(c, c->rec_sx.ensure(sb));
  PB_CUDA(c, c->dsig.ensure((size_t)6 * n * sizeof(double)));
  if (want_scale) {
    PB_CUDA(c, c->rec_P.ensure((size_t)CK * sb));
    PB_CUDA(c, c->rec_Q.ensure((size_t)CK * sb));
    PB_CUDA(c, c->gs.ensure(sb));
    PB_CUDA(c, cudaMemsetAsync(c->gs.p, 0, sb, st));
  }
  const int n_inj = c->n_inj_rows;
  if (want_inj) PB_CUDA(c, c->gb_inj.ensure((size_t)std::max<int64_t>(S, 1) * std::max(n_inj, 1) * ld * sizeof(double)));
  if ((rc = upload(c, c->nact, a->n_active, (size_t)std::max<int64_t>(S, 1)))) return rc;
  PB_CUDA(c, cudaMemsetAsync(c->lam.p, 0, sb, st));
  const int* rmap = c->have_row_map ? c->row_map.as<int>() : nullptr;
  const bool ocols = a->out_cols && K > 1;
  if (ocols || rmap) {  // the seed in the caller's row and column order: one copy, then a gather on the device
    if (ocols) {
      for (int j = 0; j < K; ++j)
        if (a->out_cols[j] < 0 || a->out_cols[j] >= K) return fail(c, PB_ERR_ARG, "pb_adjoint: out_cols[%d] out of range", j);
      if ((rc = upload(c, c->outcols, a->out_cols, (size_t)K))) return rc;
    }
    PB_CUDA(c, c->F.ensure(sb));
    PB_CUDA(c, cudaMemcpyAsync(c->F.p, seed, (size_t)n * K * sizeof(double),
                               seed_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    k_pick_cols<<<dim3(blocks_for(n, 8), blocks_for(K, kColTile)), 256, 0, st>>>(
        c->F.as<double>(), n, K, ocols ? c->outcols.as<int>() : nullptr, rmap, c->lam.as<double>(), ld);
    PB_CUDA(c, cudaGetLastError());
  } else {
    PB_CUDA(c, cudaMemcpy2DAsync(c->lam.p, ld * sizeof(double), seed, K * sizeof(double), K * sizeof(double), n,
                                 seed_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  }

  // ---- forward parameters (recording) and backward sweep per checkpoint segment
  StepParams p;
  memset(&p, 0, sizeof(p));
  const int ctiles = ld / (K == 1 ? 1 : kColTile);
  fill_step_params(c, p, K, ld, flags, pair, inj, S, ctiles);
  p.inv_scale = 1.0 / a->photon_scale;
  p.rec_rf = c->rec_rf.as<double>();
  p.rec_sx = c->rec_sx.as<double>();
  if (want_scale) {
    p.dsig = c->dsig.as<double>();
    p.dphi1 = p.dsig + 2 * n;
    p.dphi2 = p.dsig + 4 * n;
    p.rec_P = c->rec_P.as<double>();
    p.rec_Q = c->rec_Q.as<double>();
    if (use_blocked(c, K) && pair) {  // the bin-blocked record pass needs D_off (kappa_pair v)
      PB_CUDA(c, c->fdkp.ensure(sb));
      p.fdkp = c->fdkp.as<double>();
    }
  }
  double* lam = c->lam.as<double>();
  double* lam2 = c->lam2.as<double>();
  const int64_t nseg = (S + CK - 1) / CK;
  const int W = a->n_windows;
  // the bin-blocked sweep needs the transposed structures, one band pair and the FD table
  const bool blockedT = c->blockedT_ok && c->fdT_ok && use_blocked(c, K) && c->last_W == W;
  if (blockedT) {
    PB_CUDA(c, c->vbuf.ensure(sb));
    PB_CUDA(c, c->vbuf2.ensure(sb));
    if ((rc = ensure_tmapsT(c, ld))) return rc;
    PB_CUDA(c, c->bTbuf.ensure(sb));
    PB_CUDA(c, c->fdTbuf.ensure(sb));
    PB_CUDA(c, c->bandT_vals.ensure((size_t)W * std::max<int64_t>(c->band_stride, 1) * sizeof(double)));
    PB_CUDA(c, c->slabT_vals.ensure((size_t)W * std::max<int64_t>(c->slabT_nent, 1) * sizeof(double)));
    PB_CUDA(c, cudaMemsetAsync(c->bandT_vals.p, 0, (size_t)W * c->band_stride * sizeof(double), st));
    PB_CUDA(c, cudaMemsetAsync(c->slabT_vals.p, 0, (size_t)W * c->slabT_nent * sizeof(double), st));
    PB_CUDA(c, cudaMemsetAsync(c->bTbuf.p, 0, sb, st));
    if (R > 0)
      k_transpose_blocks<<<blocks_for(R, 256), 256, 0, st>>>(
          c->band_slot.as<int>(), c->bandT_slot.as<int>(), c->slab_slot.as<int>(), c->slabT_slot.as<int>(), R, W,
          c->band_vals.as<double>(), c->bandT_vals.as<double>(), c->band_stride, c->slab_vals.as<double>(),
          c->slab_nent, c->slabT_vals.as<double>(), c->slabT_nent);
    PB_CUDA(c, cudaGetLastError());
  }
  for (int64_t sg = nseg - 1; sg >= 0; --sg) {
    const int64_t k0 = sg * CK, k1 = std::min<int64_t>(S, k0 + CK);
    int64_t kf = k0;
    while (kf < k1 && a->n_active[kf] == 0) ++kf;
    if (kf == k1) continue;  // no active column in this segment
    p.rec_k0 = k0;
    p.rec_len = (int)(k1 - k0);
    if (want_scale) {  // the sensitivities P, Q need the states: recompute the segment from its checkpoint
      PB_CUDA(c, cudaMemcpyAsync(c->X.p, c->ckpt.as<double>() + (size_t)sg * n * ld, sb, cudaMemcpyDeviceToDevice, st));
      PB_CUDA(c, cudaMemsetAsync(c->counter.p, 0, (size_t)std::max<size_t>(c->h_long_rows.size(), 1) * ctiles * sizeof(int), st));
      launch_steps(c, p, K, a->n_active, k0, k1, st, nullptr, 0);
    } else {  // the operator factors depend on z alone: record them without recomputing the states
      for (int64_t k = kf; k < k1; ++k) {
        if (a->n_active[k] == 0) continue;
        p.step = k;
        p.step_w = c->h_win[k];
        k_prep<<<blocks_for(n, 256), 256, 0, st>>>(p);
      }
    }
    if (blockedT) {
      for (int64_t k = k1 - 1; k >= kf; --k) {
        const size_t j = (size_t)(k - k0);
        AdjBlk q;
        memset(&q, 0, sizeof(q));
        q.n = n;
        q.d = c->lay_d;
        q.nsp = c->lay_nsp;
        q.ld = ld;
        q.ncols = a->n_active[k];
        q.w = a->window[k];
        q.nb = c->band_nb;
        q.step = k;
        q.flags = p.flags;
        q.h = a->h[k];
        q.dl = a->dldz[k];
        q.bT = c->bTbuf.as<double>();
        q.fdT = c->fdTbuf.as<double>();
        q.bandT = c->bandT_vals.as<double>();
        q.band_stride = c->band_stride;
        q.slabT = c->slabT_vals.as<double>();
        q.slabT_stride = c->slabT_nent;
        q.slabT_qbase = c->slabT_rp.as<int>();
        q.slabT_q = c->slabT_offs.as<unsigned long long>();
        q.slabT_pairs = c->slabT_pairs.as<int4>();
        q.slabT_wrp = c->slabT_wrp.as<int>();
        q.slabT_maxq = c->slabT_maxbin;
        q.slabT_maxp = (c->lay_nsp + 1) / 2;
        q.fdT_cnt = c->fdT_cnt.as<int>();
        q.fdT_off = c->fdT_off.as<int>();
        q.fdT_val = c->fdT_val.as<double>();
        q.fdT_dense = c->fdT_dense.as<double>();
        q.band_spec = c->band_spec.as<int>();
        q.rf = c->rec_rf.as<double>() + j * 4 * n;
        q.rf_prev = j >= 1 ? c->rec_rf.as<double>() + (j - 1) * 4 * n : nullptr;
        q.mu = c->mu.as<double>();
        if ((flags & PB_DECAY) && c->have_decay) {
          q.lt_indptr = c->lt_indptr.as<int64_t>();
          q.lt_indices = c->lt_indices.as<int>();
          q.lt_vals = c->lt_vals.as<double>();
        }
        if (want_scale) {
          q.P = c->rec_P.as<double>() + j * n * ld;
          q.Q = c->rec_Q.as<double>() + j * n * ld;
          q.gs = c->gs.as<double>();
        }
        if (want_inj) {
          q.inj_slot = c->inj_slot.as<int>();
          q.gb_inj = c->gb_inj.as<double>() + (size_t)k * n_inj * ld;
        }
        if (em) em_hook_adjoint(em_params(c, a->window[k], ld, q.ncols, lam), st);  // the hook after step k
        if (k == k1 - 1 || em)  // v1 of the segment's last step; later steps get it from stage 2
          k_adj_v1<<<dim3(blocks_for(n, 8), blocks_for(q.ncols, kColTile)), 256, 0, st>>>(
              q.rf + 2 * n, lam, n, ld, q.ncols, c->vbuf.as<double>());
        AdjParams t;  // tail rows (species on another grid): the general adjoint kernel
        if (c->n_tail > 0) {
          memset(&t, 0, sizeof(t));
          t.n = n;
          t.row0 = c->lay_nu;
          t.ld = ld;
          t.ncols = q.ncols;
          t.step = k;
          t.flags = p.flags;
          t.h = q.h;
          t.dl = q.dl;
          t.w = q.w;
          t.t_indptr = c->t_indptr.as<int64_t>();
          t.t_indices = c->t_indices.as<int>();
          t.t_perm = c->t_perm.as<int>();
          t.m_vals = c->m_vals.as<double>() + (size_t)q.w * mstride;
          t.dt_indptr = c->dt_indptr.as<int64_t>();
          t.dt_indices = c->dt_indices.as<int>();
          t.dt_vals = c->dt_vals.as<double>();
          t.lt_indptr = q.lt_indptr;
          t.lt_indices = q.lt_indices;
          t.lt_vals = q.lt_vals;
          t.rf = q.rf;
          t.lam = lam;
          t.mu = c->mu.as<double>();
          t.lam_out = lam2;
        }
        const dim3 tgrid((unsigned)blocks_for(c->n_tail, 8), blocks_for(q.ncols, kColTile));
        q.err = c->d_err.as<int>();
        q.wait_tries = c->staging_wait_tries;
        const CUtensorMap* tm = c->tmaT_ok ? reinterpret_cast<const CUtensorMap*>(c->tmapsT.p) : nullptr;
        q.v = c->vbuf.as<double>();
        q.tmap_v = tm;
        q.lam = lam;
        q.vout = c->vbuf2.as<double>();
        launch_adj_blocked<1>(c, q, st);
        if (c->n_tail > 0) k_adj<1><<<tgrid, 256, 0, st>>>(t);
        q.v = c->vbuf2.as<double>();
        q.tmap_v = tm ? tm + 1 : nullptr;
        q.vout = c->vbuf.as<double>();
        q.lam_out = lam2;
        launch_adj_blocked<2>(c, q, st);
        if (c->n_tail > 0) k_adj<2><<<tgrid, 256, 0, st>>>(t);
        std::swap(lam, lam2);
      }
      PB_CUDA(c, cudaGetLastError());
      continue;
    }
    for (int64_t k = k1 - 1; k >= kf; --k) {
      AdjParams q;
      memset(&q, 0, sizeof(q));
      q.n = n;
      q.ld = ld;
      q.ncols = a->n_active[k];
      q.step = k;
      q.flags = p.flags;
      q.h = a->h[k];
      q.dl = a->dldz[k];
      q.w = a->window[k];
      q.t_indptr = c->t_indptr.as<int64_t>();
      q.t_indices = c->t_indices.as<int>();
      q.t_perm = c->t_perm.as<int>();
      q.m_vals = c->m_vals.as<double>() + (size_t)q.w * mstride;
      q.dt_indptr = c->dt_indptr.as<int64_t>();
      q.dt_indices = c->dt_indices.as<int>();
      q.dt_vals = c->dt_vals.as<double>();
      if ((flags & PB_DECAY) && c->have_decay) {
        q.lt_indptr = c->lt_indptr.as<int64_t>();
        q.lt_indices = c->lt_indices.as<int>();
        q.lt_vals = c->lt_vals.as<double>();
      }
      const size_t j = (size_t)(k - k0);
      q.rf = c->rec_rf.as<double>() + j * 4 * n;
      if (want_scale) {
        q.P = c->rec_P.as<double>() + j * n * ld;
        q.Q = c->rec_Q.as<double>() + j * n * ld;
        q.gs = c->gs.as<double>();
      }
      q.lam = lam;
      q.mu = c->mu.as<double>();
      q.lam_out = lam2;
      if (want_inj) {
        q.inj_slot = c->inj_slot.as<int>();
        q.gb_inj = c->gb_inj.as<double>() + (size_t)k * n_inj * ld;
      }
      if (em) em_hook_adjoint(em_params(c, a->window[k], ld, q.ncols, lam), st);  // the hook after step k
      dim3 grid(blocks_for(n, 8), K == 1 ? 1u : blocks_for(q.ncols, kColTile));
      k_adj<1><<<grid, 256, 0, st>>>(q);
      k_adj<2><<<grid, 256, 0, st>>>(q);
      std::swap(lam, lam2);
    }
    PB_CUDA(c, cudaGetLastError());
  }

  // ---- gradients ----------------------------------------------------------------
  if (want_inj) {
    PB_CUDA(c, c->g_out.ensure((size_t)std::max<int64_t>((int64_t)S * c->n_src, (int64_t)n_inj * c->n_src) * sizeof(double) + 8));
    if (grad_coeff) {
      k_grad_coeff<<<blocks_for(S * c->n_src, 256), 256, 0, st>>>(
          c->gb_inj.as<double>(), c->inj_G.as<double>(), c->s_finj.as<double>(), c->src_col_d.as<int>(),
          c->nact.as<int>(), S, c->n_src, n_inj, ld, c->g_out.as<double>());
      PB_CUDA(c, cudaMemcpyAsync(grad_coeff, c->g_out.p, (size_t)S * c->n_src * sizeof(double), cudaMemcpyDeviceToHost, st));
      PB_CUDA(c, cudaStreamSynchronize(st));
    }
    if (grad_grids) {
      k_grad_grids<<<blocks_for((int64_t)n_inj * c->n_src, 256), 256, 0, st>>>(
          c->gb_inj.as<double>(), c->s_coeff.as<double>(), c->s_finj.as<double>(), c->src_col_d.as<int>(),
          c->nact.as<int>(), S, c->n_src, n_inj, ld, c->g_out.as<double>());
      PB_CUDA(c, cudaMemcpyAsync(grad_grids, c->g_out.p, (size_t)n_inj * c->n_src * sizeof(double), cudaMemcpyDeviceToHost, st));
      PB_CUDA(c, cudaStreamSynchronize(st));
    }
  } else {
    if (grad_coeff) memset(grad_coeff, 0, (size_t)S * std::max(c->n_src, 0) * sizeof(double));
    if (grad_grids) memset(grad_grids, 0, (size_t)n_inj * std::max(c->n_src, 0) * sizeof(double));
  }
  if (want_scale) {
    PB_CUDA(c, c->g_out.ensure((size_t)std::max(K, 1) * sizeof(double) + 8));
    k_grad_scale<<<blocks_for(K, 128), 128, 0, st>>>(c->gs.as<double>(), blockedT ? (int64_t)c->lay_d : n, ld, K,
                                                       c->g_out.as<double>());
    PB_CUDA(c, cudaMemcpyAsync(grad_scale, c->g_out.p, (size_t)K * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  PB_CUDA(c, cudaGetLastError());
  PB_CUDA(c, cudaStreamSynchronize(st));
  return check_wait_flag(c, "pb_adjoint");
}

int pb_get_operator_pattern(pb_context* c, int64_t* nnz, int64_t* indptr, int32_t* indices) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_solution) return fail(c, PB_ERR_STATE, "pb_get_operator_pattern: no solve yet");
  if (!nnz) return fail(c, PB_ERR_ARG, "pb_get_operator_pattern: nnz is NULL");
  int rc = set_device(c);
  if (rc) return rc;
  int64_t tot = 0;
  PB_CUDA(c, cudaMemcpy(&tot, c->m_indptr.as<int64_t>() + c->n, sizeof(int64_t), cudaMemcpyDeviceToHost));
  *nnz = tot;
  if (indptr) PB_CUDA(c, cudaMemcpy(indptr, c->m_indptr.p, ((size_t)c->n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost));
  if (indices && tot) PB_CUDA(c, cudaMemcpy(indices, c->m_indices.p, (size_t)tot * sizeof(int), cudaMemcpyDeviceToHost));
  return PB_OK;
}

int pb_get_window(pb_context* c, int32_t w, double* offdiag, double* diag, double* kappa_pair) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (!c->have_solution) return fail(c, PB_ERR_STATE, "pb_get_window: no solve yet");
  if (w < 0 || w >= c->last_W) return fail(c, PB_ERR_ARG, "pb_get_window: window out of range");
  int rc = set_device(c);
  if (rc) return rc;
  int64_t tot = 0;
  PB_CUDA(c, cudaMemcpy(&tot, c->m_indptr.as<int64_t>() + c->n, sizeof(int64_t), cudaMemcpyDeviceToHost));
  const int64_t mstride = std::max<int64_t>(c->R, 1);
  if (offdiag && tot)
    PB_CUDA(c, cudaMemcpy(offdiag, c->m_vals.as<double>() + (size_t)w * mstride, (size_t)tot * sizeof(double),
                          cudaMemcpyDeviceToHost));
  if (diag) PB_CUDA(c, cudaMemcpy(diag, c->m_diag.as<double>() + (size_t)w * c->n, (size_t)c->n * sizeof(double), cudaMemcpyDeviceToHost));
  if (kappa_pair) PB_CUDA(c, cudaMemcpy(kappa_pair, c->kp.as<double>() + (size_t)w * c->n, (size_t)c->n * sizeof(double), cudaMemcpyDeviceToHost));
  return PB_OK;
}

int pb_integrate_const(pb_context* c, int64_t n, const double* d, int64_t nnz, const int64_t* indptr,
                       const int32_t* indices, const double* values, int64_t n_steps, const double* z_grid,
                       double* state) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (n <= 0 || n >= ((int64_t)1 << 31) || !d || nnz < 0 || n_steps < 0 || !z_grid || !state)
    return fail(c, PB_ERR_ARG, "pb_integrate_const: bad arguments");
  if (nnz > 0 && (!indptr || !indices || !values)) return fail(c, PB_ERR_ARG, "pb_integrate_const: CSR arrays missing");
  std::vector<int64_t> zp;
  if (nnz == 0) {
    zp.assign((size_t)n + 1, 0);
    indptr = zp.data();
  } else {
    if (indptr[0] != 0 || indptr[n] != nnz) return fail(c, PB_ERR_ARG, "pb_integrate_const: indptr must run from 0 to nnz");
    for (int64_t r = 0; r < n; ++r)
      if (indptr[r] > indptr[r + 1]) return fail(c, PB_ERR_ARG, "pb_integrate_const: indptr must not decrease");
    for (int64_t j = 0; j < nnz; ++j)
      if (indices[j] < 0 || indices[j] >= n) return fail(c, PB_ERR_ARG, "pb_integrate_const: column out of range");
  }
  int rc = set_device(c);
  if (rc) return rc;
  cudaStream_t st = c->stream;
  // A constant operator is one window with M_off = L_off, M_diag = d, dl/dz = 1
  // and no losses or injection.
  DBuf ip, ix, iv, dg, hs, ones, zero_i, X, A, F, rows, rowf;
  auto cleanup = [&]() {
    for (DBuf* b : {&ip, &ix, &iv, &dg, &hs, &ones, &zero_i, &X, &A, &F, &rows, &rowf}) b->release();
  };
  std::vector<double> hv((size_t)std::max<int64_t>(n_steps, 1)), one((size_t)std::max<int64_t>(n_steps, 1), 1.0);
  for (int64_t k = 0; k < n_steps; ++k) hv[k] = z_grid[k + 1] - z_grid[k];
  std::vector<int> zi((size_t)std::max<int64_t>(n_steps, 1), 0), rl((size_t)n);
  for (int64_t i = 0; i < n; ++i) rl[i] = (int)i;
  if ((rc = upload(c, ip, indptr, (size_t)n + 1)) || (rc = upload(c, ix, indices, (size_t)nnz)) ||
      (rc = upload(c, iv, values, (size_t)nnz)) || (rc = upload(c, dg, d, (size_t)n)) ||
      (rc = upload(c, hs, hv.data(), hv.size())) || (rc = upload(c, ones, one.data(), one.size())) ||
      (rc = upload(c, zero_i, zi.data(), zi.size())) || (rc = upload(c, X, state, (size_t)n)) ||
      (rc = upload(c, rows, rl.data(), rl.size()))) {
    cleanup();
    return rc;
  }
  if (A.ensure((size_t)n * sizeof(double)) != cudaSuccess || F.ensure((size_t)n * sizeof(double)) != cudaSuccess ||
      rowf.ensure((size_t)8 * n * sizeof(double)) != cudaSuccess) {
    cleanup();
    return fail(c, PB_ERR_CUDA, "pb_integrate_const: allocation failed");
  }
  StepParams p;
  memset(&p, 0, sizeof(p));
  p.n = n;
  p.ld = 1;
  p.ncols = 1;
  p.flags = PB_PHOTOHAD;
  p.h = hs.as<double>();
  p.dldz = ones.as<double>();
  p.hc = ones.as<double>();
  p.finj = ones.as<double>();
  p.win = zero_i.as<int>();
  p.m_indptr = ip.as<int64_t>();
  p.m_indices = ix.as<int>();
  p.m_vals = iv.as<double>();
  p.m_wstride = 0;
  p.m_diag = dg.as<double>();
  p.a = A.as<double>();
  p.f = F.as<double>();
  p.rows = rows.as<int>();
  p.nrows = (int)n;
  p.nsb = (int)blocks_for(n, 256);
  p.n_steps = n_steps;
  p.eD = rowf.as<double>();
  p.phi1 = p.eD + 2 * n;
  p.phi2 = p.eD + 4 * n;
  p.kap = p.eD + 6 * n;
  p.step = 0;
  if (n_steps > 0) k_prep<<<blocks_for(n, 256), 256, 0, st>>>(p);
  for (int64_t k = 0; k < n_steps; ++k) {
    p.step = k;
    p.x = X.as<double>();
    p.xout = X.as<double>();
    p.src = X.as<double>();
    k_step_plain<1><<<blocks_for(n, 256), 256, 0, st>>>(p);
    p.src = A.as<double>();
    k_step_plain<2><<<blocks_for(n, 256), 256, 0, st>>>(p);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(state, X.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cleanup();
  if (e != cudaSuccess) return fail(c, PB_ERR_CUDA, "pb_integrate_const: %s", cudaGetErrorString(e));
  return PB_OK;
}

// No-allocation variant of pb_integrate_const.  The scratch is the static
// device array g_noalloc_scratch; its device address is looked up with
// cudaGetSymbolAddress once per device (on that device's first call) and
// cached, which assumes the device's primary context lives as long as the
// process (a cudaDeviceReset by any component of the process invalidates the
// cached address).  Nothing here allocates or frees device memory.
static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[64] = {nullptr};

int pb_integrate_const_noalloc(pb_context* c, int64_t n, const double* d, int64_t nnz, const int64_t* indptr,
                               const int32_t* indices, const double* values, int64_t n_steps,
                               const double* z_grid, double* state) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (n <= 0 || n > kNaMaxStates)
    return fail(c, PB_ERR_ARG, "pb_integrate_const_noalloc: n = %lld outside [1, %lld] (static scratch limit)",
                (long long)n, (long long)kNaMaxStates);
  if (n_steps < 0 || n_steps > kNaMaxSteps)
    return fail(c, PB_ERR_ARG, "pb_integrate_const_noalloc: n_steps = %lld outside [0, %lld] (static scratch limit)",
                (long long)n_steps, (long long)kNaMaxSteps);
  if (!d || !z_grid || !state || nnz < 0 || (nnz > 0 && (!indptr || !indices || !values)))
    return fail(c, PB_ERR_ARG, "pb_integrate_const_noalloc: bad arguments");
  if (c->device < 0 || c->device >= 64) return fail(c, PB_ERR_ARG, "pb_integrate_const_noalloc: device id too large");
  int rc = set_device(c);
  if (rc) return rc;
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[c->device]) {
      void* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr)
        return fail(c, PB_ERR_CUDA, "pb_integrate_const_noalloc: cudaGetSymbolAddress failed: %s",
                    cudaGetErrorString(e));
      g_noalloc_addr[c->device] = ptr;
    }
    base = static_cast<unsigned char*>(g_noalloc_addr[c->device]);
  }
  double* a = reinterpret_cast<double*>(base);
  double* f = a + kNaMaxStates;
  double* rowf = f + kNaMaxStates;
  double* h = rowf + 8 * kNaMaxStates;
  double* ones = h + kNaMaxSteps;
  int* win = reinterpret_cast<int*>(ones + kNaMaxSteps);
  int* rows = win + kNaMaxSteps;
  int64_t* zero_indptr = reinterpret_cast<int64_t*>(rows + kNaMaxStates);
  unsigned int* csr_flag = reinterpret_cast<unsigned int*>(zero_indptr + kNaMaxStates + 1);
  cudaStream_t st = c->stream;
  if (nnz > 0) {
    // The step kernels index state[indices[j]] for j in [indptr[r], indptr[r+1]):
    // check the caller's CSR first, and run nothing on a malformed one.
    unsigned int bad = 0;
    cudaError_t e = cudaMemsetAsync(csr_flag, 0, sizeof(unsigned int), st);
    if (e == cudaSuccess) {
      k_noalloc_check_csr<<<blocks_for(std::max<int64_t>(n + 1, nnz), 256), 256, 0, st>>>(n, nnz, indptr, indices,
                                                                                         csr_flag);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, csr_flag, sizeof(unsigned int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(c, PB_ERR_CUDA, "pb_integrate_const_noalloc: %s", cudaGetErrorString(e));
    if (bad & 1u)
      return fail(c, PB_ERR_ARG, "pb_integrate_const_noalloc: malformed CSR row pointers (need indptr[0] = 0, "
                                 "non-decreasing, indptr[n] = nnz)");
    if (bad & 2u) return fail(c, PB_ERR_ARG, "pb_integrate_const_noalloc: CSR column index outside [0, n)");
  }
  const int64_t fill = std::max<int64_t>(n + 1, n_steps);
  k_noalloc_fill<<<blocks_for(fill, 256), 256, 0, st>>>(n, n_steps, z_grid, h, ones, win, rows, zero_indptr);
  StepParams p;
  memset(&p, 0, sizeof(p));
  p.n = n;
  p.ld = 1;
  p.ncols = 1;
  p.flags = PB_PHOTOHAD;
  p.h = h;
  p.dldz = ones;
  p.hc = ones;
  p.finj = ones;
  p.win = win;
  p.m_indptr = nnz > 0 ? indptr : zero_indptr;
  p.m_indices = indices;
  p.m_vals = values;
  p.m_wstride = 0;
  p.m_diag = d;
  p.a = a;
  p.f = f;
  p.rows = rows;
  p.nrows = (int)n;
  p.nsb = (int)blocks_for(n, 256);
  p.n_steps = n_steps;
  p.eD = rowf;
  p.phi1 = rowf + 2 * n;
  p.phi2 = rowf + 4 * n;
  p.kap = rowf + 6 * n;
  p.step = 0;
  if (n_steps > 0) k_prep<<<blocks_for(n, 256), 256, 0, st>>>(p);
  for (int64_t k = 0; k < n_steps; ++k) {
    p.step = k;
    p.x = state;
    p.xout = state;
    p.src = state;
    k_step_plain<1><<<blocks_for(n, 256), 256, 0, st>>>(p);
    p.src = a;
    k_step_plain<2><<<blocks_for(n, 256), 256, 0, st>>>(p);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(c, PB_ERR_CUDA, "pb_integrate_const_noalloc: %s", cudaGetErrorString(e));
  return PB_OK;
}

int pb_eval_exp(pb_context* c, int64_t n, const double* x, double* y) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (n < 0 || (n > 0 && (!x || !y))) return fail(c, PB_ERR_ARG, "pb_eval_exp: bad arguments");
  if (n == 0) return PB_OK;
  int rc = set_device(c);
  if (rc) return rc;
  DBuf dx, dy;
  if ((rc = upload(c, dx, x, (size_t)n))) return rc;
  if (dy.ensure((size_t)n * sizeof(double)) != cudaSuccess) {
    dx.release();
    return fail(c, PB_ERR_CUDA, "pb_eval_exp: allocation failed");
  }
  k_eval_exp<<<blocks_for(n, 256), 256, 0, c->stream>>>(dx.as<double>(), dy.as<double>(), n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(y, dy.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  dx.release();
  dy.release();
  if (e != cudaSuccess) return fail(c, PB_ERR_CUDA, "pb_eval_exp: %s", cudaGetErrorString(e));
  return PB_OK;
}

int pb_last_timing(pb_context* c, double* solve_ms, double* device_ms, double* steps_ms, int64_t* launches) {
  if (!c) return fail(nullptr, PB_ERR_ARG, "context is NULL");
  if (solve_ms) *solve_ms = c->last_solve_ms;
  if (device_ms) *device_ms = c->last_device_ms;
  if (steps_ms) *steps_ms = c->last_steps_ms;
  if (launches) *launches = c->last_launches;
  return PB_OK;
}

}  // extern "C"
