// kernels_learned.cuh -- the learned k-proposal of the RBE force: an exact sampler of
// q(m) = p(m) e^{h(b(m))} / Z over the lattice m in Z^3 \ {0} with |m_d| <= M_d, where p is RBE's
// Gaussian p(m) ~ exp(-pi^2 sum_d m_d^2 / (alpha L_d^2)) (RBEPSample.h:86-114), b(m) one of 256 bins
// of kappa = |k| / (2 sqrt(alpha)) on [0, 6) and h the network's output for that bin; the
// importance weight w = p(m) / q(m) = Z e^{-h} keeps the RBE estimator unbiased.  Also: the
// conditioning spectrum (importance-weighted band means of |rho_k|^2 / N_q, updated every step),
// the network inputs of each bin, and the training data of a snapshot (exact rho_k and the
// per-sample variance weight at k-vectors drawn from p).
#pragma once
#include <cmath>
#include <cstdint>

#include "common.cuh"
#include "kernels_force.cuh"
#include "mlp_forward.cuh"
#include "mlp_types.cuh"

namespace rbmd {

constexpr int kPropBins = 256;
constexpr int kPropBands = 8;
constexpr double kPropKappaMax = 6.0;     // bins cover kappa in [0, 6); p's tail beyond is < e^-36
constexpr double kPropBandWidth = 0.5;    // conditioning bands: kappa in [0.5 j, 0.5 (j + 1)), last open
constexpr int kPropMaxM = 960;            // CDF tables staged in shared memory up to this |m_d|

struct PropRep {
  double c[3];          // 2 pi / L_d
  double kscale;        // 1 / (2 sqrt(alpha))
  int M[3];             // support |m_d| <= M_d
  int cdf_off[3];       // offsets of the per-axis CDF tables (2 M_d + 1 entries each)
  int nq;               // charged atoms of the replica
  int pad;
};

// shared memory of k_prop_sample for a replica: its three CDF tables when they are staged
// (|m_d| <= kPropMaxM), else none
__host__ __device__ __forceinline__ int prop_stage_doubles(const PropRep& pr) {
  if (pr.M[0] > kPropMaxM || pr.M[1] > kPropMaxM || pr.M[2] > kPropMaxM) return 0;
  return (2 * pr.M[0] + 1) + (2 * pr.M[1] + 1) + (2 * pr.M[2] + 1);
}

// |k| bin of an integer vector; identical arithmetic on host and device (no contraction)
__host__ __device__ __forceinline__ double prop_kappa(const PropRep& pr, int mx, int my, int mz) {
#ifdef __CUDA_ARCH__
  const double k0 = __dmul_rn(pr.c[0], (double)mx), k1 = __dmul_rn(pr.c[1], (double)my),
               k2 = __dmul_rn(pr.c[2], (double)mz);
  const double s = __dadd_rn(__dadd_rn(__dmul_rn(k0, k0), __dmul_rn(k1, k1)), __dmul_rn(k2, k2));
  return __dmul_rn(__dsqrt_rn(s), pr.kscale);
#else
  const double k0 = pr.c[0] * (double)mx, k1 = pr.c[1] * (double)my, k2 = pr.c[2] * (double)mz;
  const double s = (k0 * k0 + k1 * k1) + k2 * k2;
  return std::sqrt(s) * pr.kscale;
#endif
}
__host__ __device__ __forceinline__ int prop_bin(double kappa) {
  const int b = (int)(kappa * (kPropBins / kPropKappaMax));
  return b < kPropBins ? b : kPropBins - 1;
}
__host__ __device__ __forceinline__ int prop_band(double kappa) {
  const int j = (int)(kappa / kPropBandWidth);
  return j < kPropBands ? j : kPropBands - 1;
}

// network inputs of bin b under the conditioning spectrum spec[8] (log band means)
__device__ __forceinline__ void prop_features(int b, const float* spec, float* x) {
  const float kap = (float)((b + 0.5) * (kPropKappaMax / kPropBins));
  const float u = kap / 3.0f;
  x[0] = u;
  x[1] = u * u;
  x[2] = sqrtf(u);
  x[3] = expf(-kap * kap);
#pragma unroll
  for (int j = 0; j < kPropBands; ++j) x[4 + j] = spec[j];
#pragma unroll
  for (int j = 4 + kPropBands; j < kMlpIn; ++j) x[j] = 0.f;
}

// inputs of every (group, bin) row; spec_of_group[g * 8 .. + 8]
__global__ void k_prop_features(int groups, const float* __restrict__ spec, float* __restrict__ x) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= groups * kPropBins) return;
  prop_features(row % kPropBins, spec + (size_t)(row / kPropBins) * kPropBands, x + (size_t)row * kMlpIn);
}

// h of every (replica, bin) row under the replica's conditioning spectrum: the bin's inputs
// (prop_features) and the network's forward pass on the CUDA cores (mlp_row_forward, kMlpLanes
// lanes per row, 256-thread blocks over several SMs; mlp_t = the prepared weights, k_mlp_prep).  The sampler's per-step evaluation: a
// tensor-core launch with its 94 KB of shared memory and TMEM only finds an SM once one drains
// under the near pass, and would open the k-space chain late.
__global__ void __launch_bounds__(256) k_prop_h(int nrep, const float* __restrict__ mlp_t,
                                               const float* __restrict__ spec, float* __restrict__ h) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int rows = nrep * kPropBins;
  const int row = min(gt / kMlpLanes, rows - 1);   // every lane joins the shuffles
  float x[kMlpIn];
  prop_features(row % kPropBins, spec + (size_t)(row / kPropBins) * kPropBands, x);
  const float v = mlp_row_forward<kMlpLanes>(mlp_t, x, gt % kMlpLanes);
  if (gt / kMlpLanes < rows && gt % kMlpLanes == 0) h[row] = v;
}

// 53-bit uniform in (0, 1) from two 32-bit words
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
  return ((double)(((unsigned long long)a << 21) | (b >> 11)) + 0.5) * (1.0 / 9007199254740992.0);
}

// smallest i in [0, n) with cdf[i] >= u (cdf[n - 1] == 1)
__device__ __forceinline__ int cdf_search(const double* cdf, int n, double u) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (cdf[mid] >= u) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Draw the P k-samples of each replica (one block of kSampThreads threads per replica: a round of
// that many candidates usually completes the set, and the block's 32 warps keep their share of an
// SM that the near pass also occupies).  Candidates are exact draws from p (inverse CDF per axis,
// 53-bit uniforms from Philox4x32-10 keyed by seed, counter (round * kSampThreads + thread,
// replica, step)); m = 0 is rejected; a candidate in bin b is
// accepted with probability e^{h_b - h_max} (h clamped below at h_max - 8), so accepted samples
// follow q; they are emitted in (round, thread) order, which makes the draw deterministic.
// Weight w = Z / e^{h_b - h_max} with Z = sum_b W_b e^{h_b - h_max} (W_b = p-mass of bin b),
// i.e. p / q.  h == nullptr samples p itself with unit weights.  When max_rounds run out the
// remaining samples get weight 0 and RBMD_FLAG_SAMPLER is raised.
constexpr int kSampThreads = 1024;
__global__ void __launch_bounds__(kSampThreads) k_prop_sample(
    int nrep, const RepDev* __restrict__ reps, const PropRep* __restrict__ prep, const double* __restrict__ cdf,
    const float* __restrict__ h, const double* __restrict__ wbin, unsigned long long seed, long long step_arg,
    const long long* __restrict__ step_dev, int max_rounds, int* __restrict__ kvec_out, void* __restrict__ krec, int rec_bytes, int* __restrict__ krep,
    double* __restrict__ weights, uint32_t* status) {
  const int r = blockIdx.x;
  if (r >= nrep) return;
  const long long step = step_dev ? *step_dev : step_arg;   // device counter under graph replay
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  constexpr int kW = kSampThreads / 32;
  const PropRep pr = prep[r];
  const int P = reps[r].P, kb = reps[r].k_begin;
  __shared__ float acc_s[kPropBins];
  __shared__ double red[kW];
  __shared__ double zsum;
  __shared__ int wcount[kW];
  __shared__ int total;
  // the three per-axis CDF tables, sized by the launch (prop_stage_bytes) for the largest
  // staged replica, so that the block asks for no more shared memory than it uses
  extern __shared__ double cdf_s[];
  const int n0 = 2 * pr.M[0] + 1, n1 = 2 * pr.M[1] + 1, n2 = 2 * pr.M[2] + 1;
  const bool staged = pr.M[0] <= kPropMaxM && pr.M[1] <= kPropMaxM && pr.M[2] <= kPropMaxM;
  const bool learned = h != nullptr;
  const double *c0 = cdf + pr.cdf_off[0], *c1 = cdf + pr.cdf_off[1], *c2 = cdf + pr.cdf_off[2];
  if (staged) {
    for (int i = t; i < n0; i += kSampThreads) cdf_s[i] = c0[i];
    for (int i = t; i < n1; i += kSampThreads) cdf_s[n0 + i] = c1[i];
    for (int i = t; i < n2; i += kSampThreads) cdf_s[n0 + n1 + i] = c2[i];
    c0 = cdf_s;
    c1 = cdf_s + n0;
    c2 = cdf_s + n0 + n1;
  }
  // acceptance per bin and the normaliser Z (threads t < kPropBins, one bin each; block
  // reductions over their 8 warps in a fixed order)
  constexpr int kBW = kPropBins / 32;
  const bool bin_t = t < kPropBins;
  const float hv = (h && bin_t) ? h[(size_t)r * kPropBins + t] : 0.f;
  float hmax = hv;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) hmax = fmaxf(hmax, __shfl_xor_sync(0xffffffffu, hmax, o));
  if (lane == 0 && bin_t) red[wid] = hmax;
  __syncthreads();
  hmax = (float)red[0];
  for (int k = 1; k < kBW; ++k) hmax = fmaxf(hmax, (float)red[k]);
  __syncthreads();
  const float acc = learned ? __expf(fmaxf(hv - hmax, -8.0f)) : 1.0f;
  if (bin_t) acc_s[t] = acc;
  double zpart = bin_t ? wbin[(size_t)r * kPropBins + t] * (double)acc : 0.0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) zpart += __shfl_xor_sync(0xffffffffu, zpart, o);
  if (lane == 0 && bin_t) red[wid] = zpart;
  __syncthreads();
  if (t == 0) {
    double z = 0;
    for (int k = 0; k < kBW; ++k) z += red[k];
    zsum = z;
    total = 0;
  }
  __syncthreads();
  const double Z = zsum;
  const uint32_t k0 = (uint32_t)seed ^ 0x5bd1e995u, k1 = (uint32_t)(seed >> 32) ^ 0x9e3779b9u;
  for (int round = 0; round < max_rounds; ++round) {
    const int done = total;
    if (done >= P) break;
    uint32_t ca[4] = {(uint32_t)(round * kSampThreads + t), (uint32_t)r, (uint32_t)(unsigned long long)step,
                      (uint32_t)((unsigned long long)step >> 32)};
    uint32_t cb[4] = {ca[0], ca[1] | 0x80000000u, ca[2], ca[3]};
    philox4x32(ca, k0, k1);
    philox4x32(cb, k0, k1);
    const int mx = cdf_search(c0, n0, u53(ca[0], ca[1])) - pr.M[0];
    const int my = cdf_search(c1, n1, u53(ca[2], ca[3])) - pr.M[1];
    const int mz = cdf_search(c2, n2, u53(cb[0], cb[1])) - pr.M[2];
    const double ua = u53(cb[2], cb[3]);
    int b = 0;
    bool take = !(mx == 0 && my == 0 && mz == 0);
    if (take) {
      b = prop_bin(prop_kappa(pr, mx, my, mz));
      take = ua < (double)acc_s[b];
    }
    const unsigned bal = __ballot_sync(0xffffffffu, take);
    if (lane == 0) wcount[wid] = __popc(bal);
    __syncthreads();
    int before = 0, sum = 0;
    for (int k = 0; k < kW; ++k) {
      if (k < wid) before += wcount[k];
      sum += wcount[k];
    }
    const int pos = done + before + __popc(bal & ((1u << lane) - 1u));
    if (take && pos < P) {
      const int g = kb + pos;
      int* o = kvec_out + 3 * g;
      o[0] = mx; o[1] = my; o[2] = mz;
      int* rec = reinterpret_cast<int*>(reinterpret_cast<char*>(krec) + (size_t)g * rec_bytes);
      rec[0] = mx; rec[1] = my; rec[2] = mz;
      krep[g] = r;
      weights[g] = learned ? Z / (double)acc_s[b] : 1.0;
    }
    __syncthreads();
    if (t == 0) total = done + sum;
    __syncthreads();
  }
  if (total < P) {
    if (t == 0) set_flag(status, kFlagSampler);
    for (int i = total + t; i < P; i += kSampThreads) {
      const int g = kb + i;
      int* o = kvec_out + 3 * g;
      o[0] = 1; o[1] = 0; o[2] = 0;
      int* rec = reinterpret_cast<int*>(reinterpret_cast<char*>(krec) + (size_t)g * rec_bytes);
      rec[0] = 1; rec[1] = 0; rec[2] = 0;
      krep[g] = r;
      weights[g] = 0.0;
    }
  }
}

// Conditioning spectrum of each replica (one block of 256 threads per replica): the
// importance-weighted mean of |rho_k|^2 / N_q over this step's samples in band j (weights w make
// it an estimate of the p-average, the quantity the training data record), folded into an
// exponential moving average of its logarithm (rate beta; the first update replaces).  Thread t
// accumulates samples t, t + 256, ...; the per-band partials are summed in a fixed order (warp
// butterflies, then the warps in order).
__global__ void __launch_bounds__(256) k_prop_spectrum(int nrep, const RepDev* __restrict__ reps,
                                                       const PropRep* __restrict__ prep,
                                                       const int* __restrict__ kvec, const double2* __restrict__ rho,
                                                       const double* __restrict__ weights, float beta,
                                                       float* __restrict__ spec, int* __restrict__ spec_init) {
  const int r = blockIdx.x, t = threadIdx.x;
  if (r >= nrep) return;
  const PropRep pr = prep[r];
  const int P = reps[r].P, kb = reps[r].k_begin;
  __shared__ double wsw[8][kPropBands], wss[8][kPropBands];   // per-warp band sums
  double sw[kPropBands], ss[kPropBands];
#pragma unroll
  for (int j = 0; j < kPropBands; ++j) sw[j] = ss[j] = 0.0;
  for (int i = t; i < P; i += 256) {
    const int g = kb + i;
    const int j = prop_band(prop_kappa(pr, kvec[3 * g], kvec[3 * g + 1], kvec[3 * g + 2]));
    const double w = weights ? weights[g] : 1.0;
    const double2 z = rho[g];
#pragma unroll
    for (int b = 0; b < kPropBands; ++b)
      if (b == j) {
        sw[b] += w;
        ss[b] += w * (z.x * z.x + z.y * z.y);
      }
  }
  // fixed-order reduction: a butterfly within each warp, then the 8 warp sums in warp order
#pragma unroll
  for (int j = 0; j < kPropBands; ++j)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sw[j] += __shfl_xor_sync(0xffffffffu, sw[j], o);
      ss[j] += __shfl_xor_sync(0xffffffffu, ss[j], o);
    }
  if ((t & 31) == 0)
#pragma unroll
    for (int j = 0; j < kPropBands; ++j) {
      wsw[t >> 5][j] = sw[j];
      wss[t >> 5][j] = ss[j];
    }
  __syncthreads();
  if (t < kPropBands) {
    double a = 0, b = 0;
    for (int k = 0; k < 8; ++k) {
      a += wsw[k][t];
      b += wss[k][t];
    }
    if (a > 0 && pr.nq > 0) {
      const float v = (float)log(fmax(b / (a * (double)pr.nq), 1e-6));
      float& sv = spec[r * kPropBands + t];
      sv = spec_init[r] ? (1.f - beta) * sv + beta * v : v;
    }
  }
  __syncthreads();
  if (t == 0) spec_init[r] = 1;
}

// ---------------- training data of one snapshot ----------------
// K k-vectors (drawn from p) against the nq charged atoms of one replica in fixed point.
// Pass 0: partial rho_k; pass 1: partial sum_i q_i^2 (c_i Im rho_k - s_i Re rho_k)^2, the squared
// norm (up to the factor (4 pi qqr2e |k| / (V k^2))^2) of the force field of this one sample.
// Grid: (K / 256, atom chunks); thread = one k; atoms staged in shared memory.
constexpr int kTrainChunk = 4096;
__global__ void __launch_bounds__(256) k_train_pass(int pass, int K, int nq, const Frac32* __restrict__ frac,
                                                    const int* __restrict__ kv, const double2* __restrict__ rho,
                                                    float* __restrict__ partial) {
  __shared__ Frac32 stage[256];
  const int k = blockIdx.x * 256 + threadIdx.x;
  const bool ok = k < K;
  const uint32_t mx = ok ? (uint32_t)kv[3 * k] : 0u, my = ok ? (uint32_t)kv[3 * k + 1] : 0u,
                 mz = ok ? (uint32_t)kv[3 * k + 2] : 0u;
  float rre = 0.f, rim = 0.f;
  if (pass == 1 && ok) {
    rre = (float)rho[k].x;
    rim = (float)rho[k].y;
  }
  const int a0 = blockIdx.y * kTrainChunk, a1 = min(nq, a0 + kTrainChunk);
  float s0 = 0.f, s1 = 0.f;
  for (int base = a0; base < a1; base += 256) {
    const int cnt = min(256, a1 - base);
    __syncthreads();
    if ((int)threadIdx.x < cnt) stage[threadIdx.x] = frac[base + threadIdx.x];
    __syncthreads();
    if (!ok) continue;
    for (int a = 0; a < cnt; ++a) {
      const Frac32 f = stage[a];
      float s, c;
      turn_sincos(mx * f.x + my * f.y + mz * f.z, s, c);   // angle shifted by half a turn
      if (pass == 0) {
        s0 = fmaf(f.q, c, s0);
        s1 = fmaf(f.q, s, s1);
      } else {
        const float v = f.q * (c * rim - s * rre);         // rho from pass 0 carries the same shift
        s0 = fmaf(v, v, s0);
      }
    }
  }
  if (ok) {
    const size_t o = ((size_t)blockIdx.y * K + k) * 2;
    partial[o] = s0;
    partial[o + 1] = s1;
  }
}

// fixed-order FP64 sum of the chunk partials; pass 0 -> rho (shifted convention kept), pass 1 ->
// a_k = sum / |k|^2 (the k-dependent factor of the squared force norm) and the sample's bin and
// band (bin | band << 16)
__global__ void k_train_finish(int pass, int K, int nchunks, const PropRep* __restrict__ prep,
                               const int* __restrict__ kv, const float* __restrict__ partial,
                               double2* __restrict__ rho, double* __restrict__ ak, int* __restrict__ kbin) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  double a = 0, b = 0;
  for (int c = 0; c < nchunks; ++c) {
    a += (double)partial[((size_t)c * K + k) * 2];
    b += (double)partial[((size_t)c * K + k) * 2 + 1];
  }
  if (pass == 0) {
    rho[k] = make_double2(a, b);
  } else {
    const PropRep pr = prep[0];
    const double kap = prop_kappa(pr, kv[3 * k], kv[3 * k + 1], kv[3 * k + 2]);
    const double k2 = kap * kap / (pr.kscale * pr.kscale);
    ak[k] = a / k2;
    kbin[k] = prop_bin(kap) | (prop_band(kap) << 16);
  }
}

// Per snapshot (one block, thread b = bin): C_b = (1/K) sum of a_k over the samples in bin b (an
// unbiased estimate of sum_{m in b} a(m) / p(m), since the samples come from p), and the
// conditioning spectrum of the snapshot (log band means of |rho_k|^2 / N_q).  Deterministic.
__global__ void k_train_bins(int K, int nq, const int* __restrict__ kbin, const double2* __restrict__ rho,
                             const double* __restrict__ ak, float* __restrict__ cbin, float* __restrict__ spec) {
  const int b = threadIdx.x;
  double cs = 0, bs = 0;
  int bn = 0;
  for (int k = 0; k < K; ++k) {
    const int code = __ldg(kbin + k);
    if ((code & 0xFFFF) == b) cs += ak[k];
    if (b < kPropBands && (code >> 16) == b) {
      bs += rho[k].x * rho[k].x + rho[k].y * rho[k].y;
      ++bn;
    }
  }
  cbin[b] = (float)(cs / (double)K);
  if (b < kPropBands) spec[b] = bn > 0 ? (float)log(fmax(bs / ((double)bn * (double)nq), 1e-6)) : 0.f;
}

}  // namespace rbmd
