// kernels_force.cuh -- near-field pair force (LJ 12-6 + real-space erfc Coulomb), the RBE
// k-space force fused into the same per-atom pass, RBE structure factors, the RBE k-sampler,
// and the EAM density / force passes.
#pragma once
#include <type_traits>

#include "common.cuh"
#include "kernels_bonded.cuh"

namespace rbmd {

// ------------------------------------------------------------------------------------------
// k-sample record: integer m vector plus the per-sample force coefficient w*k (w folds S/P,
// qqr2e, -4 pi / (V k^2), the importance weight and the sign of the phase convention) and the
// structure factor rho = sum_j q_j e^{i k.r_j}.  32 B (FP32) so that a record is two 16-byte
// shared-memory loads; the owning replica of record g is krep[g].
// ------------------------------------------------------------------------------------------
struct KRec32 { int mx, my, mz; float wx, wy, wz, re, im; };                 // 32 B
struct KRec64 { int mx, my, mz, pad; double wx, wy, wz, re, im, pad2; };     // 64 B

// phase -> (cos, sin) of 2*pi*(t - 1/2) for a 32-bit fixed-point turn t: the top 23 bits form a
// float in [1, 2), so tf - 1.5 lies in [-0.5, 0.5); MUFU sin/cos are accurate on [-pi, pi].
__device__ __forceinline__ void turn_sincos(uint32_t ph, float& s, float& c) {
  float tf = __uint_as_float((ph >> 9) | 0x3F800000u) - 1.5f;
  float th = tf * 6.28318530717958647692f;
  __sincosf(th, &s, &c);
}
// 64-bit fixed-point turn -> exact double angle 2*pi*(t - 1/2) with t - 1/2 in [-0.5, 0.5)
__device__ __forceinline__ void turn_sincos(unsigned long long ph, double& s, double& c) {
  long long sg = (long long)(ph ^ 0x8000000000000000ull);   // (t - 1/2) * 2^64 as signed
  double t = (double)sg * 5.42101086242752217e-20;           // 2^-64
  sincospi(2.0 * t, &s, &c);
}

struct LJTable {
  float lj24_f[kMaxReplicaTypes * kMaxReplicaTypes];    // -24 sqrt(eps_i eps_j)  (float)
  float sig6_f[kMaxReplicaTypes * kMaxReplicaTypes];    // ((sig_i + sig_j)/2)^6   (float)
  double lj24_d[kMaxReplicaTypes * kMaxReplicaTypes];
  double sig6_d[kMaxReplicaTypes * kMaxReplicaTypes];
};

struct NearParams {
  int n, stride, ntypes, cap;
  int with_lj, with_coul, molecular;
  double rc, alpha, coul_scale;   // coul_scale multiplies the erfc Coulomb pair force
  double sqrt_alpha, two_sqrt_alpha_over_sqrt_pi;
  int kstage;                     // records of shared memory available for k staging
  int orig;                       // neighbour type "ORIGINAL": pairs with d^2 < rc^2 (no 1e-4 margin)
  SpecialDev sp;                  // molecular == 2: special-bond partner lists
};

template <class R> struct KRec;
template <> struct KRec<float> { using T = KRec32; };
template <> struct KRec<double> { using T = KRec64; };
template <class R> struct FracT;
template <> struct FracT<float> { using T = Frac32; };
template <> struct FracT<double> { using T = Frac64; };

__device__ __forceinline__ float exp_r(float x) { return __expf(x); }
__device__ __forceinline__ double exp_r(double x) { return exp(x); }
__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }
__device__ __forceinline__ float sqrt_r(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_r(double x) { return sqrt(x); }
__device__ __forceinline__ double rsqrt_r(double x) { return 1.0 / sqrt(x); }

// erfc(x) for x >= 0 given e = exp(-x^2).  FP32: Abramowitz & Stegun, Handbook of Mathematical
// Functions, eq. 7.1.26 (rational approximation in t = 1/(1 + p x), |error| <= 1.5e-7), which
// reuses the Gaussian factor the real-space force needs anyway.  FP64: the library erfc.
__device__ __forceinline__ float erfc_shared(float x, float e) {
  const float t = __frcp_rn(fmaf(0.3275911f, x, 1.0f));
  float poly = fmaf(1.061405429f, t, -1.453152027f);
  poly = fmaf(poly, t, 1.421413741f);
  poly = fmaf(poly, t, -0.284496736f);
  poly = fmaf(poly, t, 0.254829592f);
  return poly * t * e;
}
__device__ __forceinline__ double erfc_shared(double x, double) { return erfc(x); }

template <class R> __host__ __device__ __forceinline__ R lj24(const LJTable& t, int k);
template <> __host__ __device__ __forceinline__ float lj24<float>(const LJTable& t, int k) { return t.lj24_f[k]; }
template <> __host__ __device__ __forceinline__ double lj24<double>(const LJTable& t, int k) { return t.lj24_d[k]; }
template <class R> __host__ __device__ __forceinline__ R sig6(const LJTable& t, int k);
template <> __host__ __device__ __forceinline__ float sig6<float>(const LJTable& t, int k) { return t.sig6_f[k]; }
template <> __host__ __device__ __forceinline__ double sig6<double>(const LJTable& t, int k) { return t.sig6_d[k]; }

// RBE force terms of one atom over k records [0, P) of `kr` (shared or global memory).
template <class R>
__device__ __forceinline__ void rbe_terms(const typename FracT<R>::T& fr, const typename KRec<R>::T* kr,
                                          int P, R& ax, R& ay, R& az) {
#pragma unroll 4
  for (int l = 0; l < P; ++l) {
    const typename KRec<R>::T k = kr[l];
    R s, c;
    if constexpr (sizeof(R) == 4) {
      const uint32_t ph = (uint32_t)k.mx * fr.x + (uint32_t)k.my * fr.y + (uint32_t)k.mz * fr.z;
      turn_sincos(ph, s, c);
    } else {
      const unsigned long long ph = (unsigned long long)(long long)k.mx * fr.x +
                                    (unsigned long long)(long long)k.my * fr.y +
                                    (unsigned long long)(long long)k.mz * fr.z;
      turn_sincos(ph, s, c);
    }
    const R val = c * (R)k.im - s * (R)k.re;
    ax += val * (R)k.wx;
    ay += val * (R)k.wy;
    az += val * (R)k.wz;
  }
}

// Minimum-image handling of the pair vector in the near pass:
//   kMiNone  every replica has >= 3 cells per axis and the list is rebuilt every step: listed
//            pairs have |r_d| < rc < L/2, MinDistanceVec is the identity;
//   kMiLJ    the reference's semantics for small boxes: MinDistanceVec on the LJ vector only;
//   kMiAll   Verlet skin: pairs listed at rc + skin are filtered by the list predicate at rc;
//            the cached positions are unwrapped since the build (k_regather), so the stored
//            image shift still gives the minimum-image vector.
constexpr int kMiNone = 0, kMiLJ = 1, kMiAll = 2;
// Added to MI: the LJ pairs of one bond-graph component take their special-bond weight
// (molecular == 2).  A separate instantiation, so the passes without topology carry none of it.
constexpr int kMiSpecial = 4;

template <class R>
__device__ __forceinline__ void min_image(R& q0, R& q1, R& q2, const R* box) {
  if (fabs(q0) > box[0] * (R)0.5) q0 -= (q0 > 0 ? box[0] : -box[0]);
  if (fabs(q1) > box[1] * (R)0.5) q1 -= (q1 > 0 ? box[1] : -box[1]);
  if (fabs(q2) > box[2] * (R)0.5) q2 -= (q2 > 0 ? box[2] : -box[2]);
}

// approximate reciprocal (one MUFU op, about 1 ulp): the pair terms carry a 1e-5 budget
__device__ __forceinline__ float rcp_r(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ double rcp_r(double x) { return 1.0 / x; }

// Near force of one slot per thread over its transposed list row (nbr[p * stride + slot]).
// Pair physics: ComputeNearForceVerletWorklet / ComputeLJForceVerletWorklet
// (rbmd/framework/run/worklet/RunWorklet.cpp:170-303) with ComputeLJForce and
// ComputeNearEnergyForce (rbmd/framework/forceFunction/ExecForceFunction.h:74-140):
//   LJ on MinDistanceVec(p_j', p_i) skipped within a molecule; Coulomb on p_j' - p_i for
//   0.01 < d < rc with G = erfc(sqrt(a) d)/d^2 + 2 sqrt(a) e^{-a d^2}/(sqrt(pi) d); pairs with
//   q_i q_j = 0 skip the Coulomb term.  Under list reuse (MI == kMiAll, list built at rc + skin)
//   a pair also has to pass the list predicate at rc (rc^2 - d^2 > 1e-4 && d^2 > 1e-4), as the
//   reference's per-call list would.
// Per-type LJ coefficients are staged in shared memory.  The loop is software-pipelined: the
// list entry two iterations ahead and the neighbour position one iteration ahead are in flight
// while the current pair is evaluated.  Accumulation: groups of four pair forces are summed in
// FP32 and folded into a two-float (TwoSum) per-atom accumulator.
template <class R, bool COUL, int MI>
__global__ void __launch_bounds__(256) k_near_force(
    NearParams prm, const LJTable* __restrict__ ljt, const typename Traits<R>::V4* __restrict__ pos4,
    const int2* __restrict__ meta, const int* __restrict__ nbr, const int* __restrict__ count,
    const RepDev* __restrict__ reps, const int* __restrict__ rep_of_slot,
    const int* __restrict__ slot_atom, double* __restrict__ force,
    double* __restrict__ energy_slot, uint32_t* status) {
  using V4 = typename Traits<R>::V4;
  __shared__ R lj_a[kMaxReplicaTypes * kMaxReplicaTypes], lj_s6[kMaxReplicaTypes * kMaxReplicaTypes];
  const int nt2 = prm.ntypes * prm.ntypes;
  for (int t = threadIdx.x; t < nt2; t += blockDim.x) {
    lj_a[t] = lj24<R>(*ljt, t);
    lj_s6[t] = sig6<R>(*ljt, t);
  }
  __syncthreads();
  const bool MOLEC = prm.molecular != 0;
  constexpr bool SPW = (MI & kMiSpecial) != 0;
  const bool ENERGY = energy_slot != nullptr;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= prm.n) return;
  const RepDev& rp = reps[rep_of_slot ? rep_of_slot[i] : 0];
  const V4 pi = pos4[i];
  const bool typed = MOLEC || prm.ntypes > 1;
  const int2 mi = typed ? meta[i] : make_int2(0, 0);
  const R rc = (R)prm.rc;
  const R cut2 = rc * rc;
  const R box[3] = {Traits<R>::box(rp, 0), Traits<R>::box(rp, 1), Traits<R>::box(rp, 2)};
  const R wrap[3] = {Traits<R>::wrap(rp, 0), Traits<R>::wrap(rp, 1), Traits<R>::wrap(rp, 2)};
  const R sa = (R)prm.sqrt_alpha, aa = (R)prm.alpha, c2 = (R)prm.two_sqrt_alpha_over_sqrt_pi;
  const R cs = (R)prm.coul_scale;
  const R qi = pi.w;
  const int trow = prm.ntypes > 1 ? mi.x * prm.ntypes : 0;   // one LJ type when all types agree
  const int* col = nbr + i;
  const size_t st = (size_t)prm.stride;
  Acc<R> fx, fy, fz;
  R gx = 0, gy = 0, gz = 0;   // FP32 group sum folded into the accumulators every 4 pairs
  R e_lj = 0, e_coul = 0;
  const int cnt = min(count[i], prm.cap);   // an overflowed row is redone after regrowth
  // pipeline prologue
  int e_cur = cnt > 0 ? __ldg(col) : 0;
  int e_nxt = cnt > 1 ? __ldg(col + st) : 0;
  V4 pj_cur = pos4[cnt > 0 ? (e_cur >> kShiftBits) : i];
  for (int p = 0; p < cnt; ++p) {
    const int e = e_cur;
    const V4 pj = pj_cur;
    // issue the loads of the next iterations before the arithmetic of this one
    e_cur = e_nxt;
    if (p + 1 < cnt) pj_cur = pos4[e_cur >> kShiftBits];
    if (p + 2 < cnt) e_nxt = __ldg(col + (size_t)(p + 2) * st);
    R px = pj.x, py = pj.y, pz = pj.z;
    if (e & 63) {   // periodic image: p_j - offset (PeriodicCoordOffset)
      const int c0 = e & 3, c1 = (e >> 2) & 3, c2b = (e >> 4) & 3;
      px = px - (c0 == 1 ? wrap[0] : (c0 == 2 ? -wrap[0] : (R)0));
      py = py - (c1 == 1 ? wrap[1] : (c1 == 2 ? -wrap[1] : (R)0));
      pz = pz - (c2b == 1 ? wrap[2] : (c2b == 2 ? -wrap[2] : (R)0));
    }
    const R r0 = px - pi.x, r1 = py - pi.y, r2 = pz - pi.z;
    const R d2 = r0 * r0 + r1 * r1 + r2 * r2;
    if ((MI & 3) == kMiAll && !((prm.orig ? cut2 - d2 > (R)0 : cut2 - d2 > (R)1.0e-4) && d2 > (R)1.0e-4)) continue;
    R f = 0;
    if (COUL) {
      const R qq = qi * pj.w;
      if (qq != (R)0) {
        const R inv = rsqrt_r(d2);
        const R dis = d2 * inv;
        if (dis < rc && dis > (R)0.01) {
          const R ex = exp_r(-aa * d2);
          const R erfcv = erfc_shared(sa * dis, ex);
          const R g = (erfcv * inv + c2 * ex) * inv;
          f = -qq * g * inv * cs;
          if (ENERGY) e_coul += qq * erfcv * inv * cs;
        }
      }
    }
    R fl0 = 0, fl1 = 0, fl2 = 0;
    bool same = false;
    int tj = 0;
    R wsp = (R)1;   // special-bond LJ weight (molecular == 2: meta.y is the bond-graph component)
    if (typed) {
      const int2 mj = meta[e >> kShiftBits];
      same = MOLEC && (mj.y == mi.y);
      tj = prm.ntypes > 1 ? mj.x : 0;
      if (SPW && same) {
        wsp = special_weight<R>(prm.sp, slot_atom[i], slot_atom[e >> kShiftBits]);
        same = false;
      }
    }
    if (!same) {
      R q0 = r0, q1 = r1, q2 = r2;   // MinDistanceVec(p_j', p_i)
      R dl2 = d2;
      if ((MI & 3) == kMiLJ) {
        min_image(q0, q1, q2, box);
        dl2 = q0 * q0 + q1 * q1 + q2 * q2;
      }
      if (dl2 < cut2 && dl2 > (R)0.0001) {
        const R inv2 = rcp_r(dl2);
        const R sd6 = lj_s6[trow + tj] * inv2 * inv2 * inv2;
        const R a24 = lj_a[trow + tj];
        R scal = a24 * (((R)2 * sd6 - (R)1) * sd6) * inv2;
        if (SPW) scal *= wsp;
        fl0 = scal * q0; fl1 = scal * q1; fl2 = scal * q2;
        // 4 eps (s6 - 1) s6 with 4 eps = -lj24/6
        if (ENERGY) e_lj += (SPW ? wsp : (R)1) * (-a24 / (R)6 * (sd6 - (R)1) * sd6);
      }
    }
    gx += f * r0 + fl0;
    gy += f * r1 + fl1;
    gz += f * r2 + fl2;
    if ((p & 3) == 3) {
      fx.add(gx); fy.add(gy); fz.add(gz);
      gx = gy = gz = 0;
    }
  }
  fx.add(gx); fy.add(gy); fz.add(gz);
  const double F[3] = {fx.value(), fy.value(), fz.value()};
  if (!isfinite(F[0]) || !isfinite(F[1]) || !isfinite(F[2])) set_flag(status, kFlagNonFinite);
  const int id = slot_atom[i];
  force[3 * id] = F[0];
  force[3 * id + 1] = F[1];
  force[3 * id + 2] = F[2];
  if (ENERGY) {
    energy_slot[2 * i] = 0.5 * (double)e_lj;
    energy_slot[2 * i + 1] = 0.5 * (double)e_coul;
  }
}

// Near force, one thread per atom, for the common case of one LJ coefficient pair for every type
// pair and no molecules (the electrolyte benchmarks): the same pair set,
// predicates and pair arithmetic as k_near_force, with less work per listed pair:
//   * the LJ coefficients live in registers (no per-pair shared-memory lookups);
//   * the list is walked four entries at a time, software-pipelined by whole chunks: the entries
//     of chunk c + 2 and the neighbour positions of chunk c + 1 are in flight while chunk c is
//     evaluated; the last chunk repeats the row's last entry and masks the repeats (a variant
//     with rows padded by the atom's own slot instead held more registers and ran 15 % slower);
//   * the LJ term is evaluated branch-free and selected by the pair predicate (the predicate of
//     the list at rc under list reuse), so skin pairs cost no divergent branch;
//   * the periodic image offsets are decoded only when some lane of the warp holds an image
//     entry in the chunk (most warps hold none);
//   * the four pair forces of a chunk are summed in R and folded into the two-float accumulator.
// Pair physics as k_near_force: ComputeNearForceVerletWorklet / ComputeLJForceVerletWorklet
// (rbmd/framework/run/worklet/RunWorklet.cpp:170-303), ExecForceFunction::ComputeLJForce and
// ComputeNearEnergyForce (rbmd/framework/forceFunction/ExecForceFunction.h:74-140).
template <class R, bool COUL, int MI, bool ENERGY>
__global__ void __launch_bounds__(256) k_near_lean(
    NearParams prm, R a24, R s6, const typename Traits<R>::V4* __restrict__ pos4, const int* __restrict__ nbr,
    const int* __restrict__ count, const RepDev* __restrict__ reps, const int* __restrict__ rep_of_slot,
    const int* __restrict__ slot_atom, double* __restrict__ force, double* __restrict__ energy_slot,
    uint32_t* status) {
  static_assert((MI & 3) != kMiLJ && (MI & kMiSpecial) == 0, "k_near_lean: no per-pair minimum image, no weights");
  using V4 = typename Traits<R>::V4;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= prm.n) return;
  const RepDev& rp = reps[rep_of_slot ? rep_of_slot[i] : 0];
  const V4 pi = pos4[i];
  const R rc = (R)prm.rc;
  const R cut2 = rc * rc;
  const R w0 = Traits<R>::wrap(rp, 0), w1 = Traits<R>::wrap(rp, 1), w2 = Traits<R>::wrap(rp, 2);
  const R sa = (R)prm.sqrt_alpha, aa = (R)prm.alpha, c2 = (R)prm.two_sqrt_alpha_over_sqrt_pi;
  const R cs = (R)prm.coul_scale;
  const R qi = pi.w;
  const int cnt = min(count[i], prm.cap);
  Acc<R> fx, fy, fz;
  R e_lj = 0, e_coul = 0;
  // a chunk's entries; indices past the end repeat the last entry (valid memory), masked below
  const unsigned ust = (unsigned)prm.stride;
  auto load_chunk = [&](int p0, int (&e)[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) e[k] = __ldg(nbr + i + (size_t)min(p0 + k, cnt - 1) * (size_t)ust);
  };
  int e_cur[4] = {0, 0, 0, 0}, e_nxt[4] = {0, 0, 0, 0};
  V4 pj[4];
  if (cnt > 0) {
    load_chunk(0, e_cur);
#pragma unroll
    for (int k = 0; k < 4; ++k) pj[k] = pos4[e_cur[k] >> kShiftBits];
    if (cnt > 4) load_chunk(4, e_nxt);
  }
  for (int p = 0; p < cnt; p += 4) {
    const unsigned act = __activemask();
    const bool img = __any_sync(act, ((e_cur[0] | e_cur[1] | e_cur[2] | e_cur[3]) & 63) != 0);
    R gx = 0, gy = 0, gz = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      R px = pj[k].x, py = pj[k].y, pz = pj[k].z;
      if (img) {   // p_j - PeriodicCoordOffset
        const int e = e_cur[k];
        const int c0 = e & 3, c1 = (e >> 2) & 3, c2b = (e >> 4) & 3;
        px = px - (c0 == 1 ? w0 : (c0 == 2 ? -w0 : (R)0));
        py = py - (c1 == 1 ? w1 : (c1 == 2 ? -w1 : (R)0));
        pz = pz - (c2b == 1 ? w2 : (c2b == 2 ? -w2 : (R)0));
      }
      const R r0 = px - pi.x, r1 = py - pi.y, r2 = pz - pi.z;
      const R d2 = r0 * r0 + r1 * r1 + r2 * r2;
      bool in = (p + k < cnt) && d2 > (R)1.0e-4;
      if ((MI & 3) == kMiAll) in = in && (prm.orig ? cut2 - d2 > (R)0 : cut2 - d2 > (R)1.0e-4);
      else in = in && d2 < cut2;
      const R inv2 = rcp_r(d2);
      const R sd6 = s6 * inv2 * inv2 * inv2;
      const R scal = in ? a24 * (((R)2 * sd6 - (R)1) * sd6) * inv2 : (R)0;
      // 4 eps (s6 - 1) s6 with 4 eps = -lj24/6
      if (ENERGY && in) e_lj += -a24 / (R)6 * (sd6 - (R)1) * sd6;
      R f = 0;
      if (COUL) {
        const R qq = qi * pj[k].w;
        if (in && qq != (R)0) {
          const R inv = rsqrt_r(d2);
          const R dis = d2 * inv;
          if (dis < rc && dis > (R)0.01) {
            const R ex = exp_r(-aa * d2);
            const R erfcv = erfc_shared(sa * dis, ex);
            const R g = (erfcv * inv + c2 * ex) * inv;
            f = -qq * g * inv * cs;
            if (ENERGY) e_coul += qq * erfcv * inv * cs;
          }
        }
      }
      const R t = scal + f;
      gx += t * r0;
      gy += t * r1;
      gz += t * r2;
    }
    fx.add(gx); fy.add(gy); fz.add(gz);
    // advance the pipeline: positions of the next chunk, entries of the one after
#pragma unroll
    for (int k = 0; k < 4; ++k) e_cur[k] = e_nxt[k];
    if (p + 4 < cnt) {
#pragma unroll
      for (int k = 0; k < 4; ++k) pj[k] = pos4[e_cur[k] >> kShiftBits];
      if (p + 8 < cnt) load_chunk(p + 8, e_nxt);
    }
  }
  const double F[3] = {fx.value(), fy.value(), fz.value()};
  if (!isfinite(F[0]) || !isfinite(F[1]) || !isfinite(F[2])) set_flag(status, kFlagNonFinite);
  const int id = slot_atom[i];
  force[3 * id] = F[0];
  force[3 * id + 1] = F[1];
  force[3 * id + 2] = F[2];
  if (ENERGY) {
    energy_slot[2 * i] = 0.5 * (double)e_lj;
    energy_slot[2 * i + 1] = 0.5 * (double)e_coul;
  }
}

// Near force with G lanes per atom (G = 4 .. 32) for systems with few atoms and long lists
// (water at 10 A: ~550 neighbours, 30,000 atoms), where one thread per atom leaves most of the
// GPU idle.  Lane s of an atom's group takes list entries s, s + G, ...; the pair terms are
// those of k_near_force (same predicates and arithmetic); each lane accumulates in a two-float
// accumulator and the group combines its G partial sums in FP64 with a fixed butterfly, so the
// result does not depend on scheduling.
template <class R, bool COUL, int MI, int G>
__global__ void __launch_bounds__(256) k_near_force_group(
    NearParams prm, const LJTable* __restrict__ ljt, const typename Traits<R>::V4* __restrict__ pos4,
    const int2* __restrict__ meta, const int* __restrict__ nbr, const int* __restrict__ count,
    const RepDev* __restrict__ reps, const int* __restrict__ rep_of_slot,
    const int* __restrict__ slot_atom, double* __restrict__ force,
    double* __restrict__ energy_slot, uint32_t* status) {
  using V4 = typename Traits<R>::V4;
  __shared__ R lj_a[kMaxReplicaTypes * kMaxReplicaTypes], lj_s6[kMaxReplicaTypes * kMaxReplicaTypes];
  const int nt2 = prm.ntypes * prm.ntypes;
  for (int t = threadIdx.x; t < nt2; t += blockDim.x) {
    lj_a[t] = lj24<R>(*ljt, t);
    lj_s6[t] = sig6<R>(*ljt, t);
  }
  __syncthreads();
  const bool MOLEC = prm.molecular != 0;
  constexpr bool SPW = (MI & kMiSpecial) != 0;
  const bool ENERGY = energy_slot != nullptr;
  const int gid = (int)((blockIdx.x * blockDim.x + threadIdx.x) / G);
  const int sub = threadIdx.x % G;
  const bool active = gid < prm.n;   // inactive groups still join the shuffles below
  const int i = active ? gid : prm.n - 1;
  const RepDev& rp = reps[rep_of_slot ? rep_of_slot[i] : 0];
  const V4 pi = pos4[i];
  const bool typed = MOLEC || prm.ntypes > 1;
  const int2 mi = typed ? meta[i] : make_int2(0, 0);
  const R rc = (R)prm.rc;
  const R cut2 = rc * rc;
  const R box[3] = {Traits<R>::box(rp, 0), Traits<R>::box(rp, 1), Traits<R>::box(rp, 2)};
  const R wrap[3] = {Traits<R>::wrap(rp, 0), Traits<R>::wrap(rp, 1), Traits<R>::wrap(rp, 2)};
  const R sa = (R)prm.sqrt_alpha, aa = (R)prm.alpha, c2 = (R)prm.two_sqrt_alpha_over_sqrt_pi;
  const R cs = (R)prm.coul_scale;
  const R qi = pi.w;
  const int trow = prm.ntypes > 1 ? mi.x * prm.ntypes : 0;
  const size_t st = (size_t)prm.stride;
  Acc<R> fx, fy, fz;
  R gx = 0, gy = 0, gz = 0;
  R e_lj = 0, e_coul = 0;
  const int cnt = active ? min(count[i], prm.cap) : 0;
  int k = 0;
  for (int p = sub; p < cnt; p += G, ++k) {
    const int e = __ldg(nbr + (size_t)p * st + i);
    const V4 pj = pos4[e >> kShiftBits];
    R px = pj.x, py = pj.y, pz = pj.z;
    if (e & 63) {
      const int c0 = e & 3, c1 = (e >> 2) & 3, c2b = (e >> 4) & 3;
      px = px - (c0 == 1 ? wrap[0] : (c0 == 2 ? -wrap[0] : (R)0));
      py = py - (c1 == 1 ? wrap[1] : (c1 == 2 ? -wrap[1] : (R)0));
      pz = pz - (c2b == 1 ? wrap[2] : (c2b == 2 ? -wrap[2] : (R)0));
    }
    const R r0 = px - pi.x, r1 = py - pi.y, r2 = pz - pi.z;
    const R d2 = r0 * r0 + r1 * r1 + r2 * r2;
    if ((MI & 3) == kMiAll && !((prm.orig ? cut2 - d2 > (R)0 : cut2 - d2 > (R)1.0e-4) && d2 > (R)1.0e-4)) continue;
    R f = 0;
    if (COUL) {
      const R qq = qi * pj.w;
      if (qq != (R)0) {
        const R inv = rsqrt_r(d2);
        const R dis = d2 * inv;
        if (dis < rc && dis > (R)0.01) {
          const R ex = exp_r(-aa * d2);
          const R erfcv = erfc_shared(sa * dis, ex);
          const R g = (erfcv * inv + c2 * ex) * inv;
          f = -qq * g * inv * cs;
          if (ENERGY) e_coul += qq * erfcv * inv * cs;
        }
      }
    }
    R fl0 = 0, fl1 = 0, fl2 = 0;
    bool same = false;
    int tj = 0;
    R wsp = (R)1;   // special-bond LJ weight (molecular == 2: meta.y is the bond-graph component)
    if (typed) {
      const int2 mj = meta[e >> kShiftBits];
      same = MOLEC && (mj.y == mi.y);
      tj = prm.ntypes > 1 ? mj.x : 0;
      if (SPW && same) {
        wsp = special_weight<R>(prm.sp, slot_atom[i], slot_atom[e >> kShiftBits]);
        same = false;
      }
    }
    if (!same) {
      R q0 = r0, q1 = r1, q2 = r2;
      R dl2 = d2;
      if ((MI & 3) == kMiLJ) {
        min_image(q0, q1, q2, box);
        dl2 = q0 * q0 + q1 * q1 + q2 * q2;
      }
      if (dl2 < cut2 && dl2 > (R)0.0001) {
        const R inv2 = rcp_r(dl2);
        const R sd6 = lj_s6[trow + tj] * inv2 * inv2 * inv2;
        const R a24 = lj_a[trow + tj];
        R scal = a24 * (((R)2 * sd6 - (R)1) * sd6) * inv2;
        if (SPW) scal *= wsp;
        fl0 = scal * q0; fl1 = scal * q1; fl2 = scal * q2;
        if (ENERGY) e_lj += (SPW ? wsp : (R)1) * (-a24 / (R)6 * (sd6 - (R)1) * sd6);
      }
    }
    gx += f * r0 + fl0;
    gy += f * r1 + fl1;
    gz += f * r2 + fl2;
    if ((k & 3) == 3) {
      fx.add(gx); fy.add(gy); fz.add(gz);
      gx = gy = gz = 0;
    }
  }
  fx.add(gx); fy.add(gy); fz.add(gz);
  double F[3] = {fx.value(), fy.value(), fz.value()};
  double el = (double)e_lj, ec = (double)e_coul;
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    F[0] += __shfl_xor_sync(0xffffffffu, F[0], o);
    F[1] += __shfl_xor_sync(0xffffffffu, F[1], o);
    F[2] += __shfl_xor_sync(0xffffffffu, F[2], o);
    el += __shfl_xor_sync(0xffffffffu, el, o);
    ec += __shfl_xor_sync(0xffffffffu, ec, o);
  }
  if (!active || sub != 0) return;
  if (!isfinite(F[0]) || !isfinite(F[1]) || !isfinite(F[2])) set_flag(status, kFlagNonFinite);
  const int id = slot_atom[i];
  force[3 * id] = F[0];
  force[3 * id + 1] = F[1];
  force[3 * id + 2] = F[2];
  if (ENERGY) {
    energy_slot[2 * i] = 0.5 * el;
    energy_slot[2 * i + 1] = 0.5 * ec;
  }
}

// RBE k-space force, one thread per charged atom (compact index c, caller id qidx[c]):
// F_i = q_i sum_l w_l k_l (cos(k_l.r_i) Im rho_l - sin(k_l.r_i) Re rho_l)
// (ComputeNewRBEForceWorklet, RunWorklet.cpp:1508-1548; S/P and qqr2e are folded into the
// records).  The block stages the k records of the replicas its atoms belong to in shared
// memory (two 16-byte broadcast loads per sample) when they fit.  Runs on the k-space stream
// concurrently with the near pass and writes far_force[c]; k_add_far folds it into the force.
template <class R>
__global__ void __launch_bounds__(128) k_rbe_force(int nq, int kstage, const int* __restrict__ qidx,
                                                   const typename FracT<R>::T* __restrict__ frac,
                                                   const typename KRec<R>::T* __restrict__ krec,
                                                   const RepDev* __restrict__ reps,
                                                   const int* __restrict__ rep_of,
                                                   double* __restrict__ far_force) {
  extern __shared__ __align__(16) unsigned char ksm_raw[];
  typename KRec<R>::T* ksm = reinterpret_cast<typename KRec<R>::T*>(ksm_raw);
  const int c0 = blockIdx.x * blockDim.x;
  const int c = c0 + threadIdx.x;
  const int last = min(nq, c0 + (int)blockDim.x) - 1;
  const int ra = rep_of ? rep_of[qidx[c0]] : 0;
  const int rb = rep_of ? rep_of[qidx[last]] : 0;
  const int kfirst = reps[ra].k_begin;
  const int kcount = reps[rb].k_begin + reps[rb].P - kfirst;
  const bool staged = kcount <= kstage;
  if (staged) {
    const int nwords = kcount * (int)(sizeof(typename KRec<R>::T) / 16);
    const int4* src = reinterpret_cast<const int4*>(krec + kfirst);
    int4* dst = reinterpret_cast<int4*>(ksm);
    for (int t = threadIdx.x; t < nwords; t += blockDim.x) dst[t] = src[t];
  }
  __syncthreads();
  if (c >= nq) return;
  const RepDev& rp = reps[rep_of ? rep_of[qidx[c]] : 0];
  const typename FracT<R>::T fr = frac[c];
  R ax = 0, ay = 0, az = 0;
  if (staged) rbe_terms<R>(fr, ksm + (rp.k_begin - kfirst), rp.P, ax, ay, az);
  else rbe_terms<R>(fr, krec + rp.k_begin, rp.P, ax, ay, az);
  const double q = (double)fr.q;
  far_force[3 * c] = q * (double)ax;
  far_force[3 * c + 1] = q * (double)ay;
  far_force[3 * c + 2] = q * (double)az;
}

__global__ void k_add_far(int nq, const int* __restrict__ qidx, const double* __restrict__ far_force,
                          double* __restrict__ force, uint32_t* status) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * nq) return;
  const int c = t / 3, d = t - 3 * c;
  const int id = qidx[c];
  const double v = force[3 * id + d] + far_force[t];
  if (!isfinite(v)) set_flag(status, kFlagNonFinite);
  force[3 * id + d] = v;
}

// ------------------------------------------------------------------------------------------
// RBE structure factors, one k per lane.  Work item = (replica, atom chunk, k tile of
// 32*KL*warps samples).  Lane l of warp w owns samples w*32*KL + l + 32*j (j < KL): its m
// vector and (Re, Im) accumulators live in registers.  The block stages the chunk's atoms
// (fixed-point fractional coordinates + charge) in shared memory, 256 at a time, and every lane
// reads each staged atom by a broadcast load, so one 16-byte load serves 32*KL (atom, k) pairs.
// Each (item, k) partial is owned by one lane: no cross-lane reduction.  There is no N x P
// buffer (the reference materialises rho_Re/Im[P*N] and reduces by key, ExecutionMD.cpp:412-448).
// ------------------------------------------------------------------------------------------
struct RhoItem { int atom_begin, atom_end, k_first, k_count; };
constexpr int kRhoStage = 256;

template <class R, int KL>
__global__ void __launch_bounds__(256) k_rho_lanes(const RhoItem* __restrict__ items,
                                                   const typename FracT<R>::T* __restrict__ frac,
                                                   const typename KRec<R>::T* __restrict__ krec,
                                                   R* __restrict__ partial, int ktile) {
  using FT = typename FracT<R>::T;
  __shared__ FT stage[kRhoStage];
  const RhoItem it = items[blockIdx.x];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  using MT = typename std::conditional<sizeof(R) == 4, uint32_t, unsigned long long>::type;
  MT mx[KL], my[KL], mz[KL];
  R re[KL], im[KL];
  int kk[KL];
  bool any = false;
#pragma unroll
  for (int j = 0; j < KL; ++j) {
    kk[j] = w * 32 * KL + j * 32 + lane;
    const bool ok = kk[j] < it.k_count;
    any |= ok;
    const typename KRec<R>::T k = ok ? krec[it.k_first + kk[j]] : typename KRec<R>::T{};
    mx[j] = (MT)(long long)k.mx;
    my[j] = (MT)(long long)k.my;
    mz[j] = (MT)(long long)k.mz;
    re[j] = 0;
    im[j] = 0;
  }
  const bool warp_any = __any_sync(0xffffffffu, any);
  for (int base = it.atom_begin; base < it.atom_end; base += kRhoStage) {
    const int cnt = min(kRhoStage, it.atom_end - base);
    __syncthreads();
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) stage[t] = frac[base + t];
    __syncthreads();
    if (!warp_any) continue;
#pragma unroll 4
    for (int a = 0; a < cnt; ++a) {
      const FT f = stage[a];
#pragma unroll
      for (int j = 0; j < KL; ++j) {
        const MT ph = mx[j] * (MT)f.x + my[j] * (MT)f.y + mz[j] * (MT)f.z;
        R s, c;
        turn_sincos(ph, s, c);
        re[j] = fma((R)f.q, c, re[j]);
        im[j] = fma((R)f.q, s, im[j]);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < KL; ++j)
    if (kk[j] < it.k_count) {
      partial[((size_t)blockIdx.x * ktile + kk[j]) * 2] = re[j];
      partial[((size_t)blockIdx.x * ktile + kk[j]) * 2 + 1] = im[j];
    }
}

// Per-replica reduction layout: items are ordered (replica, chunk, tile); replica r's partials
// for tile t and chunk c sit at item_base_r + c * ntiles_r + t.
struct RhoRep { int item_base, ntiles, nchunks, pad; };

// One warp per k sample: lanes sum the chunk partials in a fixed strided order (FP64) and a
// butterfly combines them (deterministic); then undo the half-turn phase convention
// (rho = -sum) and fill the force coefficients of the k record.
// k-space energy estimate per replica: (S/P) qqr2e sum_l w_l (2 pi / V) |rho_l|^2 / k_l^2.
template <class R>
__global__ void k_rho_finish(int nk_total, int ktile, const int* __restrict__ krep,
                             const RhoRep* __restrict__ rr, const RepDev* __restrict__ reps,
                             const R* __restrict__ partial, const double* __restrict__ weights,
                             double qqr2e, typename KRec<R>::T* __restrict__ krec,
                             double2* __restrict__ rho_out, double* __restrict__ ek_out) {
  const int g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (g >= nk_total) return;
  const int r = krep[g];
  const RepDev& rp = reps[r];
  const RhoRep q = rr[r];
  const int l = g - rp.k_begin;
  const int tile = l / ktile, kk = l % ktile;
  double re = 0, im = 0;
  for (int c = lane; c < q.nchunks; c += 32) {
    const size_t item = (size_t)q.item_base + (size_t)c * q.ntiles + tile;
    re += (double)partial[(item * ktile + kk) * 2];
    im += (double)partial[(item * ktile + kk) * 2 + 1];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  if (lane != 0) return;
  typename KRec<R>::T k = krec[g];
  re = -re;
  im = -im;
  const double twopi = 6.283185307179586476925;
  const double kx = twopi * k.mx / rp.box_d[0], ky = twopi * k.my / rp.box_d[1],
               kz = twopi * k.mz / rp.box_d[2];
  const double k2 = kx * kx + ky * ky + kz * kz;
  const double wgt = weights ? weights[g] : 1.0;
  // F_i = q_i (S/P) qqr2e sum_l wgt (-4 pi /(V k^2)) k (cos Im - sin Re); the kernel evaluates
  // the angle shifted by half a turn, which flips cos and sin: store -w.
  const double w = -(rp.S / rp.P) * qqr2e * wgt * (-4.0 * 3.14159265358979323846 / (rp.volume * k2));
  k.wx = (decltype(k.wx))(w * kx);
  k.wy = (decltype(k.wy))(w * ky);
  k.wz = (decltype(k.wz))(w * kz);
  k.re = (decltype(k.re))re;
  k.im = (decltype(k.im))im;
  krec[g] = k;
  if (rho_out) rho_out[g] = make_double2(re, im);
  if (ek_out)
    ek_out[g] = (rp.S / rp.P) * qqr2e * wgt * (2.0 * 3.14159265358979323846 / rp.volume) *
                (re * re + im * im) / k2;
}

// ------------------------------------------------------------------------------------------
// RBE k-sampler: RBEPSAMPLE::Fetch_P_Sample + MH_Algorithm (rbmd/framework/model/
// RBEPSample.h:63-173) with mu = 0, sigma_d = sqrt(alpha/2) L_d / pi.  The MH ratio
// (P(m')/P(m)) (q(m)/q(m')) is G(m')/G(m) with G = exp(-pi^2 m^2/(alpha L^2)) / q(m) tabulated
// on the host (FP64); u <= min(1, ratio) is evaluated as u * G(m) <= G(m').
// One block per replica: phase 1 draws the Gaussian proposals, their G values and the
// acceptance uniforms of the first D steps in parallel (they do not depend on the chain);
// phase 2 resolves every per-axis chain state of those D steps in parallel (a step with
// u gmax <= G(m) accepts whatever the state, and the states between two such steps are replayed
// exactly), then assigns sample indices to the states that are not all zero (the all-zero retry
// of the reference couples the axes only there) with a block scan.  Steps past D, and windows
// holding a proposal beyond the tables, run the chain sequentially on one thread as the
// reference does.  Same k-sets as the sequential chain, bit for bit.
// ------------------------------------------------------------------------------------------
struct SamplerRep {
  double sigma[3];
  double gmax[3];   // largest finite G of each axis' table
  int qmax;
  int g_offset;     // offset of this replica's G tables (3 * (qmax+1) doubles)
};

__device__ __forceinline__ double sampler_draw(uint32_t k0, uint32_t k1, long long step, int rep,
                                               int axis, long long draw, double* ua) {
  uint32_t c[4] = {(uint32_t)draw, (uint32_t)axis | ((uint32_t)rep << 2), (uint32_t)(unsigned long long)step,
                   (uint32_t)((unsigned long long)step >> 32)};
  philox4x32(c, k0, k1);
  double U1 = ((double)c[0] + 0.5) * (1.0 / 4294967296.0);
  if (U1 < 1e-6) U1 = ((double)c[3] + 0.5) * (1.0 / 4294967296.0);
  if (U1 < 1e-6) U1 = 1e-6;
  const double U2 = ((double)c[1] + 0.5) * (1.0 / 4294967296.0);
  *ua = ((double)c[2] + 0.5) * (1.0 / 4294967296.0);
  return sqrt(-2.0 * log(U1)) * cos(2.0 * 3.14159265358979323846 * U2);
}

__device__ __forceinline__ double sampler_g(const double* g, int qmax, int axis, int m) {
  m = abs(m);
  return m <= qmax ? g[axis * (qmax + 1) + m] : __longlong_as_double(0x7ff0000000000000ll);
}

template <int D>
__global__ void __launch_bounds__(256) k_sample(int nrep, const SamplerRep* __restrict__ srep,
                                                const double* __restrict__ gtab,
                                                const RepDev* __restrict__ reps, unsigned long long seed,
                                                long long step_arg, const long long* __restrict__ step_dev,
                                                int* __restrict__ kvec_out,
                                                void* __restrict__ krec, int rec_bytes,
                                                int* __restrict__ krep, uint32_t* status) {
  const int r = blockIdx.x;
  if (r >= nrep) return;
  const long long step = step_dev ? *step_dev : step_arg;   // device counter under graph replay
  const SamplerRep s = srep[r];
  const int P = reps[r].P, kb = reps[r].k_begin;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  const double* g = gtab + s.g_offset;
  __shared__ int mw[3][D];
  __shared__ double ua[3][D];
  __shared__ double gw[3][D];
  for (int t = threadIdx.x; t < 3 * D; t += blockDim.x) {
    const int axis = t / D, d = t % D;
    double u;
    const double gs = sampler_draw(k0, k1, step, r, axis, d, &u);
    const int m = (int)round(s.sigma[axis] * gs);
    mw[axis][d] = m;
    ua[axis][d] = u;
    gw[axis][d] = sampler_g(g, s.qmax, axis, m);
  }
  __syncthreads();
  auto prop = [&](int axis, long long d, double* u, double* gm) -> int {
    if (d < D) { *u = ua[axis][d]; *gm = gw[axis][d]; return mw[axis][d]; }
    const double gs = sampler_draw(k0, k1, step, r, axis, d, u);
    const int m = (int)round(s.sigma[axis] * gs);
    *gm = sampler_g(g, s.qmax, axis, m);
    return m;
  };
  auto emit = [&](int i, const int* X) {
    int* o = kvec_out + 3 * (kb + i);
    o[0] = X[0]; o[1] = X[1]; o[2] = X[2];
    int* rec = reinterpret_cast<int*>(reinterpret_cast<char*>(krec) + (size_t)(kb + i) * rec_bytes);
    rec[0] = X[0]; rec[1] = X[1]; rec[2] = X[2];
    krep[kb + i] = r;
  };
  // first sample: the first draw that is not all zero (the reference's Fetch_P_Sample do-while)
  __shared__ int s_d0, s_x0[3], s_seq, s_total;
  __shared__ double s_g0[3];
  if (threadIdx.x == 0) {
    long long draw = 0;
    int X0[3];
    double G0[3];
    for (int guard = 0;; ++guard) {
      double u;
      for (int a = 0; a < 3; ++a) X0[a] = prop(a, draw, &u, &G0[a]);
      ++draw;
      if (!(X0[0] == 0 && X0[1] == 0 && X0[2] == 0)) break;
      if (guard > 100000) { set_flag(status, kFlagSampler); X0[0] = 1; G0[0] = sampler_g(g, s.qmax, 0, 1); break; }
    }
    emit(0, X0);
    s_d0 = (int)min(draw, (long long)D);
    for (int a = 0; a < 3; ++a) { s_x0[a] = X0[a]; s_g0[a] = G0[a]; }
    // the parallel chain below needs a non-empty window and every state in it with a finite G
    s_seq = draw >= D || !(isfinite(G0[0]) && isfinite(G0[1]) && isfinite(G0[2]));
    s_total = 1;
  }
  __syncthreads();
  const int d0 = s_d0;
  // The Metropolis-Hastings chain of each axis (MH_Algorithm, RBEPSample.h:63-85) is an
  // independence sampler: proposals do not depend on the state, and a step accepts when
  // u G(X_prev) <= G(m).  A step with u gmax <= G(m) accepts whatever the state (rounding is
  // monotonic, and every state of the window has G <= gmax), so each state is resolved in
  // parallel from the nearest such step before it, replaying the few steps in between exactly as
  // the sequential chain would.  Draws whose G is infinite (proposals past the table) fall back
  // to the sequential chain.
  int bad = 0;
  for (int t = threadIdx.x; t < 3 * (D - d0); t += blockDim.x) bad |= !isfinite(gw[t / (D - d0)][d0 + t % (D - d0)]);
  if (__syncthreads_or(bad) || s_seq) {
    if (threadIdx.x != 0) return;
    // sequential chain from the first sample (the reference's loop, Fetch_P_Sample:155-172)
    int X0[3] = {s_x0[0], s_x0[1], s_x0[2]};
    double G0[3] = {s_g0[0], s_g0[1], s_g0[2]};
    long long draw = d0;
    int i = 1;
    long long guard = 0;
    while (i < P) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        double u, gm;
        const int m_w = prop(a, draw, &u, &gm);
        if (u * G0[a] <= gm) { X0[a] = m_w; G0[a] = gm; }
      }
      ++draw;
      if (++guard > 64LL * P + 100000) { set_flag(status, kFlagSampler); break; }
      if (X0[0] == 0 && X0[1] == 0 && X0[2] == 0) continue;
      emit(i, X0);
      ++i;
    }
    return;
  }
  __shared__ int chain[3][D];
  for (int t = threadIdx.x; t < 3 * (D - d0); t += blockDim.x) {
    const int a = t / (D - d0), d = d0 + t % (D - d0);
    int sidx = d;
    while (sidx >= d0 && !(ua[a][sidx] * s.gmax[a] <= gw[a][sidx])) --sidx;
    int X;
    double G;
    if (sidx < d0) { X = s_x0[a]; G = s_g0[a]; sidx = d0 - 1; }
    else { X = mw[a][sidx]; G = gw[a][sidx]; }
    for (int k = sidx + 1; k <= d; ++k)
      if (ua[a][k] * G <= gw[a][k]) { X = mw[a][k]; G = gw[a][k]; }
    chain[a][d] = X;
  }
  __syncthreads();
  // emission: samples 1, 2, ... are the states of the draws that are not all zero, in draw order
  constexpr int kPer = (D + 255) / 256;
  const int base = d0 + threadIdx.x * kPer;
  int cnt = 0;
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int d = base + j;
    if (d < D && !(chain[0][d] == 0 && chain[1][d] == 0 && chain[2][d] == 0)) ++cnt;
  }
  // block exclusive scan of cnt (blockDim.x == 256)
  __shared__ int wsum[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  int off = 0;
  for (int w = 0; w < wid; ++w) off += wsum[w];
  int i = 1 + off + incl - cnt;
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int d = base + j;
    if (d < D && !(chain[0][d] == 0 && chain[1][d] == 0 && chain[2][d] == 0)) {
      if (i < P) {
        const int X[3] = {chain[0][d], chain[1][d], chain[2][d]};
        emit(i, X);
      }
      ++i;
    }
  }
  if (threadIdx.x == 255) s_total = i;   // 1 + every non-zero state of the window
  __syncthreads();
  if (threadIdx.x != 0 || s_total >= P) return;
  // more samples than the window holds: continue the chain sequentially from its last state
  int X0[3] = {chain[0][D - 1], chain[1][D - 1], chain[2][D - 1]};
  double G0[3];
  for (int a = 0; a < 3; ++a) G0[a] = sampler_g(g, s.qmax, a, X0[a]);
  long long draw = D;
  int k = s_total;
  long long guard = D - d0;
  while (k < P) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double u, gm;
      const int m_w = prop(a, draw, &u, &gm);
      if (u * G0[a] <= gm) { X0[a] = m_w; G0[a] = gm; }
    }
    ++draw;
    if (++guard > 64LL * P + 100000) { set_flag(status, kFlagSampler); break; }
    if (X0[0] == 0 && X0[1] == 0 && X0[2] == 0) continue;
    emit(k, X0);
    ++k;
  }
}

// ------------------------------------------------------------------------------------------
// EAM passes (funcfl, 7-coefficient splines): pass 1 = ComputeEAMfpVerletWorklet
// (RunWorklet.cpp:305-359) -> fp[slot]; pass 2 = ComputeEAMForceVerletWorklet (:361-417).
// Spline rows are stored as two float4 (c0..c3, c4..c6,0).  MI: MinDistanceVec on the pair
// vector, needed only when a replica has fewer than 3 cells on an axis (otherwise the stored
// image shift already gives the nearest image, also under list reuse: the slot cache is
// unwrapped since the build).  FP32 uses r = rsq * rsqrt(rsq) and 1/r = rsqrt(rsq).
// ------------------------------------------------------------------------------------------
struct EamDev {
  const float4* frho;   // 2 float4 per row
  const float4* rhor;
  const float4* z2r;
  int nrho, nr;
  float rdr, rdrho;
  double rdr_d, rdrho_d;
  float rhomax;
};

template <class R, bool MI>
__global__ void __launch_bounds__(128) k_eam_fp(int n, int stride, int cap, double rc, EamDev eam,
                                                const typename Traits<R>::V4* __restrict__ pos4,
                                                const int* __restrict__ nbr, const int* __restrict__ count,
                                                const RepDev* __restrict__ reps,
                                                const int* __restrict__ rep_of_slot, R* __restrict__ fp,
                                                double* __restrict__ embed_slot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RepDev& rp = reps[rep_of_slot ? rep_of_slot[i] : 0];
  const typename Traits<R>::V4 pi = pos4[i];
  const R wrap[3] = {Traits<R>::wrap(rp, 0), Traits<R>::wrap(rp, 1), Traits<R>::wrap(rp, 2)};
  const R box[3] = {Traits<R>::box(rp, 0), Traits<R>::box(rp, 1), Traits<R>::box(rp, 2)};
  const R ibox[3] = {(R)1 / box[0], (R)1 / box[1], (R)1 / box[2]};
  const R cut2 = (R)rc * (R)rc;
  const R rdr = sizeof(R) == 4 ? (R)eam.rdr : (R)eam.rdr_d;
  Acc<R> rho;
  const int cnt = min(count[i], cap);
  for (int p = 0; p < cnt; ++p) {
    const int e = __ldg(nbr + (size_t)p * stride + i);
    const int j = e >> kShiftBits;
    const typename Traits<R>::V4 pj = pos4[j];
    R r[3];
    const R pjv[3] = {pj.x, pj.y, pj.z}, piv[3] = {pi.x, pi.y, pi.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int cd = (e >> (2 * d)) & 3;
      const R off = cd == 1 ? wrap[d] : (cd == 2 ? -wrap[d] : (R)0);
      R v = piv[d] - (pjv[d] - off);
      if (MI) v -= box[d] * rint(v * ibox[d]);   // MinDistanceVec
      r[d] = v;
    }
    const R rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    if (rsq < cut2 && rsq > (R)0.01) {
      R pp = rsq * rsqrt_r(rsq) * rdr + (R)1;
      int m = (int)pp;
      m = min(m, eam.nr - 1);
      pp -= (R)m;
      pp = fmin(pp, (R)1);
      const float4 b = __ldg(eam.rhor + 2 * m + 0);
      const float4 c = __ldg(eam.rhor + 2 * m + 1);
      rho.add((((R)b.w * pp + (R)c.x) * pp + (R)c.y) * pp + (R)c.z);
    }
  }
  const R rr = (R)rho.value();
  R pp = rr * (sizeof(R) == 4 ? (R)eam.rdrho : (R)eam.rdrho_d) + (R)1;
  int m = (int)pp;
  m = max(1, min(m, eam.nrho - 1));
  pp -= (R)m;
  pp = fmin(pp, (R)1);
  const float4 a = __ldg(eam.frho + 2 * m + 0);
  const float4 b = __ldg(eam.frho + 2 * m + 1);
  fp[i] = ((R)a.x * pp + (R)a.y) * pp + (R)a.z;
  if (embed_slot) {
    double phi = (((double)a.w * pp + (double)b.x) * pp + (double)b.y) * pp + (double)b.z;
    if ((double)rr > eam.rhomax) phi += (double)fp[i] * ((double)rr - eam.rhomax);
    embed_slot[i] = phi;
  }
}

template <class R, bool MI>
__global__ void __launch_bounds__(128) k_eam_force(int n, int stride, int cap, double rc, EamDev eam,
                                                   const typename Traits<R>::V4* __restrict__ pos4,
                                                   const int* __restrict__ nbr, const int* __restrict__ count,
                                                   const RepDev* __restrict__ reps,
                                                   const int* __restrict__ rep_of_slot,
                                                   const R* __restrict__ fp, const int* __restrict__ slot_atom,
                                                   double* __restrict__ force, double* __restrict__ pair_slot,
                                                   uint32_t* status, int ref_sign) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RepDev& rp = reps[rep_of_slot ? rep_of_slot[i] : 0];
  const typename Traits<R>::V4 pi = pos4[i];
  const R wrap[3] = {Traits<R>::wrap(rp, 0), Traits<R>::wrap(rp, 1), Traits<R>::wrap(rp, 2)};
  const R box[3] = {Traits<R>::box(rp, 0), Traits<R>::box(rp, 1), Traits<R>::box(rp, 2)};
  const R ibox[3] = {(R)1 / box[0], (R)1 / box[1], (R)1 / box[2]};
  const R cut2 = (R)rc * (R)rc;
  const R rdr = sizeof(R) == 4 ? (R)eam.rdr : (R)eam.rdr_d;
  const R fpi = fp[i];
  Acc<R> fx, fy, fz;
  R epair = 0;
  const int cnt = min(count[i], cap);
  for (int p = 0; p < cnt; ++p) {
    const int e = __ldg(nbr + (size_t)p * stride + i);
    const int j = e >> kShiftBits;
    const typename Traits<R>::V4 pj = pos4[j];
    R r[3];
    const R pjv[3] = {pj.x, pj.y, pj.z}, piv[3] = {pi.x, pi.y, pi.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int cd = (e >> (2 * d)) & 3;
      const R off = cd == 1 ? wrap[d] : (cd == 2 ? -wrap[d] : (R)0);
      // pair vector p_i - p_j' (the sign for which F = -grad E, as LAMMPS' pair_eam and the
      // reference's RBL pass, RunWorklet.cpp:1180); ref_sign: the reference's Verlet pass uses
      // MinDistanceVec(p_j, p_i) (RunWorklet.cpp:402), which reverses the force
      R v = ref_sign ? (pjv[d] - off) - piv[d] : piv[d] - (pjv[d] - off);
      if (MI) v -= box[d] * rint(v * ibox[d]);
      r[d] = v;
    }
    const R rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    if (rsq < cut2 && rsq > (R)0.01) {
      const R recip = rsqrt_r(rsq);
      const R rv = rsq * recip;
      R pp = rv * rdr + (R)1;
      int m = (int)pp;
      m = min(m, eam.nr - 1);
      pp -= (R)m;
      pp = fmin(pp, (R)1);
      const float4 ra = __ldg(eam.rhor + 2 * m + 0);
      const float4 za = __ldg(eam.z2r + 2 * m + 0);
      const float4 zb = __ldg(eam.z2r + 2 * m + 1);
      const R rhop = ((R)ra.x * pp + (R)ra.y) * pp + (R)ra.z;
      const R z2p = ((R)za.x * pp + (R)za.y) * pp + (R)za.z;
      const R z2 = (((R)za.w * pp + (R)zb.x) * pp + (R)zb.y) * pp + (R)zb.z;
      const R phi = z2 * recip;
      const R phip = z2p * recip - phi * recip;
      const R psip = fpi * rhop + fp[j] * rhop + phip;
      const R fpair = -psip * recip;
      fx.add(r[0] * fpair);
      fy.add(r[1] * fpair);
      fz.add(r[2] * fpair);
      epair += phi;
    }
  }
  const double F[3] = {fx.value(), fy.value(), fz.value()};
  if (!isfinite(F[0]) || !isfinite(F[1]) || !isfinite(F[2])) set_flag(status, kFlagNonFinite);
  const int id = slot_atom[i];
  force[3 * id] = F[0];
  force[3 * id + 1] = F[1];
  force[3 * id + 2] = F[2];
  if (pair_slot) pair_slot[i] = 0.5 * (double)epair;
}

}  // namespace rbmd
