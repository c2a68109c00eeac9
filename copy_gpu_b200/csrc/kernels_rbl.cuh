// kernels_rbl.cuh -- the RBL ("random batch list") near field of RBMD's default neighbor mode:
// a core list inside r_core plus every pice-th shell pair in [r_core, rc) in the reference's
// traversal order, the LJ / erfc-Coulomb and EAM passes over it with the shell terms scaled by
// pice, and the removal of the mean near force.
#pragma once

#include "common.cuh"
#include "kernels_cells.cuh"
#include "kernels_force.cuh"
#include "kernels_md.cuh"

namespace rbmd {

// Squared lower bound of the distance from coordinate x to the cells of unwrapped index u
// (wrapped index w) along axis d, less a rounding allowance `slack`; a boundary cell is open on
// its outer side, because atoms outside the box are binned into it.  A stencil cell whose bound
// summed over the axes exceeds rc^2 holds no pair (the predicate needs d^2 < rc^2 - 1e-4), so
// the list builds skip it without changing which pairs are found or their order.
template <class R>
__device__ __forceinline__ R rbl_gap2(const RepDev& rp, int d, int u, int w, R x, R slack) {
  const R dx = Traits<R>::dx(rp, d);
  const R sl = Traits<R>::lo(rp, d) + (R)u * dx, sh = sl + dx;
  R g = (R)0;
  if (w != 0 && x < sl) g = sl - x;
  else if (w != rp.dims[d] - 1 && x > sh) g = x - sh;
  g -= slack;
  return g > (R)0 ? g * g : (R)0;
}

template <class R>
__device__ __forceinline__ R rbl_slack(const RepDev& rp, int d, R x, R rc) {
  return (R)1e-5 * (fabs(x) + fabs(Traits<R>::lo(rp, d)) + (R)rp.dims[d] * Traits<R>::dx(rp, d) + rc) + (R)1e-6;
}

// RBL list of slot i: ComputeRBLNeighboursOnceWorklet (rbmd/framework/run/worklet/RunWorklet.cpp:
// 634-708).  The stencil is walked as the reference walks it (x offset outermost, z innermost,
// the points of a cell in slot order = ascending caller id), because which shell pairs are kept
// depends on that order: a candidate with rc^2 - d^2 > 1e-4 && d^2 - rs^2 > 1e-4 is a shell pair
// and is kept when its running shell index is a multiple of pice; otherwise a pair with
// rs^2 - d^2 > 1e-4 && d^2 > 1e-4 is a core pair.  d^2 is formed with uncontracted ops on
// (p_j - offset) - p_i, as in the full list.  Core entries fill rows [0, core_cap) of the
// transposed list, kept shell entries rows [core_cap, core_cap + shell_cap).
constexpr int kRblBatch = 4;   // candidate positions loaded ahead of their classification (8: slower)

template <class R>
__global__ void __launch_bounds__(128) k_rbl_list(
    int n, const typename Traits<R>::V4* __restrict__ pos4, const int* __restrict__ cell_start,
    const RepDev* __restrict__ reps, const int* __restrict__ rep_of_slot, int num_cycles, R rc, R rs,
    int core_cap, int shell_cap, int stride, int* __restrict__ nbr, int* __restrict__ ncore,
    int* __restrict__ nshell, int* __restrict__ max_count, uint32_t* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RepDev& rp = reps[rep_of_slot ? rep_of_slot[i] : 0];
  const int pice = rp.rbl_pice;
  const typename Traits<R>::V4 pi = pos4[i];
  const R pix[3] = {pi.x, pi.y, pi.z};
  int ci[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    ci[d] = (int)div_rn(sub_rn(pix[d], Traits<R>::lo(rp, d)), Traits<R>::dx(rp, d));
  const R rc2 = mul_rn(rc, rc), rs2 = mul_rn(rs, rs);
  const int nc = num_cycles;
  const int dx0 = rp.dims[0], dx1 = rp.dims[1], dx2 = rp.dims[2];
  const R sl0 = rbl_slack(rp, 0, pix[0], rc), sl1 = rbl_slack(rp, 1, pix[1], rc), sl2 = rbl_slack(rp, 2, pix[2], rc);
  int n_core = 0, n_shell = 0, shell_index = 0;
  int next_kept = 0;   // shell index of the next kept shell pair: 0, pice, 2 pice, ...
  for (int a = -nc; a <= nc; ++a) {
    const int nbx = ci[0] + a;
    const int wx = wrap_cell(nbx, dx0);
    const int ddx = wx - nbx;
    const R off0 = mul_rn(Traits<R>::dx(rp, 0), (R)ddx);
    const int cx = ddx > 0 ? 1 : (ddx < 0 ? 2 : 0);
    const R gx2 = rbl_gap2(rp, 0, nbx, wx, pix[0], sl0);
    for (int b = -nc; b <= nc; ++b) {
      const int nby = ci[1] + b;
      const int wy = wrap_cell(nby, dx1);
      const int ddy = wy - nby;
      const R off1 = mul_rn(Traits<R>::dx(rp, 1), (R)ddy);
      const int cy = ddy > 0 ? 1 : (ddy < 0 ? 2 : 0);
      const R gxy2 = gx2 + rbl_gap2(rp, 1, nby, wy, pix[1], sl1);
      if (gxy2 > rc2) continue;
      for (int c = -nc; c <= nc; ++c) {
        const int nbz = ci[2] + c;
        const int wz = wrap_cell(nbz, dx2);
        if (gxy2 + rbl_gap2(rp, 2, nbz, wz, pix[2], sl2) > rc2) continue;   // no pair in this cell
        const int ddz = wz - nbz;
        const R off2 = mul_rn(Traits<R>::dx(rp, 2), (R)ddz);
        const int code = cx | (cy << 2) | ((ddz > 0 ? 1 : (ddz < 0 ? 2 : 0)) << 4);
        const int cell = rp.cell_base + wx + wy * dx0 + wz * dx0 * dx1;
        const int s1 = cell_start[cell + 1];
        // the candidates of a cell in groups of kRblBatch: the positions are loaded before any
        // is classified (kRblBatch loads in flight), then classified in slot order
        for (int s = cell_start[cell]; s < s1; s += kRblBatch) {
          typename Traits<R>::V4 pj[kRblBatch];
#pragma unroll
          for (int u = 0; u < kRblBatch; ++u) pj[u] = pos4[s + u < s1 ? s + u : s];
#pragma unroll
          for (int u = 0; u < kRblBatch; ++u) {
            if (s + u < s1) {
              const R r0 = sub_rn(sub_rn(pj[u].x, off0), pix[0]);
              const R r1 = sub_rn(sub_rn(pj[u].y, off1), pix[1]);
              const R r2 = sub_rn(sub_rn(pj[u].z, off2), pix[2]);
              const R d2 = add_rn(add_rn(mul_rn(r0, r0), mul_rn(r1, r1)), mul_rn(r2, r2));
              const int e = ((s + u) << kShiftBits) | code;
              if (gt_small(sub_rn(rc2, d2)) && gt_small(sub_rn(d2, rs2))) {
                if (shell_index == next_kept) {   // shell_index % pice == 0
                  if (n_shell < shell_cap) nbr[(size_t)(core_cap + n_shell) * stride + i] = e;
                  ++n_shell;
                  next_kept += pice;
                }
                ++shell_index;
              } else if (gt_small(sub_rn(rs2, d2)) && gt_small(d2)) {
                if (n_core < core_cap) nbr[(size_t)n_core * stride + i] = e;
                ++n_core;
              }
            }
          }
        }
      }
    }
  }
  ncore[i] = n_core;
  nshell[i] = n_shell;
  if (n_core > core_cap || n_shell > shell_cap) {
    set_flag(status, kFlagListOverflow);
    atomicMax(max_count, n_core);
    atomicMax(max_count + 1, n_shell);
  }
}

// The same list with one warp per atom (systems of 10^4 - 10^5 atoms leave the thread-per-atom
// build with a few thousand warps of long serial loops).  The (2 num_cycles + 1)^3 stencil cells
// are laid out in the reference's walk order in shared memory (first slot, number of candidates
// before the cell, periodic wrap count per axis), which flattens the atom's candidates into one
// sequence; each round the warp's lanes take 32 consecutive candidates (cell found by binary
// search over the running counts), classify them with the same predicates and arithmetic, and a
// ballot prefix gives each shell pair its running index and each kept / core pair its row, so the
// list is identical entry for entry to k_rbl_list's.
constexpr int kRblStencilMax = 343;   // num_cycles <= 3
constexpr int kRblWarps = 4;

template <class R>
__global__ void __launch_bounds__(32 * kRblWarps) k_rbl_list_warp(
    int n, const typename Traits<R>::V4* __restrict__ pos4, const int* __restrict__ cell_start,
    const RepDev* __restrict__ reps, const int* __restrict__ rep_of_slot, int num_cycles, R rc, R rs,
    int core_cap, int shell_cap, int stride, int* __restrict__ nbr, int* __restrict__ ncore,
    int* __restrict__ nshell, int* __restrict__ max_count, uint32_t* status) {
  __shared__ int s_start[kRblWarps][kRblStencilMax];
  __shared__ int s_pre[kRblWarps][kRblStencilMax + 1];
  __shared__ int s_wrap[kRblWarps][kRblStencilMax];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kRblWarps + w;
  if (i >= n) return;   // uniform across the warp
  const unsigned full = 0xffffffffu;
  const RepDev& rp = reps[rep_of_slot ? rep_of_slot[i] : 0];
  const int pice = rp.rbl_pice;
  const typename Traits<R>::V4 pi = pos4[i];
  const R pix[3] = {pi.x, pi.y, pi.z};
  int ci[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    ci[d] = (int)div_rn(sub_rn(pix[d], Traits<R>::lo(rp, d)), Traits<R>::dx(rp, d));
  const R rc2 = mul_rn(rc, rc), rs2 = mul_rn(rs, rs);
  const int nc = num_cycles, side = 2 * num_cycles + 1, ncs = side * side * side;
  const int dims[3] = {rp.dims[0], rp.dims[1], rp.dims[2]};
  // stencil table: cell k = ((a + nc) * side + (b + nc)) * side + (c + nc), x outermost
  int carry = 0;
  for (int k0 = 0; k0 < ncs; k0 += 32) {
    const int k = k0 + lane;
    int cnt = 0;
    if (k < ncs) {
      const int off[3] = {k / (side * side) - nc, (k / side) % side - nc, k % side - nc};
      int wr[3], q = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int nb = ci[d] + off[d];
        wr[d] = wrap_cell(nb, dims[d]);
        q |= (((wr[d] - nb) / dims[d]) & 0xff) << (8 * d);   // wrap count (wx - nbx) / dims
      }
      const int cell = rp.cell_base + wr[0] + wr[1] * dims[0] + wr[2] * dims[0] * dims[1];
      const int s0 = cell_start[cell];
      R g2 = (R)0;
#pragma unroll
      for (int d = 0; d < 3; ++d)
        g2 += rbl_gap2(rp, d, ci[d] + off[d], wr[d], pix[d], rbl_slack(rp, d, pix[d], rc));
      cnt = g2 > rc2 ? 0 : cell_start[cell + 1] - s0;   // a cell beyond rc contributes no candidate
      s_start[w][k] = s0;
      s_wrap[w][k] = q;
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(full, incl, o);
      if (lane >= o) incl += t;
    }
    if (k < ncs) s_pre[w][k] = carry + incl - cnt;
    carry += __shfl_sync(full, incl, 31);
  }
  if (lane == 0) s_pre[w][ncs] = carry;
  __syncwarp();
  const int total = carry;
  const unsigned lt = (1u << lane) - 1u;
  int n_core = 0, n_shell = 0, shell_index = 0;
  for (int base = 0; base < total; base += 32) {
    const int k = base + lane;
    bool shell = false, core = false;
    int entry = 0;
    if (k < total) {
      int lo = 0, hi = ncs;   // s_pre[lo] <= k < s_pre[hi]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (s_pre[w][mid] <= k) lo = mid;
        else hi = mid;
      }
      const int sj = s_start[w][lo] + (k - s_pre[w][lo]);
      const int q = s_wrap[w][lo];
      const int dd[3] = {(int)(signed char)(q & 0xff) * dims[0], (int)(signed char)((q >> 8) & 0xff) * dims[1],
                         (int)(signed char)((q >> 16) & 0xff) * dims[2]};
      const R off0 = mul_rn(Traits<R>::dx(rp, 0), (R)dd[0]);
      const R off1 = mul_rn(Traits<R>::dx(rp, 1), (R)dd[1]);
      const R off2 = mul_rn(Traits<R>::dx(rp, 2), (R)dd[2]);
      const int code = (dd[0] > 0 ? 1 : (dd[0] < 0 ? 2 : 0)) | ((dd[1] > 0 ? 1 : (dd[1] < 0 ? 2 : 0)) << 2) |
                       ((dd[2] > 0 ? 1 : (dd[2] < 0 ? 2 : 0)) << 4);
      const typename Traits<R>::V4 pj = pos4[sj];
      const R r0 = sub_rn(sub_rn(pj.x, off0), pix[0]);
      const R r1 = sub_rn(sub_rn(pj.y, off1), pix[1]);
      const R r2 = sub_rn(sub_rn(pj.z, off2), pix[2]);
      const R d2 = add_rn(add_rn(mul_rn(r0, r0), mul_rn(r1, r1)), mul_rn(r2, r2));
      shell = gt_small(sub_rn(rc2, d2)) && gt_small(sub_rn(d2, rs2));
      core = !shell && gt_small(sub_rn(rs2, d2)) && gt_small(d2);
      entry = (sj << kShiftBits) | code;
    }
    const unsigned bsh = __ballot_sync(full, shell);
    const bool keep = shell && ((shell_index + __popc(bsh & lt)) % pice == 0);
    const unsigned bkeep = __ballot_sync(full, keep);
    const unsigned bcore = __ballot_sync(full, core);
    if (keep) {
      const int at = n_shell + __popc(bkeep & lt);
      if (at < shell_cap) nbr[(size_t)(core_cap + at) * stride + i] = entry;
    }
    if (core) {
      const int at = n_core + __popc(bcore & lt);
      if (at < core_cap) nbr[(size_t)at * stride + i] = entry;
    }
    shell_index += __popc(bsh);
    n_shell += __popc(bkeep);
    n_core += __popc(bcore);
  }
  if (lane == 0) {
    ncore[i] = n_core;
    nshell[i] = n_shell;
    if (n_core > core_cap || n_shell > shell_cap) {
      set_flag(status, kFlagListOverflow);
      atomicMax(max_count, n_core);
      atomicMax(max_count + 1, n_shell);
    }
  }
}

struct RblParams {
  int n, stride, ntypes, core_cap, molecular;
  int table_mode;   // 1: G from the reference's ERF table (alpha 0.1, one value per bucket)
  int shell_coul;   // 0: shell Coulomb dropped as the reference does; 1: x pice
  const float* erf_tab;   // 2048 entries of the reference's ERF table (table_mode 1)
  double rc, rs, alpha, qqr2e;
  double sqrt_alpha, two_sqrt_alpha_over_sqrt_pi;
  SpecialDev sp;    // molecular == 2: special-bond partner lists
};

// The reference's ERF table (rbmd/framework/staticTable/ExecStaticTable.h:37-39,96-135): the
// entry index is bits 15..25 of the float distance (3 low exponent bits and 8 mantissa bits), so
// one entry serves a whole bucket of distances; entries exist for 0.1 <= d < 12 (indices 921..2047
// below d = 2, 0..639 above) and hold G(alpha = 0.1) at a representative distance of the bucket
// (tab, built on the host by rbl_erf_table).  Outside that range the reference reads past its
// arrays; here G(0.1, d) is evaluated exactly instead.
__device__ __forceinline__ float rbl_table_g(const float* __restrict__ tab, float dis) {
  if (dis >= 0.1f && dis < 12.0f) return __ldg(tab + ((__float_as_int(dis) & 0x3FF8000) >> 15));
  const double d = (double)dis, sa = 0.31622776601683794;
  return (float)(erfc(sa * d) / (d * d) + 2.0 * sa * exp(-0.1 * d * d) / (1.7724538509055160273 * d));
}

// RBL near force of slot i: ComputeNearForceRBLERFWorklet (RunWorklet.cpp:710-814) and, without
// charges, ComputeLJForceRBLWorklet (:1218-1302).  Core pairs: Coulomb -q_i q_j G r/d on
// r = p_j' - p_i for 1e-4 < d^2 < rc^2 with G at |MinDistanceVec(p_j', p_i)|, then (outside the
// molecule) LJ on MinDistanceVec for 1e-4 < d^2 < rc^2.  Shell pairs: LJ x pice for
// rs^2 < d^2 < rc^2 (ComputeLJForceRcs) and, unless dropped, Coulomb x pice on the same range.
// The result is the reference's corr_force = LJ + qqr2e * Coulomb; k_force_sub_mean removes its
// mean afterwards.
// G > 1: G lanes per atom (small systems, where one thread per atom leaves most SMs idle); lane
// s takes entries s, s + G, ... and the lanes' sums are combined in FP64 by a fixed butterfly.
// Capped at 64 registers (8 blocks per SM, a few bytes of spill): 0.200 -> 0.187 ms at 98k atoms.
template <class R, bool COUL, bool SPW, int G>
__global__ void __launch_bounds__(128, 8) k_rbl_force(
    RblParams prm, const LJTable* __restrict__ ljt, const typename Traits<R>::V4* __restrict__ pos4,
    const int2* __restrict__ meta, const int* __restrict__ nbr, const int* __restrict__ ncore,
    const int* __restrict__ nshell, const RepDev* __restrict__ reps, const int* __restrict__ rep_of_slot,
    const int* __restrict__ slot_atom, int shell_cap, double* __restrict__ force,
    double* __restrict__ energy_slot, uint32_t* status) {
  using V4 = typename Traits<R>::V4;
  __shared__ R lj_a[kMaxReplicaTypes * kMaxReplicaTypes], lj_s6[kMaxReplicaTypes * kMaxReplicaTypes];
  const int nt2 = prm.ntypes * prm.ntypes;
  for (int t = threadIdx.x; t < nt2; t += blockDim.x) {
    lj_a[t] = lj24<R>(*ljt, t);
    lj_s6[t] = sig6<R>(*ljt, t);
  }
  __syncthreads();
  const int gid = (int)((blockIdx.x * blockDim.x + threadIdx.x) / G);
  const int sub = G == 1 ? 0 : (int)(threadIdx.x % G);
  if (G == 1 && gid >= prm.n) return;
  const bool active = gid < prm.n;   // inactive lanes of a partial group still join the shuffles
  const int i = active ? gid : prm.n - 1;
  const RepDev& rp = reps[rep_of_slot ? rep_of_slot[i] : 0];
  const R pice = (R)rp.rbl_pice;
  const V4 pi = pos4[i];
  const bool MOLEC = prm.molecular != 0;
  const bool typed = MOLEC || prm.ntypes > 1;
  const int2 mi = typed ? meta[i] : make_int2(0, 0);
  const int trow = prm.ntypes > 1 ? mi.x * prm.ntypes : 0;   // one LJ type when all types agree
  const R rc = (R)prm.rc, rs = (R)prm.rs;
  const R rc2 = rc * rc, rs2 = rs * rs;
  const R box[3] = {Traits<R>::box(rp, 0), Traits<R>::box(rp, 1), Traits<R>::box(rp, 2)};
  const R wrap[3] = {Traits<R>::wrap(rp, 0), Traits<R>::wrap(rp, 1), Traits<R>::wrap(rp, 2)};
  const R sa = (R)prm.sqrt_alpha, aa = (R)prm.alpha, c2 = (R)prm.two_sqrt_alpha_over_sqrt_pi;
  const R qqr2e = (R)prm.qqr2e;
  const R qi = pi.w;
  const size_t st = (size_t)prm.stride;
  Acc<R> fx, fy, fz;
  double e_lj = 0, e_coul = 0;
  const int nco = min(ncore[i], prm.core_cap), nsh = active ? min(nshell[i], shell_cap) : 0;
  const int nall = active ? nco + nsh : 0;
  for (int p = sub; p < nall; p += G) {
    const bool shell = p >= nco;
    const int row = shell ? prm.core_cap + (p - nco) : p;
    const int e = __ldg(nbr + (size_t)row * st + i);
    const int js = e >> kShiftBits;
    const V4 pj = pos4[js];
    R px = pj.x, py = pj.y, pz = pj.z;
    if (e & 63) {
      const int k0 = e & 3, k1 = (e >> 2) & 3, k2 = (e >> 4) & 3;
      px = px - (k0 == 1 ? wrap[0] : (k0 == 2 ? -wrap[0] : (R)0));
      py = py - (k1 == 1 ? wrap[1] : (k1 == 2 ? -wrap[1] : (R)0));
      pz = pz - (k2 == 1 ? wrap[2] : (k2 == 2 ? -wrap[2] : (R)0));
    }
    const R r0 = px - pi.x, r1 = py - pi.y, r2 = pz - pi.z;
    R m0 = r0, m1 = r1, m2 = r2;   // MinDistanceVec(p_j', p_i)
    min_image(m0, m1, m2, box);
    const R dm2 = m0 * m0 + m1 * m1 + m2 * m2;
    const R w = shell ? pice : (R)1;
    R t0 = 0, t1 = 0, t2 = 0;
    if (COUL && (!shell || prm.shell_coul)) {
      const R qq = qi * pj.w;
      const R d2 = r0 * r0 + r1 * r1 + r2 * r2;
      const bool ok = shell ? (d2 < rc2 && d2 > rs2) : (d2 < rc2 && d2 > (R)1.0e-4);
      if (qq != (R)0 && ok) {
        const R dis = sqrt_r(d2);
        const R dism = sqrt_r(dm2);
        R g;
        if (prm.table_mode) {
          g = (R)rbl_table_g(prm.erf_tab, (float)dism);
        } else {
          const R inv = (R)1 / dism;
          const R ex = exp_r(-aa * dm2);
          g = (erfc_shared(sa * dism, ex) * inv + c2 * ex) * inv;
        }
        const R s = -qq * g / dis * qqr2e * w;
        t0 += s * r0; t1 += s * r1; t2 += s * r2;
        if (energy_slot) {
          const double dd = (double)dism;
          e_coul += (double)w * (double)qqr2e * (double)qq * erfc(prm.sqrt_alpha * dd) / dd;
        }
      }
    }
    bool same = false;
    int tj = 0;
    R wsp = (R)1;   // special-bond LJ weight (molecular == 2: meta.y is the bond-graph component)
    if (typed) {
      const int2 mj = meta[js];
      same = MOLEC && (mj.y == mi.y);
      tj = prm.ntypes > 1 ? mj.x : 0;
      if (SPW && same) {
        wsp = special_weight<R>(prm.sp, slot_atom[i], slot_atom[js]);
        same = false;
      }
    }
    if (!same) {
      const bool ok = shell ? (dm2 < rc2 && dm2 > rs2) : (dm2 < rc2 && dm2 > (R)0.0001);
      if (ok) {
        const R inv2 = (R)1 / dm2;
        const R sd6 = lj_s6[trow + tj] * inv2 * inv2 * inv2;
        const R a24 = lj_a[trow + tj];
        R scal = w * (a24 * (((R)2 * sd6 - (R)1) * sd6) * inv2);
        if (SPW) scal *= wsp;
        t0 += scal * m0; t1 += scal * m1; t2 += scal * m2;
        if (energy_slot) e_lj += (double)(w * wsp) * (double)(-a24 / (R)6 * (sd6 - (R)1) * sd6);
      }
    }
    fx.add(t0); fy.add(t1); fz.add(t2);
  }
  double F[3] = {fx.value(), fy.value(), fz.value()};
  if (G > 1) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      F[0] += __shfl_xor_sync(0xffffffffu, F[0], o);
      F[1] += __shfl_xor_sync(0xffffffffu, F[1], o);
      F[2] += __shfl_xor_sync(0xffffffffu, F[2], o);
      e_lj += __shfl_xor_sync(0xffffffffu, e_lj, o);
      e_coul += __shfl_xor_sync(0xffffffffu, e_coul, o);
    }
    if (!active || sub != 0) return;
  }
  if (!isfinite(F[0]) || !isfinite(F[1]) || !isfinite(F[2])) set_flag(status, kFlagNonFinite);
  const int id = slot_atom[i];
  force[3 * id] = F[0];
  force[3 * id + 1] = F[1];
  force[3 * id + 2] = F[2];
  if (energy_slot) {
    energy_slot[2 * i] = 0.5 * e_lj;
    energy_slot[2 * i + 1] = 0.5 * e_coul;
  }
}

// EAM over the RBL lists: ComputeEAMfp_Worklet and ComputeEAMRBLWorklet (RunWorklet.cpp:
// 1052-1216) with ComputeEAMrhoRs / ComputeEAMforceRBL (rbmd/framework/forceFunction/
// ExecForceFunction.h:358-381,484-520): core pairs as the full-list passes (0.01 < r^2 < rc^2),
// shell pairs x pice for rs^2 < r^2 < rc^2, pair vector MinDistanceVec(p_i, p_j').
template <class R>
__device__ __forceinline__ void rbl_eam_pair(const typename Traits<R>::V4& pi, const typename Traits<R>::V4& pj,
                                             int e, const R* wrap, const R* box, R* r) {
  const R pjv[3] = {pj.x, pj.y, pj.z}, piv[3] = {pi.x, pi.y, pi.z};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int cd = (e >> (2 * d)) & 3;
    const R off = cd == 1 ? wrap[d] : (cd == 2 ? -wrap[d] : (R)0);
    r[d] = piv[d] - (pjv[d] - off);
  }
  min_image(r[0], r[1], r[2], box);
}

template <class R>
__global__ void __launch_bounds__(128) k_rbl_eam_fp(int n, int stride, int core_cap, int shell_cap, double rc,
                                                    double rs, EamDev eam,
                                                    const typename Traits<R>::V4* __restrict__ pos4,
                                                    const int* __restrict__ nbr, const int* __restrict__ ncore,
                                                    const int* __restrict__ nshell,
                                                    const RepDev* __restrict__ reps,
                                                    const int* __restrict__ rep_of_slot, R* __restrict__ fp,
                                                    double* __restrict__ embed_slot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RepDev& rp = reps[rep_of_slot ? rep_of_slot[i] : 0];
  const R pice = (R)rp.rbl_pice;
  const typename Traits<R>::V4 pi = pos4[i];
  const R wrap[3] = {Traits<R>::wrap(rp, 0), Traits<R>::wrap(rp, 1), Traits<R>::wrap(rp, 2)};
  const R box[3] = {Traits<R>::box(rp, 0), Traits<R>::box(rp, 1), Traits<R>::box(rp, 2)};
  const R cut2 = (R)rc * (R)rc, rs2 = (R)rs * (R)rs;
  const R rdr = sizeof(R) == 4 ? (R)eam.rdr : (R)eam.rdr_d;
  Acc<R> rho;
  const int nco = min(ncore[i], core_cap), nsh = min(nshell[i], shell_cap);
  for (int p = 0; p < nco + nsh; ++p) {
    const bool shell = p >= nco;
    const int e = __ldg(nbr + (size_t)(shell ? core_cap + (p - nco) : p) * stride + i);
    R r[3];
    rbl_eam_pair<R>(pi, pos4[e >> kShiftBits], e, wrap, box, r);
    const R rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    const bool ok = shell ? (rsq < cut2 && rsq > rs2) : (rsq < cut2 && rsq > (R)0.01);
    if (!ok) continue;
    R pp = sqrt_r(rsq) * rdr + (R)1;
    int m = min((int)pp, eam.nr - 1);
    pp -= (R)m;
    pp = fmin(pp, (R)1);
    const float4 b = __ldg(eam.rhor + 2 * m + 0);
    const float4 c = __ldg(eam.rhor + 2 * m + 1);
    const R v = (((R)b.w * pp + (R)c.x) * pp + (R)c.y) * pp + (R)c.z;
    rho.add(shell ? pice * v : v);
  }
  const R rr = (R)rho.value();
  R pp = rr * (sizeof(R) == 4 ? (R)eam.rdrho : (R)eam.rdrho_d) + (R)1;
  int m = max(1, min((int)pp, eam.nrho - 1));
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

template <class R>
__global__ void __launch_bounds__(128) k_rbl_eam_force(int n, int stride, int core_cap, int shell_cap, double rc,
                                                       double rs, EamDev eam,
                                                       const typename Traits<R>::V4* __restrict__ pos4,
                                                       const int* __restrict__ nbr, const int* __restrict__ ncore,
                                                       const int* __restrict__ nshell,
                                                       const RepDev* __restrict__ reps,
                                                       const int* __restrict__ rep_of_slot,
                                                       const R* __restrict__ fp, const int* __restrict__ slot_atom,
                                                       double* __restrict__ force, double* __restrict__ pair_slot,
                                                       uint32_t* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RepDev& rp = reps[rep_of_slot ? rep_of_slot[i] : 0];
  const R pice = (R)rp.rbl_pice;
  const typename Traits<R>::V4 pi = pos4[i];
  const R wrap[3] = {Traits<R>::wrap(rp, 0), Traits<R>::wrap(rp, 1), Traits<R>::wrap(rp, 2)};
  const R box[3] = {Traits<R>::box(rp, 0), Traits<R>::box(rp, 1), Traits<R>::box(rp, 2)};
  const R cut2 = (R)rc * (R)rc, rs2 = (R)rs * (R)rs;
  const R rdr = sizeof(R) == 4 ? (R)eam.rdr : (R)eam.rdr_d;
  const R fpi = fp[i];
  Acc<R> fx, fy, fz;
  double epair = 0;
  const int nco = min(ncore[i], core_cap), nsh = min(nshell[i], shell_cap);
  for (int p = 0; p < nco + nsh; ++p) {
    const bool shell = p >= nco;
    const int e = __ldg(nbr + (size_t)(shell ? core_cap + (p - nco) : p) * stride + i);
    const int j = e >> kShiftBits;
    R r[3];
    rbl_eam_pair<R>(pi, pos4[j], e, wrap, box, r);
    const R rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    const bool ok = shell ? (rsq < cut2 && rsq > rs2) : (rsq < cut2 && rsq > (R)0.01);
    if (!ok) continue;
    const R rv = sqrt_r(rsq);
    R pp = rv * rdr + (R)1;
    int m = min((int)pp, eam.nr - 1);
    pp -= (R)m;
    pp = fmin(pp, (R)1);
    const float4 ra = __ldg(eam.rhor + 2 * m + 0);
    const float4 za = __ldg(eam.z2r + 2 * m + 0);
    const float4 zb = __ldg(eam.z2r + 2 * m + 1);
    const R rhop = ((R)ra.x * pp + (R)ra.y) * pp + (R)ra.z;
    const R z2p = ((R)za.x * pp + (R)za.y) * pp + (R)za.z;
    const R z2 = (((R)za.w * pp + (R)zb.x) * pp + (R)zb.y) * pp + (R)zb.z;
    const R recip = (R)1 / rv;
    const R phi = z2 * recip;
    const R phip = z2p * recip - phi * recip;
    const R psip = fpi * rhop + fp[j] * rhop + phip;
    const R fpair = -psip * recip;
    const R w = shell ? pice : (R)1;
    fx.add(w * (r[0] * fpair));
    fy.add(w * (r[1] * fpair));
    fz.add(w * (r[2] * fpair));
    epair += (double)w * (double)phi;
  }
  const double F[3] = {fx.value(), fy.value(), fz.value()};
  if (!isfinite(F[0]) || !isfinite(F[1]) || !isfinite(F[2])) set_flag(status, kFlagNonFinite);
  const int id = slot_atom[i];
  force[3 * id] = F[0];
  force[3 * id + 1] = F[1];
  force[3 * id + 2] = F[2];
  if (pair_slot) pair_slot[i] = 0.5 * epair;
}

// Mean removal F_i -= (sum_j F_j) / N_replica (SumRBLCorrForceWorklet, RunWorklet.cpp:1304-1321,
// after the Reduce of ExecutionMD.cpp:568-569): per-chunk FP64 sums in a fixed order, then every
// block re-sums its replica's chunk partials in chunk order (deterministic) and subtracts.
__global__ void __launch_bounds__(256) k_force_chunk_sum(const MdChunk* __restrict__ chunks,
                                                         const double* __restrict__ force,
                                                         double* __restrict__ partial) {
  const MdChunk c = chunks[blockIdx.x];
  double s[3] = {0, 0, 0};
  for (int a = c.begin + threadIdx.x; a < c.end; a += blockDim.x)
#pragma unroll
    for (int d = 0; d < 3; ++d) s[d] += force[3 * a + d];
  __shared__ double red[3][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double v = s[d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[d][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
    partial[3 * blockIdx.x + threadIdx.x] = v;
  }
}

__global__ void __launch_bounds__(256) k_force_sub_mean(const MdChunk* __restrict__ chunks,
                                                        const int* __restrict__ chunk_rep_begin,
                                                        const RepDev* __restrict__ reps,
                                                        const double* __restrict__ partial,
                                                        double* __restrict__ force) {
  const MdChunk c = chunks[blockIdx.x];
  __shared__ double mean[3];
  if (threadIdx.x < 3) {
    double v = 0;
    for (int k = chunk_rep_begin[c.rep]; k < chunk_rep_begin[c.rep + 1]; ++k) v += partial[3 * k + threadIdx.x];
    const RepDev& rp = reps[c.rep];
    mean[threadIdx.x] = v / (double)(rp.atom_end - rp.atom_begin);
  }
  __syncthreads();
  for (int a = c.begin + threadIdx.x; a < c.end; a += blockDim.x)
#pragma unroll
    for (int d = 0; d < 3; ++d) force[3 * a + d] -= mean[d];
}

}  // namespace rbmd
