// kernels_cells.cuh -- cell binning, deterministic cell sort and the full neighbour list.
//
// Reference: ContPointLocator::Build + BinPointsWorklet (rbmd/framework/locator/
// ContPointLocator.cxx:38-92) does bin -> SortByKey -> Lower/UpperBounds with library calls.
// Here: fused bin + per-cell atomic count (in the integrator or k_bin), one-block scan, atomic
// scatter, then a warp per cell ranks its atoms by caller id so the slot order is deterministic
// (a stable sort by (cell, id)), and the same warp gathers the slot-ordered caches.
#pragma once
#include "common.cuh"

namespace rbmd {

// cell index of a position, BinPointsWorklet semantics (truncate, clamp to [0, dims-1])
template <class R>
__device__ __forceinline__ int cell_of_pos(const RepDev& rp, R x, R y, R z) {
  R p[3] = {x, y, z};
  int ijk[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int c = (int)div_rn(sub_rn(p[d], Traits<R>::lo(rp, d)), Traits<R>::dx(rp, d));
    c = max(c, 0);
    c = min(c, rp.dims[d] - 1);
    ijk[d] = c;
  }
  return rp.cell_base + ijk[0] + ijk[1] * rp.dims[0] + ijk[2] * rp.dims[0] * rp.dims[1];
}

// Verlet-skin rebuild flags: rebuild[r] for replica r and rebuild[n_replicas] for "any replica";
// a replica whose atoms all stayed within skin/2 keeps its cells, slots and list.
// rebuild (nullable): bin only the atoms of rebuilding replicas.
template <class R>
__global__ void k_bin(int n, const double* __restrict__ pos, const int* __restrict__ rep_of,
                      const RepDev* __restrict__ reps, int* __restrict__ cell_of,
                      int* __restrict__ cell_count, uint32_t* status, const int* __restrict__ rebuild) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = rep_of ? rep_of[i] : 0;
  if (rebuild && !rebuild[r]) return;
  const RepDev& rp = reps[r];
  double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
  if (!isfinite(x) || !isfinite(y) || !isfinite(z)) set_flag(status, kFlagNonFinite);
  int c = cell_of_pos<R>(rp, (R)x, (R)y, (R)z);
  cell_of[i] = c;
  atomicAdd(&cell_count[c], 1);
}

// Exclusive scan of the cell counts in two parallel passes: k_cell_block_sums reduces blocks of
// kScanBlock cells; k_cell_scan gives each block its prefix (sum of the preceding block sums)
// and scans its cells.  cell_start[ncell] = n; scatter cursors are cleared; over-full cells flag.
// `rebuild` (nullable, the "any replica" flag): skip the pass when every list is reused.  Cells
// of replicas that keep their list keep their counts, so their starts come out unchanged.
constexpr int kScanBlock = 4096;

// Number of replicas whose list is rebuilt in this pass (the list-build counter counts replica
// lists: with one replica, the number of rebuilding passes).
__device__ __forceinline__ unsigned long long rebuilt_replicas(const int* rebuild, int n_rep) {
  if (!rebuild) return (unsigned long long)n_rep;
  unsigned long long c = 0;
  for (int r = 0; r < n_rep; ++r) c += rebuild[r] != 0;
  return c;
}

// Zero the cell counts of the rebuilding replicas (all of them when rebuild is null).
__global__ void k_zero_counts(int ncell, const int* __restrict__ cell_rep, const int* __restrict__ rebuild,
                              int* __restrict__ cell_count) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  if (rebuild && !rebuild[cell_rep ? cell_rep[c] : 0]) return;
  cell_count[c] = 0;
}

__global__ void __launch_bounds__(1024) k_cell_block_sums(int ncell, const int* __restrict__ count,
                                                          int* __restrict__ block_sums,
                                                          const int* __restrict__ rebuild,
                                                          uint32_t* status) {
  if (rebuild && !*rebuild) return;
  __shared__ int red[32];
  const int b0 = blockIdx.x * kScanBlock;
  int s = 0, mx = 0;
  for (int c = b0 + threadIdx.x; c < min(ncell, b0 + kScanBlock); c += blockDim.x) {
    const int v = count[c];
    s += v;
    mx = max(mx, v);
  }
  if (mx > kMaxCellAtoms) set_flag(status, kFlagCellOverflow);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    block_sums[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(1024) k_cell_scan(int ncell, const int* __restrict__ count,
                                                    const int* __restrict__ block_sums,
                                                    int* __restrict__ start, int* __restrict__ cursor,
                                                    const int* __restrict__ rebuild) {
  if (rebuild && !*rebuild) return;
  __shared__ int warp_sums[32];
  __shared__ int base_sh;
  const int t = threadIdx.x, nt = blockDim.x;
  const int b0 = blockIdx.x * kScanBlock, b1 = min(ncell, b0 + kScanBlock);
  if (t < 32) {
    int v = 0;
    for (int b = t; b < (int)blockIdx.x; b += 32) v += block_sums[b];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (t == 0) base_sh = v;
  }
  // each thread owns kScanBlock / nt consecutive cells
  const int per = kScanBlock / nt;
  const int c0 = b0 + t * per;
  int local = 0;
  for (int c = c0; c < min(b1, c0 + per); ++c) local += count[c];
  const int lane = t & 31, w = t >> 5;
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_sums[w] = incl;
  __syncthreads();
  if (w == 0) {
    const int v = lane < (nt >> 5) ? warp_sums[lane] : 0;
    int inc2 = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, inc2, o);
      if (lane >= o) inc2 += y;
    }
    warp_sums[lane] = inc2 - v;
  }
  __syncthreads();
  int run = base_sh + warp_sums[w] + incl - local;
  for (int c = c0; c < min(b1, c0 + per); ++c) {
    start[c] = run;
    cursor[c] = 0;
    run += count[c];
  }
  if (b1 == ncell && t == nt - 1) start[ncell] = run;
}

__global__ void k_scatter(int n, const int* __restrict__ cell_of, const int* __restrict__ start,
                          int* __restrict__ cursor, int* __restrict__ tmp_slot_atom,
                          const int* __restrict__ rep_of, const int* __restrict__ rebuild) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (rebuild && !rebuild[rep_of ? rep_of[i] : 0]) return;
  int c = cell_of[i];
  int s = start[c] + atomicAdd(&cursor[c], 1);
  tmp_slot_atom[s] = i;
}

// Total order of positions for the cell sort: IEEE bits mapped so that unsigned comparison
// follows the float order (NaNs land at the ends, so a rank is always a permutation).
__device__ __forceinline__ uint32_t ord_key(float x) {
  const uint32_t b = __float_as_uint(x);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ unsigned long long ord_key(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

// One warp per cell: rank the cell's atoms by caller id (ids are distinct), or with sort_x by
// (x in the run precision, caller id), and gather the slot-ordered caches.  With sort_x every
// row of consecutive x cells is ordered by x, which lets the list build skip the candidates
// beyond the cutoff in x by binary search.  Cells above kMaxCellAtoms keep the scatter order
// (flagged by the scan).
constexpr int kSortWarps = 4;   // cells (one per warp) per block of k_cell_sort_gather

template <class R>
__global__ void __launch_bounds__(32 * kSortWarps) k_cell_sort_gather(
    int ncell, const int* __restrict__ start, const int* __restrict__ tmp_slot_atom,
    const double* __restrict__ pos, const double* __restrict__ charge,
    const int* __restrict__ type, const int* __restrict__ mol, const int* __restrict__ rep_of,
    const RepDev* __restrict__ reps, int* __restrict__ slot_atom, int* __restrict__ atom_slot,
    typename Traits<R>::V4* __restrict__ pos4, void* __restrict__ frac_out,
    int2* __restrict__ meta, double* __restrict__ xref, const int* __restrict__ rebuild, int sort_x,
    const int* __restrict__ cell_rep) {
  using Key = decltype(ord_key((R)0));
  __shared__ int ids[kSortWarps][kMaxCellAtoms];
  __shared__ Key keys[kSortWarps][kMaxCellAtoms];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int cell = blockIdx.x * kSortWarps + w;
  if (cell >= ncell) return;
  if (rebuild && !rebuild[cell_rep ? cell_rep[cell] : 0]) return;
  const int s0 = start[cell], n = start[cell + 1] - s0;
  if (n == 0) return;
  const bool sortable = n <= kMaxCellAtoms;
  if (sortable)
    for (int k = lane; k < n; k += 32) {
      const int id = tmp_slot_atom[s0 + k];
      ids[w][k] = id;
      if (sort_x) keys[w][k] = ord_key((R)pos[3 * id]);
    }
  __syncwarp();
  for (int k = lane; k < n; k += 32) {
    int id = sortable ? ids[w][k] : tmp_slot_atom[s0 + k];
    int rank = k;
    if (sortable) {
      rank = 0;
      if (sort_x) {
        const Key kk = keys[w][k];
        for (int m = 0; m < n; ++m) {
          const Key km = keys[w][m];
          rank += km < kk || (km == kk && ids[w][m] < id);
        }
      } else {
        for (int m = 0; m < n; ++m) rank += ids[w][m] < id;
      }
    }
    const int slot = s0 + rank;
    slot_atom[slot] = id;
    atom_slot[id] = slot;
    const double x = pos[3 * id], y = pos[3 * id + 1], z = pos[3 * id + 2];
    const double q = charge ? charge[id] : 0.0;
    if (xref) { xref[3 * id] = x; xref[3 * id + 1] = y; xref[3 * id + 2] = z; }
    typename Traits<R>::V4 v;
    v.x = (R)x; v.y = (R)y; v.z = (R)z; v.w = (R)q;
    pos4[slot] = v;
    if (meta) meta[slot] = make_int2(type ? type[id] : 0, mol ? mol[id] : id);
    if (frac_out) {
      const RepDev& rp = reps[rep_of ? rep_of[id] : 0];
      double u[3] = {(x - rp.lo_d[0]) / rp.box_d[0], (y - rp.lo_d[1]) / rp.box_d[1],
                     (z - rp.lo_d[2]) / rp.box_d[2]};
      if (sizeof(R) == 4) {
        uint32_t U[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          U[d] = turn32(u[d] - floor(u[d]));
        }
        Frac32 fr{U[0], U[1], U[2], (float)q};
        reinterpret_cast<Frac32*>(frac_out)[slot] = fr;
      } else {
        unsigned long long U[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          U[d] = turn64(u[d] - floor(u[d]));
        }
        Frac64 fr{U[0], U[1], U[2], q};
        reinterpret_cast<Frac64*>(frac_out)[slot] = fr;
      }
    }
  }
}

// Refresh the slot caches from the master positions without re-binning (list reuse with skin).
// With xref (positions at the last build) the cached position is unwrapped: xref plus the
// minimum-image displacement since the build.  A listed pair's stored image shift then stays
// valid however often either atom crossed a face, so the pair kernels need no minimum-image
// step; the displacement is below skin/2, far under half a box.
template <class R>
__global__ void k_regather(int n, const int* __restrict__ slot_atom, const double* __restrict__ pos,
                           const double* __restrict__ charge, const int* __restrict__ rep_of,
                           const RepDev* __restrict__ reps, typename Traits<R>::V4* __restrict__ pos4,
                           void* __restrict__ frac_out, const double* __restrict__ xref,
                           const int* __restrict__ rebuild) {
  int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= n) return;
  int id = slot_atom[slot];
  if (rebuild && rebuild[rep_of ? rep_of[id] : 0]) return;   // the cell sort refreshed these caches
  const double x = pos[3 * id], y = pos[3 * id + 1], z = pos[3 * id + 2];
  const double q = charge ? charge[id] : 0.0;
  typename Traits<R>::V4 v;
  if (xref) {
    const RepDev& rp = reps[rep_of ? rep_of[id] : 0];
    double u[3] = {x, y, z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double r0 = xref[3 * id + d];
      double dd = u[d] - r0;
      if (fabs(dd) > 0.5 * rp.box_d[d]) dd -= (dd > 0 ? rp.box_d[d] : -rp.box_d[d]);
      u[d] = r0 + dd;
    }
    v.x = (R)u[0]; v.y = (R)u[1]; v.z = (R)u[2];
  } else {
    v.x = (R)x; v.y = (R)y; v.z = (R)z;
  }
  v.w = (R)q;
  pos4[slot] = v;
  if (frac_out) {
    const RepDev& rp = reps[rep_of ? rep_of[id] : 0];
    double u[3] = {(x - rp.lo_d[0]) / rp.box_d[0], (y - rp.lo_d[1]) / rp.box_d[1],
                   (z - rp.lo_d[2]) / rp.box_d[2]};
    if (sizeof(R) == 4) {
      uint32_t U[3];
      for (int d = 0; d < 3; ++d) {
        U[d] = turn32(u[d] - floor(u[d]));
      }
      reinterpret_cast<Frac32*>(frac_out)[slot] = Frac32{U[0], U[1], U[2], (float)q};
    } else {
      unsigned long long U[3];
      for (int d = 0; d < 3; ++d) {
        U[d] = turn64(u[d] - floor(u[d]));
      }
      reinterpret_cast<Frac64*>(frac_out)[slot] = Frac64{U[0], U[1], U[2], q};
    }
  }
}

// Periodic cell index: v mod d in [0, d).  Stencil rows stay within one period of the box for
// atoms inside or near it, where one compare and add replace the integer division; atoms
// further out take the division.
__device__ __forceinline__ int wrap_cell(int v, int d) {
  if (v >= 0 && v < d) return v;
  if (v < 0 && v >= -d) return v + d;
  if (v >= d && v < 2 * d) return v - d;
  return ((v % d) + d) % d;
}

// 1e-4 threshold of the neighbour predicate: the reference compares a float against the double
// literal 0.0001; for float x, (double)x > 1e-4 <=> x > 1e-4f (1e-4f < 1e-4 < nextafterf(1e-4f)).
__device__ __forceinline__ bool gt_small(float x) { return x > 1.0e-4f; }
__device__ __forceinline__ bool gt_small(double x) { return x > 1.0e-4; }
// cut2 - d2 of a candidate: the list keeps it above 1e-4 (ComputeNeighboursWorklet); the
// "ORIGINAL" neighbour type, which leaves the cutoff to the force function, keeps d2 < cut2
template <class R>
__device__ __forceinline__ bool inside_cut(R margin, int orig) { return orig ? margin > (R)0 : gt_small(margin); }

// Full Verlet list of slot i with the predicate of ComputeNeighboursWorklet
// (rbmd/framework/run/worklet/RunWorklet.cpp:40-96): rc^2 - d^2 > 1e-4 && d^2 > 1e-4 on
// r = (p_j - offset) - p_i with uncontracted float ops and the reference's cell-based periodic
// offsets (PeriodicCoordOffset).  Traversal: for each of the (2nc+1)^2 (y, z) neighbour rows the
// x cells ci-nc .. ci+nc are consecutive cell indices, hence one contiguous slot range when no x
// wrap occurs; rows that wrap in x are walked cell by cell.  The pair set equals the
// reference's 27-cell stencil; the order inside a row differs (sets are order-free).
template <class R>
__device__ __forceinline__ int nlist_range(int s, const int s1, const typename Traits<R>::V4* __restrict__ pos4,
                                           const R* pix, const R* off, int code, R cut2, int idx, int cap,
                                           int stride, int i, int* __restrict__ nbr, int orig) {
#pragma unroll 4
  for (; s < s1; ++s) {
    const typename Traits<R>::V4 pj = pos4[s];
    const R r0 = sub_rn(sub_rn(pj.x, off[0]), pix[0]);
    const R r1 = sub_rn(sub_rn(pj.y, off[1]), pix[1]);
    const R r2 = sub_rn(sub_rn(pj.z, off[2]), pix[2]);
    const R d2 = add_rn(add_rn(mul_rn(r0, r0), mul_rn(r1, r1)), mul_rn(r2, r2));
    if (inside_cut(sub_rn(cut2, d2), orig) && gt_small(d2)) {
      if (idx < cap) __stcs(nbr + (size_t)idx * stride + i, (s << kShiftBits) | code);
      ++idx;
    }
  }
  return idx;
}

// Per-thread traversal of slot i's 27-cell stencil straight from global memory; returns the
// number of pairs found (entries beyond cap are counted, not stored).
// First slot s in [lo, hi) with pos4[s].x >= bound (the range is ordered by x).
template <class R>
__device__ __forceinline__ int lower_x(const typename Traits<R>::V4* __restrict__ pos4, int lo, int hi, R bound) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (pos4[mid].x < bound) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// trim_x: cells are ordered by x (k_cell_sort_gather with sort_x), so each contiguous x range
// is cut to the candidates with |x_j' - x_i| below the cutoff plus a rounding margin before the
// exact predicate runs; the accepted pairs and their order are unchanged.
template <class R>
__device__ int nlist_thread(int i, const typename Traits<R>::V4 pi, const RepDev& rp,
                            const typename Traits<R>::V4* __restrict__ pos4,
                            const int* __restrict__ cell_start, int num_cycles, R rc, int cap, int stride,
                            int* __restrict__ nbr, bool trim_x = false, int orig = 0) {
  const R pix[3] = {pi.x, pi.y, pi.z};
  const R xm = rc + (fabs(pix[0]) + (R)2 * rc) * (R)1e-5 + (R)1e-6;   // cutoff + margin in x
  int ci[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    ci[d] = (int)div_rn(sub_rn(pix[d], Traits<R>::lo(rp, d)), Traits<R>::dx(rp, d));
  const R cut2 = mul_rn(rc, rc);
  const int nc = num_cycles;
  const int dx0 = rp.dims[0], dx1 = rp.dims[1], dx2 = rp.dims[2];
  const bool x_contig = ci[0] - nc >= 0 && ci[0] + nc < dx0;
  int idx = 0;
  for (int b = -nc; b <= nc; ++b) {
    const int nby = ci[1] + b;
    const int wy = wrap_cell(nby, dx1), dy = wy - nby;
    for (int c = -nc; c <= nc; ++c) {
      R off[3];
      const int nbz = ci[2] + c;
      const int wz = wrap_cell(nbz, dx2), dz = wz - nbz;
      off[1] = mul_rn(Traits<R>::dx(rp, 1), (R)dy);
      off[2] = mul_rn(Traits<R>::dx(rp, 2), (R)dz);
      const int code_yz = ((dy > 0 ? 1 : (dy < 0 ? 2 : 0)) << 2) | ((dz > 0 ? 1 : (dz < 0 ? 2 : 0)) << 4);
      const int row = rp.cell_base + wy * dx0 + wz * dx0 * dx1;
      if (x_contig) {
        off[0] = (R)0;
        int s0 = cell_start[row + ci[0] - nc], s1 = cell_start[row + ci[0] + nc + 1];
        if (trim_x) {
          s0 = lower_x<R>(pos4, s0, s1, pix[0] - xm);
          s1 = lower_x<R>(pos4, s0, s1, pix[0] + xm);
        }
        idx = nlist_range<R>(s0, s1, pos4, pix, off, code_yz, cut2, idx, cap, stride, i, nbr, orig);
      } else {
        for (int a = -nc; a <= nc; ++a) {
          const int nbx = ci[0] + a;
          const int wx = wrap_cell(nbx, dx0);
          const int ddx = wx - nbx;
          off[0] = mul_rn(Traits<R>::dx(rp, 0), (R)ddx);
          const int code = code_yz | (ddx > 0 ? 1 : (ddx < 0 ? 2 : 0));
          int s0 = cell_start[row + wx], s1 = cell_start[row + wx + 1];
          if (trim_x) {
            const R xw = xm + fabs(off[0]) * (R)1e-5;   // the shifted bound rounds at |x_i + offset|
            s0 = lower_x<R>(pos4, s0, s1, pix[0] + off[0] - xw);
            s1 = lower_x<R>(pos4, s0, s1, pix[0] + off[0] + xw);
          }
          idx = nlist_range<R>(s0, s1, pos4, pix, off, code, cut2, idx, cap, stride, i, nbr, orig);
        }
      }
    }
  }
  return idx;
}

__device__ __forceinline__ void nlist_finish(int i, int idx, int cap, int* __restrict__ count,
                                             int* __restrict__ max_count, uint32_t* status) {
  count[i] = idx;
  if (idx > cap) {
    set_flag(status, kFlagListOverflow);
    atomicMax(max_count, idx);
  }
}

template <class R>
__global__ void __launch_bounds__(256) k_nlist(
    int n, const typename Traits<R>::V4* __restrict__ pos4, const int* __restrict__ cell_start,
    const RepDev* __restrict__ reps, const int* __restrict__ rep_of_slot, int num_cycles, R rc,
    int cap, int stride, int* __restrict__ nbr, int* __restrict__ count, int* __restrict__ max_count,
    uint32_t* status, const int* __restrict__ rebuild, unsigned long long* __restrict__ nbuilds,
    int trim_x, int n_rep, int orig) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && nbuilds) atomicAdd(nbuilds, rebuilt_replicas(rebuild, n_rep));
  if (i >= n) return;
  const int r = rep_of_slot ? rep_of_slot[i] : 0;
  if (rebuild && !rebuild[r]) return;
  const RepDev& rp = reps[r];
  const int idx = nlist_thread<R>(i, pos4[i], rp, pos4, cell_start, num_cycles, rc, cap, stride, nbr,
                                  trim_x != 0, orig);
  nlist_finish(i, idx, cap, count, max_count, status);
}

// Warp-per-atom list build for systems with few atoms and many candidates per atom (long
// cutoffs): the 32 lanes test consecutive candidates of a cell range together and a ballot
// compacts the accepted ones in candidate order, so the list equals k_nlist's entry for entry.
template <class R>
__global__ void __launch_bounds__(256) k_nlist_warp(
    int n, const typename Traits<R>::V4* __restrict__ pos4, const int* __restrict__ cell_start,
    const RepDev* __restrict__ reps, const int* __restrict__ rep_of_slot, R rc, int cap, int stride,
    int* __restrict__ nbr, int* __restrict__ count, int* __restrict__ max_count, uint32_t* status,
    const int* __restrict__ rebuild, unsigned long long* __restrict__ nbuilds, int n_rep, int orig) {
  using V4 = typename Traits<R>::V4;
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i == 0 && lane == 0 && nbuilds) atomicAdd(nbuilds, rebuilt_replicas(rebuild, n_rep));
  if (i >= n) return;
  const int r = rep_of_slot ? rep_of_slot[i] : 0;
  if (rebuild && !rebuild[r]) return;
  const RepDev& rp = reps[r];
  const V4 pi = pos4[i];
  const R pix[3] = {pi.x, pi.y, pi.z};
  int ci[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    ci[d] = (int)div_rn(sub_rn(pix[d], Traits<R>::lo(rp, d)), Traits<R>::dx(rp, d));
  const R cut2 = mul_rn(rc, rc);
  const int dx0 = rp.dims[0], dx1 = rp.dims[1], dx2 = rp.dims[2];
  const bool x_contig = ci[0] - 1 >= 0 && ci[0] + 1 < dx0;
  const unsigned below = (1u << lane) - 1u;
  int idx = 0;
  // (no x-window search here: a serial binary search per row costs the warp more latency than
  // the 32-wide candidate test it would save)
  auto scan = [&](int s0, int s1, R o0, R o1, R o2, int code) {
    for (int base = s0; base < s1; base += 32) {
      const int sj = base + lane;
      bool ok = false;
      if (sj < s1) {
        const V4 pj = pos4[sj];
        const R r0 = sub_rn(sub_rn(pj.x, o0), pix[0]);
        const R r1 = sub_rn(sub_rn(pj.y, o1), pix[1]);
        const R r2 = sub_rn(sub_rn(pj.z, o2), pix[2]);
        const R d2 = add_rn(add_rn(mul_rn(r0, r0), mul_rn(r1, r1)), mul_rn(r2, r2));
        ok = inside_cut(sub_rn(cut2, d2), orig) && gt_small(d2);
      }
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        const int at = idx + __popc(m & below);
        if (at < cap) __stcs(nbr + (size_t)at * stride + i, (sj << kShiftBits) | code);
      }
      idx += __popc(m);
    }
  };
  for (int b = -1; b <= 1; ++b)
    for (int c = -1; c <= 1; ++c) {
      const int nby = ci[1] + b, nbz = ci[2] + c;
      const int wy = wrap_cell(nby, dx1), wz = wrap_cell(nbz, dx2);
      const int dy = wy - nby, dz = wz - nbz;
      const R o1 = mul_rn(Traits<R>::dx(rp, 1), (R)dy), o2 = mul_rn(Traits<R>::dx(rp, 2), (R)dz);
      const int code_yz = ((dy > 0 ? 1 : (dy < 0 ? 2 : 0)) << 2) | ((dz > 0 ? 1 : (dz < 0 ? 2 : 0)) << 4);
      const int row = rp.cell_base + wy * dx0 + wz * dx0 * dx1;
      if (x_contig) {
        scan(cell_start[row + ci[0] - 1], cell_start[row + ci[0] + 2], (R)0, o1, o2, code_yz);
      } else {
        for (int a = -1; a <= 1; ++a) {
          const int nbx = ci[0] + a;
          const int wx = wrap_cell(nbx, dx0);
          const int ddx = wx - nbx;
          scan(cell_start[row + wx], cell_start[row + wx + 1], mul_rn(Traits<R>::dx(rp, 0), (R)ddx), o1, o2,
               code_yz | (ddx > 0 ? 1 : (ddx < 0 ? 2 : 0)));
        }
      }
    }
  if (lane == 0) nlist_finish(i, idx, cap, count, max_count, status);
}

// ---- staged list build ------------------------------------------------------------------
// One block per segment of kSeg consecutive x cells of one (y, z) cell row.  The block copies
// the positions of its 9 neighbour rows x (segment + 1 cell each side) into shared memory once,
// already shifted by their periodic offsets and tagged with (slot << 6 | image code), and every
// atom of the segment walks its 27 cells there.  Cells are visited in the same order, with the
// same float operations, as k_nlist, so the list is identical entry for entry.  A segment whose
// staged atoms exceed the shared buffer, or an atom whose own cell index falls outside the
// segment (binning clamps positions at the upper face), takes k_nlist's global-memory path.
struct ListSeg { int rep, y, z, x0, x1, pad0, pad1, pad2; };
constexpr int kStageThreads = 256;
constexpr int kSegMaxCells = 32;
constexpr int kStageCells = 9 * (kSegMaxCells + 2);

__device__ __forceinline__ float pack_tag(float, int v) { return __int_as_float(v); }
__device__ __forceinline__ double pack_tag(double, int v) { return (double)v; }
__device__ __forceinline__ int unpack_tag(float v) { return __float_as_int(v); }
__device__ __forceinline__ int unpack_tag(double v) { return (int)v; }

template <class R>
__global__ void __launch_bounds__(kStageThreads, 2) k_nlist_staged(
    const ListSeg* __restrict__ segs, int stage_cap, const typename Traits<R>::V4* __restrict__ pos4,
    const int* __restrict__ cell_start, const RepDev* __restrict__ reps, R rc, int cap, int stride,
    int* __restrict__ nbr, int* __restrict__ count, int* __restrict__ max_count, uint32_t* status,
    const int* __restrict__ rebuild, unsigned long long* __restrict__ nbuilds, int trim_x, int n_rep,
    int orig) {
  using V4 = typename Traits<R>::V4;
  if (blockIdx.x == 0 && threadIdx.x == 0 && nbuilds) atomicAdd(nbuilds, rebuilt_replicas(rebuild, n_rep));
  if (rebuild && !rebuild[segs[blockIdx.x].rep]) return;
  extern __shared__ __align__(16) unsigned char stage_raw[];
  V4* stage = reinterpret_cast<V4*>(stage_raw);
  __shared__ int cs[kStageCells + 1];     // staged start of staged cell k = row * W + u
  __shared__ int cell_k[kStageCells];     // its global cell index
  __shared__ int cnt_k[kStageCells];      // its atom count
  const ListSeg sg = segs[blockIdx.x];
  const RepDev& rp = reps[sg.rep];
  const int S = sg.x1 - sg.x0, W = S + 2, K = 9 * W;
  const int d0 = rp.dims[0], d1 = rp.dims[1], d2 = rp.dims[2];
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    const int r = k / W, u = k - r * W;
    const int wy = wrap_cell(sg.y + r / 3 - 1, d1), wz = wrap_cell(sg.z + r % 3 - 1, d2);
    const int wx = wrap_cell(sg.x0 - 1 + u, d0);
    const int cell = rp.cell_base + wx + wy * d0 + wz * d0 * d1;
    cell_k[k] = cell;
    cnt_k[k] = cell_start[cell + 1] - cell_start[cell];
  }
  __syncthreads();
  if (threadIdx.x < 32) {   // exclusive scan of the K counts: lane chunks, then a warp scan
    const int lane = threadIdx.x, per = (K + 31) / 32, k0 = min(lane * per, K), k1 = min(k0 + per, K);
    int sum = 0;
    for (int k = k0; k < k1; ++k) sum += cnt_k[k];
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    int run = incl - sum;
    for (int k = k0; k < k1; ++k) {
      cs[k] = run;
      run += cnt_k[k];
    }
    if (lane == 31) cs[K] = incl;
  }
  __syncthreads();
  const int total = cs[K];
  const bool staged = total <= stage_cap;
  const R cut2 = mul_rn(rc, rc);
  if (staged) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int k = warp; k < K; k += nw) {
      const int r = k / W, u = k - r * W;
      const int nby = sg.y + r / 3 - 1, nbz = sg.z + r % 3 - 1, nbx = sg.x0 - 1 + u;
      const int dy = wrap_cell(nby, d1) - nby, dz = wrap_cell(nbz, d2) - nbz;
      const int dx = wrap_cell(nbx, d0) - nbx;
      const R o0 = mul_rn(Traits<R>::dx(rp, 0), (R)dx), o1 = mul_rn(Traits<R>::dx(rp, 1), (R)dy),
              o2 = mul_rn(Traits<R>::dx(rp, 2), (R)dz);
      const int code = (dx > 0 ? 1 : (dx < 0 ? 2 : 0)) | ((dy > 0 ? 1 : (dy < 0 ? 2 : 0)) << 2) |
                       ((dz > 0 ? 1 : (dz < 0 ? 2 : 0)) << 4);
      const int c0 = cell_start[cell_k[k]], cnt = cnt_k[k], base = cs[k];
      for (int t = lane; t < cnt; t += 32) {
        const V4 pj = pos4[c0 + t];
        V4 v;
        v.x = sub_rn(pj.x, o0);
        v.y = sub_rn(pj.y, o1);
        v.z = sub_rn(pj.z, o2);
        v.w = pack_tag(v.x, ((c0 + t) << kShiftBits) | code);
        stage[base + t] = v;
      }
    }
  }
  __syncthreads();
  const int row0 = rp.cell_base + sg.y * d0 + sg.z * d0 * d1;
  const int s0 = cell_start[row0 + sg.x0], s1 = cell_start[row0 + sg.x1];
  for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
    const V4 pi = pos4[i];
    const R pix[3] = {pi.x, pi.y, pi.z};
    int ci[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      ci[d] = (int)div_rn(sub_rn(pix[d], Traits<R>::lo(rp, d)), Traits<R>::dx(rp, d));
    int idx = 0;
    if (staged && ci[1] == sg.y && ci[2] == sg.z && ci[0] >= sg.x0 && ci[0] < sg.x1) {
      const int u0 = ci[0] - sg.x0;   // staged cells u0 .. u0 + 2 of every row
      // staged x already carries the periodic shift, and a row's cells are ordered by x
      // (rows that wrap in x are walked whole: atoms outside the box, binned into the last or
      // first cell, break the order across the wrap)
      const R xm = rc + (fabs(pix[0]) + (R)2 * rc) * (R)1e-5 + (R)1e-6;
      const bool trim = trim_x && ci[0] - 1 >= 0 && ci[0] + 1 < d0;
      for (int r = 0; r < 9; ++r) {
        int t0 = cs[r * W + u0], t1 = cs[r * W + u0 + 3];
        if (trim) {
          for (int lo = t0, hi = t1; lo < hi;) {
            const int mid = (lo + hi) >> 1;
            if (stage[mid].x < pix[0] - xm) lo = t0 = mid + 1;
            else hi = mid;
          }
          for (int lo = t0, hi = t1; lo < hi;) {
            const int mid = (lo + hi) >> 1;
            if (stage[mid].x < pix[0] + xm) lo = mid + 1;
            else hi = t1 = mid;
          }
        }
#pragma unroll 4
        for (int t = t0; t < t1; ++t) {
          const V4 q = stage[t];
          const R r0 = sub_rn(q.x, pix[0]);
          const R r1 = sub_rn(q.y, pix[1]);
          const R r2 = sub_rn(q.z, pix[2]);
          const R dd = add_rn(add_rn(mul_rn(r0, r0), mul_rn(r1, r1)), mul_rn(r2, r2));
          if (inside_cut(sub_rn(cut2, dd), orig) && gt_small(dd)) {
            if (idx < cap) __stcs(nbr + (size_t)idx * stride + i, unpack_tag(q.w));
            ++idx;
          }
        }
      }
    } else {
      idx = nlist_thread<R>(i, pi, rp, pos4, cell_start, 1, rc, cap, stride, nbr, false, orig);
    }
    nlist_finish(i, idx, cap, count, max_count, status);
  }
}

// Fixed-point fractional coordinates + charge of the charged atoms (qidx: their caller ids,
// grouped per replica), the input of every k-space phase: U_d = floor(frac((x_d - lo_d)/L_d)
// * 2^32) (2^64 for FP64), so integer phases m . U mod 2^32 are exact.  Uncharged atoms add
// nothing to rho_k or the k-space force and are left out.
template <class R>
__global__ void k_frac(int nq, const int* __restrict__ qidx, const double* __restrict__ pos,
                       const double* __restrict__ charge, const int* __restrict__ rep_of,
                       const RepDev* __restrict__ reps, void* __restrict__ frac_out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nq) return;
  const int id = qidx[c];
  const RepDev& rp = reps[rep_of ? rep_of[id] : 0];
  const double q = charge[id];
  double u[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    u[d] = (pos[3 * id + d] - rp.lo_d[d]) / rp.box_d[d];
    u[d] -= floor(u[d]);
  }
  if (sizeof(R) == 4) {
    uint32_t U[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      U[d] = turn32(u[d]);
    }
    reinterpret_cast<Frac32*>(frac_out)[c] = Frac32{U[0], U[1], U[2], (float)q};
  } else {
    unsigned long long U[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      U[d] = turn64(u[d]);
    }
    reinterpret_cast<Frac64*>(frac_out)[c] = Frac64{U[0], U[1], U[2], q};
  }
}

}  // namespace rbmd
