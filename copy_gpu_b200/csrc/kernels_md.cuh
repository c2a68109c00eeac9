// kernels_md.cuh -- FP64 velocity-Verlet, temperature / thermostats, SHAKE / RATTLE for rigid
// 3-site water, and the CVFF intramolecular terms of water (bare-Coulomb removal, harmonic
// bond and angle).  All in caller atom order, FP64 (the reference is FP32 throughout).
#pragma once
#include "common.cuh"
#include "kernels_cells.cuh"

namespace rbmd {

struct MdParams {
  int n;
  double dt, fmt2v;
  int wrap_flags;      // update image flags in the drift (reference: fix_shake == "null")
  int save_old;        // keep x_old / v_old for SHAKE
  int apply_scale;     // multiply v by lambda[rep] before the first kick (deferred thermostat)
  int nh;              // Nose-Hoover variant of the kick (UpdateVelocityNoseHoover)
};

// Stage 1+2 of ExecutionNVT::Solve (rbmd/framework/run/ExecutionNVT.cpp:136-140):
// UpdateVelocityWorklet v += 0.5 F/m dt fmt2v (RunWorklet.cpp:1764-1782), then
// UpdatePosition(Flag)Worklet x += v dt with one wrap per axis (RunWorklet.cpp:1833-1877,
// ExecPointLocator.h:321-357), fused with the cell binning of the new positions (cell_of /
// cell_count non-null; with a Verlet skin the binning runs only on rebuild steps, in k_bin).
// With a skin the same pass checks the displacement since the last build and, given pos4,
// writes the slot cache of the near pass: xref + the minimum-image displacement (unwrapped, as
// k_regather does) and the charge.
template <class R>
__global__ void k_kick_drift(MdParams mp, double* __restrict__ pos, double* __restrict__ vel,
                             const double* __restrict__ force, const double* __restrict__ mass,
                             int* __restrict__ image, const int* __restrict__ rep_of,
                             const RepDev* __restrict__ reps, const double* __restrict__ lambda,
                             double* __restrict__ x_old, double* __restrict__ v_old,
                             int* __restrict__ cell_of, int* __restrict__ cell_count, uint32_t* status,
                             const double* __restrict__ xref, double half_skin2, int* __restrict__ rebuild,
                             int n_rep,
                             const int* __restrict__ atom_slot, const double* __restrict__ charge,
                             typename Traits<R>::V4* __restrict__ pos4) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= mp.n) return;
  const int r = rep_of ? rep_of[i] : 0;
  const RepDev& rp = reps[r];
  const double m = mass[i];
  const double lam = (mp.apply_scale && lambda) ? lambda[r] : 1.0;
  double x[3];
  bool bad = false;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double v = vel[3 * i + d] * lam;
    const double xo = pos[3 * i + d];
    if (mp.save_old) { x_old[3 * i + d] = xo; v_old[3 * i + d] = v; }
    v += 0.5 * force[3 * i + d] / m * mp.dt * mp.fmt2v;
    double xn = xo + v * mp.dt;
    if (xn < rp.lo_d[d]) {
      xn += rp.hi_d[d] - rp.lo_d[d];
      if (mp.wrap_flags && image) image[3 * i + d] -= 1;
    } else if (xn > rp.hi_d[d]) {
      xn -= rp.hi_d[d] - rp.lo_d[d];
      if (mp.wrap_flags && image) image[3 * i + d] += 1;
    }
    if (xn < rp.lo_d[d] || xn > rp.hi_d[d]) bad = true;
    vel[3 * i + d] = v;
    pos[3 * i + d] = xn;
    x[d] = xn;
  }
  if (bad) set_flag(status, kFlagOutOfBox);
  if (!isfinite(x[0]) || !isfinite(x[1]) || !isfinite(x[2])) set_flag(status, kFlagNonFinite);
  if (xref) {   // Verlet skin: rebuild once any atom moved more than skin/2 since the last build
    double d2 = 0, u[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double r0 = xref[3 * i + d];
      double dd = x[d] - r0;
      if (fabs(dd) > 0.5 * rp.box_d[d]) dd -= (dd > 0 ? rp.box_d[d] : -rp.box_d[d]);
      d2 += dd * dd;
      u[d] = r0 + dd;
    }
    if (d2 > half_skin2 && rebuild[r] == 0) {
      atomicExch(rebuild + r, 1);
      atomicExch(rebuild + n_rep, 1);
    }
    if (pos4) {   // on a rebuild step the cell sort overwrites the whole cache afterwards
      typename Traits<R>::V4 v;
      v.x = (R)u[0]; v.y = (R)u[1]; v.z = (R)u[2];
      v.w = (R)(charge ? charge[i] : 0.0);
      pos4[atom_slot[i]] = v;
    }
  }
  if (cell_of) {
    const int c = cell_of_pos<R>(rp, (R)x[0], (R)x[1], (R)x[2]);
    cell_of[i] = c;
    atomicAdd(&cell_count[c], 1);
  }
}

// Verlet-skin check for a force call on externally supplied positions: flag a list rebuild when
// any atom moved more than skin/2 (nearest image) from its position at the last build.
__global__ void k_skin_check(int n, const double* __restrict__ pos, const double* __restrict__ xref,
                             const int* __restrict__ rep_of, const RepDev* __restrict__ reps,
                             double half_skin2, int* __restrict__ rebuild, int n_rep) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = rep_of ? rep_of[i] : 0;
  const RepDev& rp = reps[r];
  double d2 = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double dd = pos[3 * i + d] - xref[3 * i + d];
    dd -= rp.box_d[d] * rint(dd / rp.box_d[d]);
    d2 += dd * dd;
  }
  if (!(d2 <= half_skin2) && rebuild[r] == 0) {
    atomicExch(rebuild + r, 1);
    atomicExch(rebuild + n_rep, 1);
  }
}

// Langevin thermostat force (ExecutionNVT::TempConTypeForce, rbmd/framework/run/ExecutionNVT.cpp:
// 735-747, UnderdampedLangevinWorklet, rbmd/framework/run/worklet/RunWorklet.cpp:1700-1728):
// F += -m gamma v + sqrt(2 m gamma kBT / dt) xi, added to the total force before the kicks.
// Default (physical): xi per atom and step, standard normal from Philox keyed by (seed, step,
// atom), m the atom's mass and kBT = kB T0, with the unit factors of the kick (force * fmt2v / m
// is an acceleration, m v^2 mvv2e an energy).  shared (the reference's form, compat): m = 1,
// kBT = 1 and one xi vector for all atoms and steps.
struct LangevinParams {
  int n, shared;
  double gamma, dt, kBT, fmt2v, mvv2e;
  double xi[3];
  unsigned long long seed;
};

__global__ void k_langevin(LangevinParams lp, const double* __restrict__ vel, const double* __restrict__ mass,
                           const long long* __restrict__ step, double* __restrict__ force) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= lp.n) return;
  double xi[3] = {lp.xi[0], lp.xi[1], lp.xi[2]};
  double m = 1.0, conv = 1.0, amp;
  if (lp.shared) {
    amp = sqrt(2.0 * lp.gamma * lp.kBT / lp.dt);
  } else {
    m = mass ? mass[i] : 1.0;
    conv = 1.0 / lp.fmt2v;   // force = (m / fmt2v) * acceleration
    amp = m * conv * sqrt(2.0 * lp.gamma * lp.kBT / (m * lp.mvv2e * lp.dt));
    const unsigned long long st = (unsigned long long)*step;
    uint32_t c[4] = {(uint32_t)i, 0x4c414e47u, (uint32_t)st, (uint32_t)(st >> 32)};
    philox4x32(c, (uint32_t)lp.seed, (uint32_t)(lp.seed >> 32));
    // Box-Muller on three of the four words (plus one more from a second counter)
    const double u1 = ((double)c[0] + 0.5) * (1.0 / 4294967296.0);
    const double u2 = ((double)c[1] + 0.5) * (1.0 / 4294967296.0);
    const double u3 = ((double)c[2] + 0.5) * (1.0 / 4294967296.0);
    const double u4 = ((double)c[3] + 0.5) * (1.0 / 4294967296.0);
    const double r1 = sqrt(-2.0 * log(u1)), r2 = sqrt(-2.0 * log(u3));
    xi[0] = r1 * cos(2.0 * 3.14159265358979323846 * u2);
    xi[1] = r1 * sin(2.0 * 3.14159265358979323846 * u2);
    xi[2] = r2 * cos(2.0 * 3.14159265358979323846 * u4);
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) force[3 * i + d] += -m * conv * lp.gamma * vel[3 * i + d] + amp * xi[d];
}

// Advance the device step counter the k-samplers read (end of a step's k-space chain).
__global__ void k_step_inc(long long* step) { *step += 1; }

// Open the rebuild body of a captured step (an IF conditional graph node) when some replica
// rebuilds its list this step: any = rebuild[n_replicas], raised by the drift kernel.
__global__ void k_open_rebuild(cudaGraphConditionalHandle h, const int* __restrict__ any) {
  cudaGraphSetConditional(h, *any != 0 ? 1u : 0u);
}

// Chunk of atoms inside one replica (kinetic-energy partials, ordered per replica).
struct MdChunk { int begin, end, rep, pad; };

// Stage 3 kick (+ NH variant) and per-chunk sum m v^2 (ComputerKineticEnergyWorklet,
// RunWorklet.cpp:1806-1816).  One block per chunk; deterministic block reduction.
__global__ void __launch_bounds__(256) k_kick_ke(MdParams mp, const MdChunk* __restrict__ chunks,
                                                 double* __restrict__ vel, const double* __restrict__ force,
                                                 const double* __restrict__ mass, int do_kick,
                                                 const double* __restrict__ xi_rep,
                                                 double* __restrict__ ke_partial) {
  const MdChunk ch = chunks[blockIdx.x];
  const double xi = (do_kick == 2 && xi_rep) ? xi_rep[ch.rep] : 0.0;
  double ke = 0;
  for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
    const double m = mass[i];
    double v2 = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double v = vel[3 * i + d];
      if (do_kick == 1) {
        v += 0.5 * force[3 * i + d] / m * mp.dt * mp.fmt2v;
        vel[3 * i + d] = v;
      } else if (do_kick == 2) {   // UpdateVelocityNoseHooverWorklet (RunWorklet.cpp:1784-1804)
        v += 0.5 * mp.dt * (force[3 * i + d] / m - xi * v) * mp.fmt2v;
        vel[3 * i + d] = v;
      }
      v2 += v * v;
    }
    ke += m * v2;
  }
  if (!ke_partial) return;
  __shared__ double red[8];
  for (int o = 16; o > 0; o >>= 1) ke += __shfl_xor_sync(0xffffffffu, ke, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ke;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    ke_partial[blockIdx.x] = s;
  }
}

struct ThermoParams {
  int nrep;
  int tstat;          // 0 none, 1 BERENDSEN, 2 TEMP_RESCALE, 3 NOSE_HOOVER
  double mvv2e, kB, dt, Tdamp, T0;
  int dof_mode;       // 0: 3n-3, 1: 3n-n-3 (shake), 2: 3n, 3: 3n/2 (inbuild)
};

// ExecutionNVT::ComputeTempe + UpdateVelocityByTempConType
// (rbmd/framework/run/ExecutionNVT.cpp:256-290,749-786) per replica: T from the chunk
// partials (fixed order), lambda for the deferred rescale, NH xi update.
__global__ void k_thermo(ThermoParams tp, const int* __restrict__ chunk_begin_of_rep,
                         const double* __restrict__ ke_partial, double* __restrict__ ke_out,
                         double* __restrict__ T_out, double* __restrict__ lambda,
                         double* __restrict__ xi, const RepDev* __restrict__ reps) {
  // one warp per replica, fixed-order lane sums then a butterfly: deterministic
  const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= tp.nrep) return;
  double s = 0;
  for (int c = chunk_begin_of_rep[r] + lane; c < chunk_begin_of_rep[r + 1]; c += 32) s += ke_partial[c];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane != 0) return;
  s *= tp.mvv2e;
  const double n = (double)(reps[r].atom_end - reps[r].atom_begin);
  double T;
  switch (tp.dof_mode) {
    case 1: T = 0.5 * s / ((3 * n - n - 3) * tp.kB / 2.0); break;
    case 2: T = 0.5 * s / ((3 * n) * tp.kB / 2.0); break;
    case 3: T = 0.5 * s / (3 * n / 2.0); break;
    default: T = 0.5 * s / ((3 * n - 3) * tp.kB / 2.0); break;
  }
  ke_out[r] = 0.5 * s;
  T_out[r] = T;
  double lam = 1.0;
  if (tp.tstat == 1) lam = sqrt(1.0 + (tp.dt / tp.Tdamp) * (tp.T0 / T - 1.0));
  else if (tp.tstat == 2) lam = sqrt(tp.T0 / T);
  else if (tp.tstat == 3 && xi) {
    const double tauT = 0.1 * tp.dt;
    xi[r] += 0.5 * tp.dt * (T / tp.T0 - 1.0) / tauT;
  }
  lambda[r] = lam;
}

__global__ void k_scale_vel(int n, const int* __restrict__ rep_of, const double* __restrict__ lambda,
                            double* __restrict__ vel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double l = lambda[rep_of ? rep_of[i] : 0];
  vel[3 * i] *= l;
  vel[3 * i + 1] *= l;
  vel[3 * i + 2] *= l;
}

__device__ __forceinline__ void mind(const double* a, const double* b, const double* box, double* v) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    v[d] = a[d] - b[d];
    if (fabs(v[d]) > box[d] * 0.5) v[d] -= (v[d] > 0 ? box[d] : -box[d]);
  }
}
__device__ __forceinline__ double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

struct ShakeParams {
  int n_mol;
  double dt, fmt2v, tol;
  int max_iter;
};

// SHAKE of one (H, O, H) triple: NewConstraintAWaterBondAngleWorklet
// (rbmd/framework/run/worklet/MolecularWorklet.h:2209-2469).  Unconstrained update from
// (x_old, v_old, F), 3x3 linearised lambda iteration with the quadratic terms, |dlambda| < tol,
// bounded by max_iter (status bit on non-convergence), then velocity correction and wrap.
__global__ void k_shake(ShakeParams sp, const int* __restrict__ hoh, double* __restrict__ pos,
                        double* __restrict__ vel, const double* __restrict__ x_old,
                        const double* __restrict__ v_old, const double* __restrict__ force,
                        const double* __restrict__ mass, int* __restrict__ image,
                        const int* __restrict__ rep_of, const RepDev* __restrict__ reps,
                        uint32_t* status) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= sp.n_mol) return;
  const int id[3] = {hoh[3 * w], hoh[3 * w + 1], hoh[3 * w + 2]};
  const RepDev& rp = reps[rep_of ? rep_of[id[0]] : 0];
  const double box[3] = {rp.box_d[0], rp.box_d[1], rp.box_d[2]};
  const double dt = sp.dt;
  double xo[3][3], sp_[3][3];
  for (int a = 0; a < 3; ++a)
    for (int d = 0; d < 3; ++d) {
      xo[a][d] = x_old[3 * id[a] + d];
      sp_[a][d] = xo[a][d] + v_old[3 * id[a] + d] * dt +
                  0.5 * dt * dt * force[3 * id[a] + d] / mass[id[a]] * sp.fmt2v;
    }
  const double bond1 = 1.0, bond2 = 1.0;
  const double bond12 = sqrt(bond1 * bond1 + bond2 * bond2 -
                             2.0 * bond1 * bond2 * cos((109.4700 / 180.0) * 3.14159265358979323846));
  double r01[3], r12[3], r20[3], s10[3], s21[3], s02[3];
  mind(xo[1], xo[0], box, r01);
  mind(xo[2], xo[1], box, r12);
  mind(xo[0], xo[2], box, r20);
  mind(sp_[0], sp_[1], box, s10);
  mind(sp_[1], sp_[2], box, s21);
  mind(sp_[2], sp_[0], box, s02);
  const double r01sq = dot3(r01, r01), r02sq = dot3(r20, r20), r12sq = dot3(r12, r12);
  const double s01sq = dot3(s10, s10), s02sq = dot3(s02, s02), s12sq = dot3(s21, s21);
  const double im0 = 1.0 / mass[id[0]], im1 = 1.0 / mass[id[1]], im2 = 1.0 / mass[id[2]];
  const double a11 = 2.0 * (im0 + im1) * dot3(s10, r01);
  const double a12 = -2.0 * im1 * dot3(s10, r12);
  const double a13 = -2.0 * im0 * dot3(s10, r20);
  const double a21 = -2.0 * im1 * dot3(s21, r01);
  const double a22 = 2.0 * (im1 + im2) * dot3(s21, r12);
  const double a23 = -2.0 * im2 * dot3(s21, r20);
  const double a31 = -2.0 * im0 * dot3(s02, r01);
  const double a32 = -2.0 * im2 * dot3(s02, r12);
  const double a33 = 2.0 * (im0 + im2) * dot3(s02, r20);
  const double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a11 * a23 * a32 -
                     a12 * a21 * a33 - a13 * a22 * a31;
  if (fabs(det) < 0.0001) set_flag(status, kFlagShakeSingular);
  const double di = 1.0 / det;
  const double b11 = di * (a22 * a33 - a23 * a32), b12 = -di * (a12 * a33 - a13 * a32),
               b13 = di * (a12 * a23 - a13 * a22), b21 = -di * (a21 * a33 - a23 * a31),
               b22 = di * (a11 * a33 - a13 * a31), b23 = -di * (a11 * a23 - a13 * a21),
               b31 = di * (a21 * a32 - a22 * a31), b32 = -di * (a11 * a32 - a12 * a31),
               b33 = di * (a11 * a22 - a12 * a21);
  const double r0120 = dot3(r01, r20), r0112 = dot3(r01, r12), r2012 = dot3(r20, r12);
  const double q1_0101 = (im0 + im1) * (im0 + im1) * r01sq, q1_1212 = im1 * im1 * r12sq,
               q1_2020 = im0 * im0 * r02sq, q1_0120 = -2.0 * (im0 + im1) * im0 * r0120,
               q1_0112 = -2.0 * (im0 + im1) * im1 * r0112, q1_2012 = 2.0 * im0 * im1 * r2012;
  const double q2_0101 = im1 * im1 * r01sq, q2_1212 = (im1 + im2) * (im1 + im2) * r12sq,
               q2_2020 = im2 * im2 * r02sq, q2_0120 = 2.0 * im1 * im2 * r0120,
               q2_0112 = -2.0 * (im1 + im2) * im1 * r0112, q2_2012 = -2.0 * (im1 + im2) * im2 * r2012;
  const double q3_0101 = im0 * im0 * r01sq, q3_1212 = im2 * im2 * r12sq,
               q3_2020 = (im0 + im2) * (im0 + im2) * r02sq, q3_0120 = -2.0 * (im0 + im2) * im0 * r0120,
               q3_0112 = 2.0 * im0 * im2 * r0112, q3_2012 = -2.0 * (im0 + im2) * im2 * r2012;
  double l01 = 0, l20 = 0, l12 = 0;
  int niter = 0, done = 0;
  while (!done && niter < sp.max_iter) {
    const double quad1 = q1_0101 * l01 * l01 + q1_2020 * l20 * l20 + q1_1212 * l12 * l12 +
                         q1_0120 * l01 * l20 + q1_0112 * l01 * l12 + q1_2012 * l20 * l12;
    const double quad2 = q2_0101 * l01 * l01 + q2_2020 * l20 * l20 + q2_1212 * l12 * l12 +
                         q2_0120 * l01 * l20 + q2_0112 * l01 * l12 + q2_2012 * l20 * l12;
    const double quad3 = q3_0101 * l01 * l01 + q3_2020 * l20 * l20 + q3_1212 * l12 * l12 +
                         q3_0120 * l01 * l20 + q3_0112 * l01 * l12 + q3_2012 * l20 * l12;
    const double b1 = bond1 * bond1 - s01sq - quad1;
    const double b2 = bond2 * bond2 - s12sq - quad2;
    const double b3 = bond12 * bond12 - s02sq - quad3;
    const double n01 = b11 * b1 + b12 * b2 + b13 * b3;
    const double n12 = b21 * b1 + b22 * b2 + b23 * b3;
    const double n20 = b31 * b1 + b32 * b2 + b33 * b3;
    done = 1;
    if (fabs(n01 - l01) > sp.tol) done = 0;
    if (fabs(n20 - l20) > sp.tol) done = 0;
    if (fabs(n12 - l12) > sp.tol) done = 0;
    l01 = n01; l20 = n20; l12 = n12;
    if (isnan(l01) || isnan(l20) || isnan(l12) || fabs(l01) > 1e20 || fabs(l20) > 1e20 ||
        fabs(l12) > 1e20) {
      done = 1;
      set_flag(status, kFlagNonFinite);
    }
    niter++;
  }
  if (!done) set_flag(status, kFlagShakeNoConv);
  double pc[3][3];
  for (int d = 0; d < 3; ++d) {
    pc[0][d] = l01 * r01[d] * im0 - l20 * r20[d] * im0;
    pc[1][d] = l12 * r12[d] * im1 - l01 * r01[d] * im1;
    pc[2][d] = l20 * r20[d] * im2 - l12 * r12[d] * im2;
  }
  for (int a = 0; a < 3; ++a)
    for (int d = 0; d < 3; ++d) {
      const double sv = v_old[3 * id[a] + d] + 0.5 * dt * force[3 * id[a] + d] / mass[id[a]] * sp.fmt2v;
      vel[3 * id[a] + d] = sv + pc[a][d] / dt;
      double x = sp_[a][d] + pc[a][d];
      if (x < rp.lo_d[d]) { x += rp.hi_d[d] - rp.lo_d[d]; if (image) image[3 * id[a] + d] -= 1; }
      if (x > rp.hi_d[d]) { x -= rp.hi_d[d] - rp.lo_d[d]; if (image) image[3 * id[a] + d] += 1; }
      pos[3 * id[a] + d] = x;
    }
}

// RATTLE velocity solve: NewConstraintBWaterBondAngleWorklet (MolecularWorklet.h:2471-2656).
// `vel` holds the already kicked velocities (v_old + 0.5 dt F/m fmt2v).
__global__ void k_rattle(int n_mol, const int* __restrict__ hoh, const double* __restrict__ pos,
                         double* __restrict__ vel, const double* __restrict__ mass,
                         const int* __restrict__ rep_of, const RepDev* __restrict__ reps,
                         uint32_t* status) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_mol) return;
  const int id[3] = {hoh[3 * w], hoh[3 * w + 1], hoh[3 * w + 2]};
  const RepDev& rp = reps[rep_of ? rep_of[id[0]] : 0];
  const double box[3] = {rp.box_d[0], rp.box_d[1], rp.box_d[2]};
  double x[3][3], sv[3][3];
  for (int a = 0; a < 3; ++a)
    for (int d = 0; d < 3; ++d) {
      x[a][d] = pos[3 * id[a] + d];
      sv[a][d] = vel[3 * id[a] + d];
    }
  double r01[3], r12[3], r20[3];
  mind(x[1], x[0], box, r01);
  mind(x[2], x[1], box, r12);
  mind(x[0], x[2], box, r20);
  double sv10[3], sv21[3], sv02[3];
  for (int d = 0; d < 3; ++d) {
    sv10[d] = sv[0][d] - sv[1][d];
    sv21[d] = sv[1][d] - sv[2][d];
    sv02[d] = sv[2][d] - sv[0][d];
  }
  const double im0 = 1.0 / mass[id[0]], im1 = 1.0 / mass[id[1]], im2 = 1.0 / mass[id[2]];
  double a[3][3];
  a[0][0] = (im1 + im0) * dot3(r01, r01);
  a[0][1] = -im1 * dot3(r01, r12);
  a[0][2] = (-im0) * dot3(r01, r20);
  a[1][0] = a[0][1];
  a[1][1] = (im1 + im2) * dot3(r12, r12);
  a[1][2] = -(im2)*dot3(r20, r12);
  a[2][0] = a[0][2];
  a[2][1] = a[1][2];
  a[2][2] = (im0 + im2) * dot3(r20, r20);
  const double c[3] = {-dot3(sv10, r01), -dot3(sv21, r12), -dot3(sv02, r20)};
  const double det = a[0][0] * a[1][1] * a[2][2] + a[0][1] * a[1][2] * a[2][0] +
                     a[0][2] * a[1][0] * a[2][1] - a[0][0] * a[1][2] * a[2][1] -
                     a[0][1] * a[1][0] * a[2][2] - a[0][2] * a[1][1] * a[2][0];
  if (fabs(det) < 0.0001) set_flag(status, kFlagShakeSingular);
  const double di = 1.0 / det;
  double ai[3][3];
  ai[0][0] = di * (a[1][1] * a[2][2] - a[1][2] * a[2][1]);
  ai[0][1] = -di * (a[0][1] * a[2][2] - a[0][2] * a[2][1]);
  ai[0][2] = di * (a[0][1] * a[1][2] - a[0][2] * a[1][1]);
  ai[1][0] = -di * (a[1][0] * a[2][2] - a[1][2] * a[2][0]);
  ai[1][1] = di * (a[0][0] * a[2][2] - a[0][2] * a[2][0]);
  ai[1][2] = -di * (a[0][0] * a[1][2] - a[0][2] * a[1][0]);
  ai[2][0] = di * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  ai[2][1] = -di * (a[0][0] * a[2][1] - a[0][1] * a[2][0]);
  ai[2][2] = di * (a[0][0] * a[1][1] - a[0][1] * a[1][0]);
  double l[3];
  for (int i = 0; i < 3; i++) {
    l[i] = 0;
    for (int j = 0; j < 3; j++) l[i] += ai[i][j] * c[j];
  }
  for (int d = 0; d < 3; ++d) {
    vel[3 * id[0] + d] = sv[0][d] + (l[0] * r01[d] * im0 - l[2] * r20[d] * im0);
    vel[3 * id[1] + d] = sv[1][d] + (l[1] * r12[d] * im1 - l[0] * r01[d] * im1);
    vel[3 * id[2] + d] = sv[2][d] + (l[2] * r20[d] * im2 - l[1] * r12[d] * im2);
  }
}

struct WaterParams {
  int n_mol;
  double bond_k, bond_r0, angle_k, angle_theta0_rad;
  double coul_const;   // 332.06371 (hard-coded REAL constant of ComputeSpecialCoulWorklet)
};

// CVFF extras of one water molecule, added to the force: ComputeSpecialCoulWorklet
// (RunWorklet.cpp:1386-1437, subtract bare q_i q_j r/r^3 inside the molecule),
// ComputeBondHarmonicWorklet (MolecularWorklet.h:57-141) for bonds (0,1) and (2,1),
// ComputeAngleHarmonicWorklet (MolecularWorklet.h:173-283) for angle 0-1-2.  Each atom belongs
// to one molecule, so the thread owns its three force rows (no atomics).
__global__ void k_water_extras(WaterParams wp, const int* __restrict__ hoh, const double* __restrict__ pos,
                               const double* __restrict__ charge, const int* __restrict__ rep_of,
                               const RepDev* __restrict__ reps, double* __restrict__ force,
                               double* __restrict__ e_bond, double* __restrict__ e_angle,
                               double* __restrict__ e_coul) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= wp.n_mol) return;
  const int id[3] = {hoh[3 * w], hoh[3 * w + 1], hoh[3 * w + 2]};
  const RepDev& rp = reps[rep_of ? rep_of[id[0]] : 0];
  const double box[3] = {rp.box_d[0], rp.box_d[1], rp.box_d[2]};
  double x[3][3], f[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, q[3];
  for (int a = 0; a < 3; ++a) {
    q[a] = charge ? charge[id[a]] : 0.0;
    for (int d = 0; d < 3; ++d) x[a][d] = pos[3 * id[a] + d];
  }
  double ec = 0;   // energy of the removed bare Coulomb pairs, -332.06371 q_a q_b / r per pair
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      if (a == b) continue;
      double r[3];
      mind(x[a], x[b], box, r);
      const double d = sqrt(dot3(r, r));
      const double fc = -wp.coul_const * q[a] * q[b] / (d * d * d);
      for (int k = 0; k < 3; ++k) f[a][k] += fc * r[k];
      ec += -0.5 * wp.coul_const * q[a] * q[b] / d;
    }
  double eb = 0;
  const int bonds[2][2] = {{0, 1}, {2, 1}};
  for (int bi = 0; bi < 2; ++bi) {
    const int i0 = bonds[bi][0], i1 = bonds[bi][1];
    double r[3];
    mind(x[i0], x[i1], box, r);
    const double d = sqrt(dot3(r, r));
    const double dr = d - wp.bond_r0, rk = wp.bond_k * dr;
    const double fb = d > 0.01 ? -2.0 * rk / d : 0.0;
    for (int k = 0; k < 3; ++k) { f[i0][k] += fb * r[k]; f[i1][k] -= fb * r[k]; }
    eb += rk * dr;
  }
  double rij[3], rkj[3];
  mind(x[0], x[1], box, rij);
  mind(x[2], x[1], box, rkj);
  const double dij2 = dot3(rij, rij), dij = sqrt(dij2), dkj2 = dot3(rkj, rkj), dkj = sqrt(dkj2);
  double c = dot3(rij, rkj) / (dij * dkj);
  c = fmin(1.0, fmax(-1.0, c));
  double s = sqrt(1.0 - c * c);
  if (s < 0.001) s = 0.001;
  s = 1.0 / s;
  const double dth = acos(c) - wp.angle_theta0_rad;
  const double tk = wp.angle_k * dth;
  const double aa = -2.0 * tk * s, a11 = aa * c / dij2, a12 = -aa / (dij * dkj), a22 = aa * c / dkj2;
  for (int k = 0; k < 3; ++k) {
    const double fi = a11 * rij[k] + a12 * rkj[k], fk = a22 * rkj[k] + a12 * rij[k];
    f[0][k] += fi;
    f[1][k] += -fi - fk;
    f[2][k] += fk;
  }
  for (int a = 0; a < 3; ++a)
    for (int k = 0; k < 3; ++k) force[3 * id[a] + k] += f[a][k];
  if (e_bond) e_bond[w] = eb;
  if (e_angle) e_angle[w] = tk * dth;
  if (e_coul) e_coul[w] = ec;
}

// Deterministic sum of a double array into out[0] (one block).
__global__ void __launch_bounds__(1024) k_sum(int n, const double* __restrict__ a, int stride,
                                              int offset, double* __restrict__ out) {
  __shared__ double red[32];
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += a[(size_t)i * stride + offset];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    out[0] = t;
  }
}

}  // namespace rbmd
