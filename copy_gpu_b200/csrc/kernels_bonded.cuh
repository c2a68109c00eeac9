// CVFF intramolecular terms for general molecules: harmonic bonds, harmonic angles, harmonic
// dihedrals and the intramolecular Coulomb correction, FP64 in caller atom order.
//
// Layout.  The terms are packed in one atom array: bond t owns entries [2t, 2t+2), angle u the
// entries [2 nb + 3u, 2 nb + 3u + 3), dihedral v the entries [2 nb + 3 na + 4v, ... + 4).  Entry
// e is also the row of the contribution buffer rows[e][3]: k_bonded_terms (one thread per term)
// writes the force of the term on each of its atoms into its own rows, and k_bonded_gather (one
// thread per atom) sums the rows of an atom through a CSR index (rows ascending, so bonds, then
// angles, then dihedrals), which keeps the sums in a fixed order without atomics, as the
// reference's keyed ReduceByKey does (ExecutionNVT.cpp:467-706).
#pragma once
#include "common.cuh"

namespace rbmd {

struct BondedParams {
  int n;                 // atoms
  int nb, na, nd;        // bonds, angles, dihedrals
  double coul_const;     // 332.06371, the REAL-units constant hard-coded in the special Coulomb
};

// MinDistanceVec(a, b) (ExecPointLocator.h:225-260): a - b folded once per axis.
__device__ __forceinline__ void bonded_mind(const double* a, const double* b, const double* box, double* v) {
  for (int d = 0; d < 3; ++d) {
    double x = a[d] - b[d];
    if (fabs(x) > box[d] * 0.5) x -= (x > 0 ? box[d] : -box[d]);
    v[d] = x;
  }
}

__device__ __forceinline__ double bdot(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// One thread per term.  Coefficients per term: k[t], a[t] (bond r0, angle theta0 in radians,
// dihedral cos_shift = +-1) and mult[t] (dihedral multiplicity).
//  bond     ComputeBondHarmonicWorklet (MolecularWorklet.h:57-141): r = x_i - x_j (min image),
//           F_i = -2 k (d - r0)/d r, F_j = -F_i when d > 0.01; E = k (d - r0)^2;
//  angle    ComputeAngleHarmonicWorklet (MolecularWorklet.h:143-283): theta from r_ij, r_kj with
//           cos clamped to [-1, 1] and 1/sin floored at sin = 0.001; E = k (theta - theta0)^2;
//  dihedral ComputeDihedralHarmonicWorklet (MolecularWorklet.h:555-818): E = K [1 + d cos(n phi)],
//           cos(n phi) and its derivative by the angle-addition recursion over n.
__global__ void __launch_bounds__(256) k_bonded_terms(BondedParams bp, const int* __restrict__ term_atom,
                                                     const double* __restrict__ tk, const double* __restrict__ ta,
                                                     const int* __restrict__ tmult, const double* __restrict__ pos,
                                                     const int* __restrict__ rep_of, const RepDev* __restrict__ reps,
                                                     double* __restrict__ rows, double* __restrict__ eterm) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nterm = bp.nb + bp.na + bp.nd;
  if (t >= nterm) return;
  int base, na;
  if (t < bp.nb) { base = 2 * t; na = 2; }
  else if (t < bp.nb + bp.na) { base = 2 * bp.nb + 3 * (t - bp.nb); na = 3; }
  else { base = 2 * bp.nb + 3 * bp.na + 4 * (t - bp.nb - bp.na); na = 4; }
  int id[4];
  double x[4][3];
  for (int a = 0; a < na; ++a) {
    id[a] = term_atom[base + a];
    for (int d = 0; d < 3; ++d) x[a][d] = pos[3 * id[a] + d];
  }
  const RepDev& rp = reps[rep_of ? rep_of[id[0]] : 0];
  const double box[3] = {rp.box_d[0], rp.box_d[1], rp.box_d[2]};
  const double k = tk[t], a0 = ta[t];
  double f[4][3];
  double e;
  if (na == 2) {
    double r[3];
    bonded_mind(x[0], x[1], box, r);
    const double d = sqrt(bdot(r, r));
    const double dr = d - a0, rk = k * dr;
    const double fb = d > 0.01 ? -2.0 * rk / d : 0.0;
    for (int c = 0; c < 3; ++c) { f[0][c] = fb * r[c]; f[1][c] = -fb * r[c]; }
    e = rk * dr;
  } else if (na == 3) {
    double rij[3], rkj[3];
    bonded_mind(x[0], x[1], box, rij);
    bonded_mind(x[2], x[1], box, rkj);
    const double dij2 = bdot(rij, rij), dij = sqrt(dij2), dkj2 = bdot(rkj, rkj), dkj = sqrt(dkj2);
    double c = bdot(rij, rkj) / (dij * dkj);
    c = fmin(1.0, fmax(-1.0, c));
    double s = sqrt(1.0 - c * c);
    if (s < 0.001) s = 0.001;
    s = 1.0 / s;
    const double dth = acos(c) - a0, tkk = k * dth;
    const double aa = -2.0 * tkk * s, a11 = aa * c / dij2, a12 = -aa / (dij * dkj), a22 = aa * c / dkj2;
    for (int q = 0; q < 3; ++q) {
      const double fi = a11 * rij[q] + a12 * rkj[q], fk = a22 * rkj[q] + a12 * rij[q];
      f[0][q] = fi;
      f[1][q] = -fi - fk;
      f[2][q] = fk;
    }
    e = tkk * dth;
  } else {
    double vb1[3], vb2[3], vb3[3], vb2m[3];
    bonded_mind(x[0], x[1], box, vb1);
    bonded_mind(x[2], x[1], box, vb2);
    for (int d = 0; d < 3; ++d) vb2m[d] = -vb2[d];
    bonded_mind(x[3], x[2], box, vb3);
    const double ax = vb1[1] * vb2m[2] - vb1[2] * vb2m[1];
    const double ay = vb1[2] * vb2m[0] - vb1[0] * vb2m[2];
    const double az = vb1[0] * vb2m[1] - vb1[1] * vb2m[0];
    const double bx = vb3[1] * vb2m[2] - vb3[2] * vb2m[1];
    const double by = vb3[2] * vb2m[0] - vb3[0] * vb2m[2];
    const double bz = vb3[0] * vb2m[1] - vb3[1] * vb2m[0];
    const double rasq = ax * ax + ay * ay + az * az;
    const double rbsq = bx * bx + by * by + bz * bz;
    const double rg = sqrt(bdot(vb2m, vb2m));
    const double rginv = rg > 0 ? 1.0 / rg : 0.0;
    const double ra2inv = rasq > 0 ? 1.0 / rasq : 0.0;
    const double rb2inv = rbsq > 0 ? 1.0 / rbsq : 0.0;
    const double rabinv = sqrt(ra2inv * rb2inv);
    double c = (ax * bx + ay * by + az * bz) * rabinv;
    const double s = rg * rabinv * (ax * vb3[0] + ay * vb3[1] + az * vb3[2]);
    c = fmin(1.0, fmax(-1.0, c));
    const int m = tmult[t];
    const double cos_shift = a0;   // sin_shift = 0
    double p = 1.0, ddf1 = 0.0, df1 = 0.0;
    for (int i = 0; i < m; ++i) {
      ddf1 = p * c - df1 * s;
      df1 = p * s + df1 * c;
      p = ddf1;
    }
    p = p * cos_shift;
    df1 = df1 * cos_shift;
    df1 *= -m;
    p += 1.0;
    if (m == 0) { p = 1.0 + cos_shift; df1 = 0.0; }
    const double fg = bdot(vb1, vb2m), hg = bdot(vb3, vb2m);
    const double fga = fg * ra2inv * rginv, hgb = hg * rb2inv * rginv;
    const double gaa = -ra2inv * rg, gbb = rb2inv * rg;
    const double dtf[3] = {gaa * ax, gaa * ay, gaa * az};
    const double dtg[3] = {fga * ax - hgb * bx, fga * ay - hgb * by, fga * az - hgb * bz};
    const double dth[3] = {gbb * bx, gbb * by, gbb * bz};
    const double df = -k * df1;
    for (int d = 0; d < 3; ++d) {
      const double s2 = df * dtg[d];
      f[0][d] = df * dtf[d];
      f[1][d] = s2 - f[0][d];
      f[3][d] = df * dth[d];
      f[2][d] = -s2 - f[3][d];
    }
    e = k * p;
  }
  for (int a = 0; a < na; ++a)
    for (int d = 0; d < 3; ++d) rows[3 * (size_t)(base + a) + d] = f[a][d];
  eterm[t] = e;
}

// One thread per atom: the intramolecular Coulomb correction (ComputeSpecialCoulWorklet /
// ComputeSpecialCoulGeneralWorklet, RunWorklet.cpp:1386-1511: -332.06371 q_i q_j r_ij / r^3 times
// fac_ij for the listed partners j; the host lists every other member of a molecule of >= 3 atoms
// with fac 1, or with special bonds the partners whose weight w != 1 with fac = 1 - w), then the
// atom's bond, angle and dihedral rows, each group added to the force in the reference's order.
// e_sc[a] = half the correction energy of the atom's pairs.
__global__ void __launch_bounds__(256) k_bonded_gather(
    BondedParams bp, const int* __restrict__ sc_off, const int* __restrict__ sc_id, const double* __restrict__ sc_fac,
    const int* __restrict__ row_off, const int* __restrict__ row_idx, const double* __restrict__ pos,
    const double* __restrict__ charge, const int* __restrict__ rep_of, const RepDev* __restrict__ reps,
    const double* __restrict__ rows, double* __restrict__ force, double* __restrict__ e_sc) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= bp.n) return;
  double F[3] = {force[3 * a], force[3 * a + 1], force[3 * a + 2]};
  const int s0 = sc_off[a], s1 = sc_off[a + 1];
  double es = 0;
  if (s1 > s0) {
    const RepDev& rp = reps[rep_of ? rep_of[a] : 0];
    const double box[3] = {rp.box_d[0], rp.box_d[1], rp.box_d[2]};
    const double xa[3] = {pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]};
    const double qa = charge ? charge[a] : 0.0;
    double fs[3] = {0, 0, 0};
    for (int k = s0; k < s1; ++k) {
      const int j = sc_id[k];
      const double xj[3] = {pos[3 * j], pos[3 * j + 1], pos[3 * j + 2]};
      double r[3];
      bonded_mind(xa, xj, box, r);
      const double d = sqrt(bdot(r, r));
      const double qq = qa * (charge ? charge[j] : 0.0);
      const double fc = -bp.coul_const * qq / (d * d * d);
      for (int c = 0; c < 3; ++c) fs[c] += sc_fac[k] * fc * r[c];
      es += -0.5 * sc_fac[k] * bp.coul_const * qq / d;
    }
    for (int c = 0; c < 3; ++c) F[c] += fs[c];
  }
  const int r0 = row_off[a], r1 = row_off[a + 1];
  const int ang0 = 2 * bp.nb, dih0 = 2 * bp.nb + 3 * bp.na;
  int k = r0;
  for (int grp = 0; grp < 3; ++grp) {
    const int lim = grp == 0 ? ang0 : (grp == 1 ? dih0 : 0x7fffffff);
    double g[3] = {0, 0, 0};
    bool any = false;
    for (; k < r1 && row_idx[k] < lim; ++k) {
      const size_t r = (size_t)row_idx[k];
      g[0] += rows[3 * r];
      g[1] += rows[3 * r + 1];
      g[2] += rows[3 * r + 2];
      any = true;
    }
    if (any)
      for (int c = 0; c < 3; ++c) F[c] += g[c];
  }
  force[3 * a] = F[0];
  force[3 * a + 1] = F[1];
  force[3 * a + 2] = F[2];
  if (e_sc) e_sc[a] = es;
}

// Special-bond LJ weight of slot pair (i, j) inside the near passes: the partner list of atom
// ai (dedup'd, one entry per partner with the weight of its last occurrence in the reference's
// list, ComputeSpecialBondsLJWorklet RunWorklet.cpp:570-632) searched for aj; 1 when absent.
struct SpecialDev {
  const int* off;      // [n + 1] per caller atom
  const int* id;       // partner atom ids
  const float* wf;     // weights (FP32 pass)
  const double* wd;    // weights (FP64 pass)
};

template <class R> __device__ __forceinline__ R special_w(const SpecialDev& sp, int k);
template <> __device__ __forceinline__ float special_w<float>(const SpecialDev& sp, int k) { return sp.wf[k]; }
template <> __device__ __forceinline__ double special_w<double>(const SpecialDev& sp, int k) { return sp.wd[k]; }

template <class R>
__device__ __noinline__ R special_weight(const SpecialDev sp, int ai, int aj) {
  const int k1 = sp.off[ai + 1];
  for (int k = sp.off[ai]; k < k1; ++k)
    if (sp.id[k] == aj) return special_w<R>(sp, k);
  return (R)1;
}

}  // namespace rbmd
