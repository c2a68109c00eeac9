// oracle.cpp -- CPU restatement of RBMD's per-timestep force path.  TEST INFRASTRUCTURE ONLY.
//
// This file is the checker for the B200 library: only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference arm of bench.py load it.  Nothing in copy_gpu_b200/ links or calls it.
//
// Every routine is templated on Real: Real=float reproduces the reference's FP32 semantics
// (rbmd/framework/Types.h:48, Real = vtkm::FloatDefault = float; mixed float/double literals are
// kept as the reference writes them), Real=double is the FP64 reference answer.  Build with
// -ffp-contract=off so that products and sums round exactly as written.
//
// Parity status: the reference cannot be built here (VTK-m 1.9 is not vendored), so outputs are
// anchored on the reference's own data (ERF table, funcfl files) and on analytic known answers
// (Madelung constant, Newton's third law, finite differences).  See tests/golden/.
#include <cmath>
#include <math.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <string>
#include <fstream>
#include <sstream>
#include <algorithm>
#include <limits>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11).  The same counter RNG is implemented in the CUDA library; it replaces the
// reference's std::mt19937(std::random_device{}()) per draw (rbmd/framework/math/Utiles.h:32-39).
// ------------------------------------------------------------------------------------------
struct U4 { uint32_t v[4]; };

inline U4 philox(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)M0 * c.v[0];
    uint64_t p1 = (uint64_t)M1 * c.v[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    U4 n;
    n.v[0] = hi1 ^ c.v[1] ^ k0;
    n.v[1] = lo1;
    n.v[2] = hi0 ^ c.v[3] ^ k1;
    n.v[3] = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

inline double u01(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

// ------------------------------------------------------------------------------------------
// Cells: ContPointLocator::SetRange/SetCutOff/SetRs + Build + BinPointsWorklet
// (rbmd/framework/locator/ContPointLocator.h:44-73, ContPointLocator.cxx:38-92).
// ------------------------------------------------------------------------------------------
template <class Real>
struct Grid {
  Real lo[3], hi[3], dx[3], box[3];
  int dims[3];
  int num_cycles;
};

template <class Real>
Grid<Real> make_grid(const double* lo, const double* hi, double cutoff, double rs) {
  Grid<Real> g;
  Real rc = (Real)cutoff, r_s = (Real)rs;
  g.num_cycles = (int)std::ceil(rc / r_s);
  for (int d = 0; d < 3; ++d) {
    g.lo[d] = (Real)lo[d];
    g.hi[d] = (Real)hi[d];
    Real cell = rc / (Real)g.num_cycles;
    Real span = g.hi[d] - g.lo[d];
    g.dims[d] = (int)(span / cell);               // Vec3f -> Id3 conversion truncates
    if (g.dims[d] < 1) g.dims[d] = 1;
    g.dx[d] = span / (Real)g.dims[d];             // _dxdydz = (max - min) / dims
    g.box[d] = span;                              // PARA_BOX = hi - lo
  }
  return g;
}

template <class Real>
inline int bin_clamped(const Grid<Real>& g, const Real* p, int* ijk) {
  for (int d = 0; d < 3; ++d) {
    int c = (int)((p[d] - g.lo[d]) / g.dx[d]);   // BinPointsWorklet: trunc, then clamp
    c = std::max(c, 0);
    c = std::min(c, g.dims[d] - 1);
    ijk[d] = c;
  }
  return ijk[0] + ijk[1] * g.dims[0] + ijk[2] * g.dims[0] * g.dims[1];
}

template <class Real>
struct Cells {
  std::vector<int> point_ids;   // sorted by (cell, id)
  std::vector<int> lower, upper;
};

template <class Real>
Cells<Real> build_cells(const Grid<Real>& g, int64_t n, const Real* pos) {
  int ncell = g.dims[0] * g.dims[1] * g.dims[2];
  std::vector<int> key(n);
  for (int64_t i = 0; i < n; ++i) {
    int ijk[3];
    key[i] = bin_clamped(g, pos + 3 * i, ijk);
  }
  Cells<Real> c;
  c.point_ids.resize(n);
  for (int64_t i = 0; i < n; ++i) c.point_ids[i] = (int)i;
  std::stable_sort(c.point_ids.begin(), c.point_ids.end(),
                   [&](int a, int b) { return key[a] < key[b]; });
  c.lower.assign(ncell, 0);
  c.upper.assign(ncell, 0);
  // LowerBounds / UpperBounds of each cell id over the sorted keys
  int64_t s = 0;
  for (int cell = 0; cell < ncell; ++cell) {
    while (s < n && key[c.point_ids[s]] < cell) ++s;
    c.lower[cell] = (int)s;
    int64_t e = s;
    while (e < n && key[c.point_ids[e]] == cell) ++e;
    c.upper[cell] = (int)e;
    s = e;
  }
  return c;
}

// ------------------------------------------------------------------------------------------
// Full Verlet list: ComputeNeighboursWorklet (rbmd/framework/run/worklet/RunWorklet.cpp:40-96)
// with ExecPointLocator::InWhichCell / PeriodicIndexOffset / PeriodicCoordOffset
// (rbmd/framework/locator/ExecPointLocator.h:271-319).  Stencil order: x offset outermost,
// z innermost; points of a cell in sorted order.  shift code per neighbour: 2 bits per axis,
// 0 = no wrap, 1 = cell index wrapped upward (offset +dims), 2 = wrapped downward (-dims).
// ------------------------------------------------------------------------------------------
template <class Real>
// orig: the neighbour type "ORIGINAL" walks the same 27 cells on the fly
// (ExecPointLocator::ExecuteOnNeighbor, rbmd/framework/locator/ExecPointLocator.h:99-124) and
// leaves the cutoff to the force function (dis_2 < cut_off_2 && dis_2 > 0.0001,
// rbmd/framework/forceFunction/ExecForceFunction.h:74-96): the same pairs as the list but for
// the thin shell rc^2 - 1e-4 <= d^2 < rc^2, which the list predicate drops.
void neighbor_list(const Grid<Real>& g, const Cells<Real>& c, int64_t n, const Real* pos,
                   double cutoff, int64_t cap, int32_t* counts, int32_t* ids, int32_t* codes,
                   int orig = 0) {
  const Real rc = (Real)cutoff;
  const int nc = g.num_cycles;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t a = 0; a < n; ++a) {
    const Real* pi = pos + 3 * a;
    int ci[3];
    for (int d = 0; d < 3; ++d) ci[d] = (int)((pi[d] - g.lo[d]) / g.dx[d]);  // InWhichCell (no clamp)
    int64_t index = 0;
    for (int i = -nc; i <= nc; ++i)
      for (int j = -nc; j <= nc; ++j)
        for (int k = -nc; k <= nc; ++k) {
          int nb[3] = {ci[0] + i, ci[1] + j, ci[2] + k};
          int w[3];
          Real off[3];
          int code = 0;
          for (int d = 0; d < 3; ++d) {
            w[d] = (nb[d] + g.dims[d]) % g.dims[d];
            int delta = w[d] - nb[d];
            off[d] = g.dx[d] * (Real)delta;       // PeriodicCoordOffset
            int cd = delta > 0 ? 1 : (delta < 0 ? 2 : 0);
            code |= cd << (2 * d);
          }
          int cell = w[0] + w[1] * g.dims[0] + w[2] * g.dims[0] * g.dims[1];
          for (int s = c.lower[cell]; s < c.upper[cell]; ++s) {
            int jd = c.point_ids[s];
            const Real* pj = pos + 3 * jd;
            Real r0 = (pj[0] - off[0]) - pi[0];
            Real r1 = (pj[1] - off[1]) - pi[1];
            Real r2 = (pj[2] - off[2]) - pi[2];
            const Real dis_2 = r0 * r0 + r1 * r1 + r2 * r2;
            const Real cut_2 = rc * rc;
            const bool inside = orig ? dis_2 < cut_2 : (double)(cut_2 - dis_2) > 0.0001;
            if (inside && (double)dis_2 > 0.0001) {
              if (index < cap) {
                ids[a * cap + index] = jd;
                if (codes) codes[a * cap + index] = code;
              }
              ++index;
            }
          }
        }
    counts[a] = (int32_t)index;
  }
}

template <class Real>
inline void shift_offset(const Grid<Real>& g, int code, Real* off) {
  for (int d = 0; d < 3; ++d) {
    int cd = (code >> (2 * d)) & 3;
    int delta = cd == 1 ? g.dims[d] : (cd == 2 ? -g.dims[d] : 0);
    off[d] = g.dx[d] * (Real)delta;
  }
}

// MinDistanceVec (rbmd/framework/locator/ExecPointLocator.h:225-260)
template <class Real>
inline void min_dist(const Real* p1, const Real* p2, const Real* box, Real* v) {
  for (int d = 0; d < 3; ++d) {
    v[d] = p1[d] - p2[d];
    if ((double)std::fabs(v[d]) > (double)box[d] * 0.5) v[d] -= (v[d] > 0 ? box[d] : -box[d]);
  }
}

// ExecForceFunction::ComputeLJForce (rbmd/framework/forceFunction/ExecForceFunction.h:74-96)
template <class Real>
inline void lj_force(const Real* r, Real eps_i, Real eps_j, Real sig_i, Real sig_j, Real rc,
                     Real* f) {
  const Real small_value = (Real)0.0001;
  f[0] = f[1] = f[2] = 0;
  const Real dis_2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  const Real cut_2 = rc * rc;
  if (dis_2 < cut_2 && dis_2 > small_value) {
    Real sigma_ij = (sig_i + sig_j) / 2;
    Real s6 = sigma_ij * sigma_ij * sigma_ij * sigma_ij * sigma_ij * sigma_ij;
    Real d6 = dis_2 * dis_2 * dis_2;
    Real sd6 = s6 / d6;
    Real scal = (Real)(-24) * (Real)std::sqrt(eps_i * eps_j) * (((Real)2 * sd6 - (Real)1) * sd6) / dis_2;
    f[0] = scal * r[0];
    f[1] = scal * r[1];
    f[2] = scal * r[2];
  }
}

template <class Real> inline Real erf_r(Real x);
template <> inline float erf_r<float>(float x) { return std::erf(x); }
template <> inline double erf_r<double>(double x) { return std::erf(x); }

// ExecForceFunction::Gnear (rbmd/framework/forceFunction/ExecForceFunction.h:217-224)
template <class Real>
inline Real gnear(Real alpha, Real dis) {
  Real erfcx = (Real)std::sqrt(alpha) * dis;
  Real expx = -alpha * dis * dis;
  // (1.0 - ERF(x)) / (dis*dis) is evaluated in double in the reference (1.0 is a double literal)
  double t1 = (1.0 - (double)erf_r<Real>(erfcx)) / (double)(dis * dis);
  Real pif = (Real)3.14159265358979323846;
  Real t2 = (Real)2 * (Real)std::sqrt(alpha) * (Real)std::exp(expx) / ((Real)std::sqrt(pif) * dis);
  return (Real)(t1 + (double)t2);
}

template <class Real>
inline Real gnear_fp64(Real alpha, Real dis) {
  double a = alpha, d = dis;
  return (Real)(std::erfc(std::sqrt(a) * d) / (d * d) +
                2.0 * std::sqrt(a) * std::exp(-a * d * d) / (std::sqrt(M_PI) * d));
}

// ComputeNearEnergyForce (rbmd/framework/forceFunction/ExecForceFunction.h:125-140)
template <class Real>
inline void coul_force(const Real* pi, const Real* pj, Real qi, Real qj, Real rc, Real alpha,
                       Real* f) {
  const Real small_value = (Real)0.01;
  f[0] = f[1] = f[2] = 0;
  Real r[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
  Real dis = (Real)std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  if (dis < rc && dis > small_value) {
    Real g = sizeof(Real) == 4 ? gnear<Real>(alpha, dis) : gnear_fp64<Real>(alpha, dis);
    Real s = -qi * qj * g;
    f[0] = s * r[0] / dis;
    f[1] = s * r[1] / dis;
    f[2] = s * r[2] / dis;
  }
}

// ------------------------------------------------------------------------------------------
// RBE sampler: RBEPSAMPLE::Fetch_P_Sample / MH_Algorithm / Distribution_P / Distribution_q /
// FetchSample_1D (rbmd/framework/model/RBEPSample.h:30-175), called from
// ExecutionNVT::PreForce (rbmd/framework/run/ExecutionNVT.cpp:331-353) with mu = 0 and
// sigma_d = sqrt(alpha/2) * L_d / pi.  Randomness: Philox counter (seed, step, replica, axis,
// draw); U1 < 1e-6 is re-drawn from the fourth Philox word (the reference loops on U1).
// Acceptance ratio and Box-Muller are evaluated in double; Distribution_q is tabulated.
// ------------------------------------------------------------------------------------------
struct SamplerTables {
  double sigma[3];
  int qmax;                    // tables cover |m| <= qmax
  std::vector<double> G[3];    // G[m] = exp(-c m^2) / q(m), c = pi^2 / (alpha L^2)
};

// Distribution_P / Distribution_q (rbmd/framework/model/RBEPSample.h:86-114): the MH ratio
// (P(m')/P(m)) (q(m)/q(m')) equals G(m')/G(m) with G = P/q up to the constant 1/H, so
// u <= min(1, ratio) is evaluated as u * G(m) <= G(m').  Tables in FP64; G = +inf where q
// underflows (such a proposal is always accepted, as the ratio is infinite).
SamplerTables sampler_tables(double alpha, const double* L) {
  SamplerTables t;
  t.qmax = 0;
  for (int d = 0; d < 3; ++d) {
    t.sigma[d] = std::sqrt(alpha / 2.0) * L[d] / M_PI;
    t.qmax = std::max(t.qmax, (int)std::ceil(14.0 * t.sigma[d]) + 8);
  }
  for (int d = 0; d < 3; ++d) {
    const double s = std::sqrt(alpha * L[d] * L[d] / (M_PI * M_PI));
    const double c = M_PI * M_PI / (alpha * L[d] * L[d]);
    t.G[d].resize(t.qmax + 1);
    for (int m = 0; m <= t.qmax; ++m) {
      const double q = m == 0 ? std::erf(0.5 / s)
                              : (std::erf((0.5 + m) / s) - std::erf((m - 0.5) / s)) / 2.0;
      t.G[d][m] = q > 0 ? std::exp(-c * (double)m * (double)m) / q : INFINITY;
    }
  }
  return t;
}

// trace (nullable): the uniforms in the order RBEPSAMPLE consumes them (FetchSample_1D's U1,
// re-drawn while below 1e-6, then U2; MH_Algorithm's acceptance u after them), so that the
// reference's sampler can be run on the same draws.
inline double gauss_draw(uint32_t k0, uint32_t k1, int64_t step, int rep, int axis, int64_t draw,
                         double* ua, std::vector<double>* trace = nullptr, bool mh = false) {
  U4 c;
  c.v[0] = (uint32_t)draw;
  c.v[1] = (uint32_t)axis | ((uint32_t)rep << 2);
  c.v[2] = (uint32_t)(uint64_t)step;
  c.v[3] = (uint32_t)((uint64_t)step >> 32);
  U4 r = philox(c, k0, k1);
  double U1 = u01(r.v[0]);
  if (trace) trace->push_back(U1);
  if (U1 < 1e-6) {
    U1 = u01(r.v[3]);
    if (trace) trace->push_back(U1);
  }
  if (U1 < 1e-6) {
    U1 = 1e-6;
    if (trace) trace->push_back(U1);
  }
  double U2 = u01(r.v[1]);
  *ua = u01(r.v[2]);
  if (trace) {
    trace->push_back(U2);
    if (mh) trace->push_back(*ua);
  }
  return std::sqrt(-2.0 * std::log(U1)) * std::cos(2.0 * M_PI * U2);
}

inline double gval(const SamplerTables& t, int d, int m) {
  m = std::abs(m);
  return m <= t.qmax ? t.G[d][m] : INFINITY;
}

void rbe_sample(const SamplerTables& t, uint64_t seed, int64_t step, int rep, int P, int32_t* out,
                std::vector<double>* trace = nullptr) {
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  int64_t draw = 0;
  int X0[3];
  for (;;) {
    for (int d = 0; d < 3; ++d) {
      double ua;
      double g = gauss_draw(k0, k1, step, rep, d, draw, &ua, trace, false);
      X0[d] = (int)std::round(t.sigma[d] * g);
    }
    ++draw;
    if (!(X0[0] == 0 && X0[1] == 0 && X0[2] == 0)) break;
  }
  out[0] = X0[0]; out[1] = X0[1]; out[2] = X0[2];
  int i = 1;
  while (i < P) {
    int X1[3];
    for (int d = 0; d < 3; ++d) {
      double ua;
      double g = gauss_draw(k0, k1, step, rep, d, draw, &ua, trace, true);
      int mw = (int)std::round(t.sigma[d] * g);
      X1[d] = (ua * gval(t, d, X0[d]) <= gval(t, d, mw)) ? mw : X0[d];
    }
    ++draw;
    X0[0] = X1[0]; X0[1] = X1[1]; X0[2] = X1[2];
    if (X1[0] == 0 && X1[1] == 0 && X1[2] == 0) continue;
    out[3 * i + 0] = X1[0]; out[3 * i + 1] = X1[1]; out[3 * i + 2] = X1[2];
    ++i;
  }
}

// RBE normaliser S = prod_d H_d - 1 (ExecForceFunction::Compute_S/Compute_H,
// rbmd/framework/forceFunction/ExecForceFunction.h:266-294)
template <class Real>
Real compute_S(Real alpha, const Real* box) {
  Real H[3] = {0, 0, 0};
  for (int i = 0; i < 3; ++i) {
    const Real factor = -(alpha * box[i] * box[i]);
    for (int m = -10; m <= 10; m++) {
      Real expx = (Real)(m * m) * factor;
      H[i] += (Real)std::exp(expx);
    }
    H[i] *= (Real)std::sqrt(-(double)factor / M_PI);
  }
  Real f3 = H[0] * H[1] * H[2];
  return f3 - (Real)1;
}

}  // namespace

// ==========================================================================================
// extern "C" surface (ctypes)
// ==========================================================================================
#define EXPORT extern "C" __attribute__((visibility("default")))

template <class Real>
static int neighbors_impl(int64_t n, const Real* pos, const double* lo, const double* hi,
                          double cutoff, double rs, int64_t cap, int32_t* counts, int32_t* ids,
                          int32_t* codes, int32_t* dims_out, int orig) {
  Grid<Real> g = make_grid<Real>(lo, hi, cutoff, rs);
  Cells<Real> c = build_cells(g, n, pos);
  neighbor_list(g, c, n, pos, cutoff, cap, counts, ids, codes, orig);
  if (dims_out) for (int d = 0; d < 3; ++d) dims_out[d] = g.dims[d];
  int64_t mx = 0;
  for (int64_t i = 0; i < n; ++i) mx = std::max<int64_t>(mx, counts[i]);
  return mx > cap ? 1 : 0;
}

EXPORT int oracle_neighbors_f32(int64_t n, const float* pos, const double* lo, const double* hi,
                                double cutoff, double rs, int64_t cap, int32_t* counts,
                                int32_t* ids, int32_t* codes, int32_t* dims, int orig) {
  return neighbors_impl<float>(n, pos, lo, hi, cutoff, rs, cap, counts, ids, codes, dims, orig);
}
EXPORT int oracle_neighbors_f64(int64_t n, const double* pos, const double* lo, const double* hi,
                                double cutoff, double rs, int64_t cap, int32_t* counts,
                                int32_t* ids, int32_t* codes, int32_t* dims, int orig) {
  return neighbors_impl<double>(n, pos, lo, hi, cutoff, rs, cap, counts, ids, codes, dims, orig);
}

EXPORT void oracle_cells_f32(int64_t n, const float* pos, const double* lo, const double* hi,
                             double cutoff, double rs, int32_t* dims, int32_t* point_ids,
                             int32_t* lower, int32_t* upper) {
  Grid<float> g = make_grid<float>(lo, hi, cutoff, rs);
  Cells<float> c = build_cells(g, n, pos);
  for (int d = 0; d < 3; ++d) dims[d] = g.dims[d];
  if (point_ids) std::copy(c.point_ids.begin(), c.point_ids.end(), point_ids);
  if (lower) std::copy(c.lower.begin(), c.lower.end(), lower);
  if (upper) std::copy(c.upper.begin(), c.upper.end(), upper);
}

// Special-bond weight of pair (i, j): the LJ pair loops of ComputeSpecialBondsLJWorklet and
// ComputeNearForceRBLERFSpecialBondsWorklet (RunWorklet.cpp:570-632, 816-933) scan i's whole
// special list and keep the weight of the LAST entry whose id is j; 1 when j is absent.
static double special_weight(const int64_t* off, const int32_t* ids, const double* w, int64_t i, int64_t j) {
  double r = 1.0;
  for (int64_t k = off[i]; k < off[i + 1]; ++k)
    if (ids[k] == j) r = w[k];
  return r;
}

// Near force over a full list: LJ (ComputeLJForceVerletWorklet, RunWorklet.cpp:239-303) and,
// when with_coul, the Coulomb term of ComputeNearForceVerletWorklet (RunWorklet.cpp:170-237)
// scaled by coul_scale (1.0 reproduces the reference's missing qqr2e; qqr2e gives the
// physical force).  sum_mode 0: accumulate in Real in list order (reference semantics);
// 1: accumulate the Real pair terms in double.
template <class Real>
static void near_impl(int64_t n, const Real* pos, const double* lo, const double* hi,
                      double cutoff, const int32_t* type, const int32_t* mol, const double* charge,
                      int ntypes, const double* eps, const double* sig, int64_t cap,
                      const int32_t* counts, const int32_t* ids, const int32_t* codes,
                      int with_lj, int with_coul, double alpha, double coul_scale, int sum_mode,
                      double* force_out, const int64_t* sp_off = nullptr, const int32_t* sp_ids = nullptr,
                      const double* sp_w = nullptr) {
  Grid<Real> g = make_grid<Real>(lo, hi, cutoff, cutoff);
  const Real rc = (Real)cutoff, a = (Real)alpha;
  (void)ntypes;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    const Real* pi = pos + 3 * i;
    int ti = type ? type[i] : 0;
    int64_t mi = mol ? mol[i] : i;
    Real eps_i = (Real)eps[ti], sig_i = (Real)sig[ti];
    Real qi = charge ? (Real)charge[i] : (Real)0;
    Real lj[3] = {0, 0, 0}, el[3] = {0, 0, 0};
    double ljd[3] = {0, 0, 0}, eld[3] = {0, 0, 0};
    for (int32_t p = 0; p < counts[i]; ++p) {
      int j = ids[i * cap + p];
      Real off[3];
      shift_offset(g, codes[i * cap + p], off);
      Real pj[3] = {pos[3 * j] - off[0], pos[3 * j + 1] - off[1], pos[3 * j + 2] - off[2]};
      int tj = type ? type[j] : 0;
      int64_t mj = mol ? mol[j] : j;
      if (with_coul) {
        Real f[3];
        Real qj = charge ? (Real)charge[j] : (Real)0;
        coul_force(pi, pj, qi, qj, rc, a, f);
        for (int d = 0; d < 3; ++d) {
          Real fs = f[d] * (Real)coul_scale;
          if (sum_mode == 0) el[d] += fs; else eld[d] += (double)fs;
        }
      }
      if (!with_lj || (!sp_off && mi == mj)) continue;
      Real r[3];
      min_dist(pj, pi, g.box, r);
      Real f[3];
      lj_force(r, eps_i, (Real)eps[tj], sig_i, (Real)sig[tj], rc, f);
      if (sp_off) {
        const Real w = (Real)special_weight(sp_off, sp_ids, sp_w, i, j);
        for (int d = 0; d < 3; ++d) f[d] = w * f[d];
      }
      for (int d = 0; d < 3; ++d) {
        if (sum_mode == 0) lj[d] += f[d]; else ljd[d] += (double)f[d];
      }
    }
    for (int d = 0; d < 3; ++d)
      force_out[3 * i + d] = sum_mode == 0 ? (double)(lj[d] + el[d]) : ljd[d] + eld[d];
  }
}

EXPORT void oracle_near_f32(int64_t n, const float* pos, const double* lo, const double* hi,
                            double cutoff, const int32_t* type, const int32_t* mol,
                            const double* charge, int ntypes, const double* eps, const double* sig,
                            int64_t cap, const int32_t* counts, const int32_t* ids,
                            const int32_t* codes, int with_lj, int with_coul, double alpha,
                            double coul_scale, int sum_mode, double* force_out) {
  near_impl<float>(n, pos, lo, hi, cutoff, type, mol, charge, ntypes, eps, sig, cap, counts, ids,
                   codes, with_lj, with_coul, alpha, coul_scale, sum_mode, force_out);
}
// The same with special-bond LJ weights (no same-molecule exclusion): sp_off[n+1], sp_ids,
// sp_w are the per-atom special lists of ModelFileInitCondition::SetSpecialBonds.
EXPORT void oracle_near_sp_f32(int64_t n, const float* pos, const double* lo, const double* hi,
                               double cutoff, const int32_t* type, const double* charge, int ntypes,
                               const double* eps, const double* sig, int64_t cap, const int32_t* counts,
                               const int32_t* ids, const int32_t* codes, int with_coul, double alpha,
                               double coul_scale, const int64_t* sp_off, const int32_t* sp_ids,
                               const double* sp_w, double* force_out) {
  near_impl<float>(n, pos, lo, hi, cutoff, type, nullptr, charge, ntypes, eps, sig, cap, counts, ids,
                   codes, 1, with_coul, alpha, coul_scale, 1, force_out, sp_off, sp_ids, sp_w);
}
EXPORT void oracle_near_sp_f64(int64_t n, const double* pos, const double* lo, const double* hi,
                               double cutoff, const int32_t* type, const double* charge, int ntypes,
                               const double* eps, const double* sig, int64_t cap, const int32_t* counts,
                               const int32_t* ids, const int32_t* codes, int with_coul, double alpha,
                               double coul_scale, const int64_t* sp_off, const int32_t* sp_ids,
                               const double* sp_w, double* force_out) {
  near_impl<double>(n, pos, lo, hi, cutoff, type, nullptr, charge, ntypes, eps, sig, cap, counts, ids,
                    codes, 1, with_coul, alpha, coul_scale, 1, force_out, sp_off, sp_ids, sp_w);
}
EXPORT void oracle_near_f64(int64_t n, const double* pos, const double* lo, const double* hi,
                            double cutoff, const int32_t* type, const int32_t* mol,
                            const double* charge, int ntypes, const double* eps, const double* sig,
                            int64_t cap, const int32_t* counts, const int32_t* ids,
                            const int32_t* codes, int with_lj, int with_coul, double alpha,
                            double coul_scale, int sum_mode, double* force_out) {
  near_impl<double>(n, pos, lo, hi, cutoff, type, mol, charge, ntypes, eps, sig, cap, counts, ids,
                    codes, with_lj, with_coul, alpha, coul_scale, sum_mode, force_out);
}

// The same draw, also returning the uniforms it used in RBEPSAMPLE's consumption order
// (trace[cap]); returns their number (the trace is cut at cap).
EXPORT int64_t oracle_rbe_sample_trace(double alpha, const double* L, uint64_t seed, int64_t step, int rep,
                                       int P, int32_t* m_out, double* trace, int64_t cap) {
  SamplerTables t = sampler_tables(alpha, L);
  std::vector<double> tr;
  rbe_sample(t, seed, step, rep, P, m_out, &tr);
  for (int64_t i = 0; i < (int64_t)tr.size() && i < cap; ++i) trace[i] = tr[i];
  return (int64_t)tr.size();
}

// RBE k-sampler (see rbe_sample above).
EXPORT void oracle_rbe_sample(double alpha, const double* L, uint64_t seed, int64_t step, int rep,
                              int P, int32_t* m_out) {
  SamplerTables t = sampler_tables(alpha, L);
  rbe_sample(t, seed, step, rep, P, m_out);
}

EXPORT double oracle_rbe_S_f32(double alpha, const double* box) {
  float b[3] = {(float)box[0], (float)box[1], (float)box[2]};
  return compute_S<float>((float)alpha, b);
}
EXPORT double oracle_rbe_S_f64(double alpha, const double* box) {
  return compute_S<double>(alpha, box);
}

// Structure factors rho_l = sum_j q_j (cos k_l.r_j, sin k_l.r_j), k = 2 pi m / L:
// ComputePnumberChargeStructureFactorWorklet + ReduceByKey (RunWorklet.cpp:1616-1677,
// ExecutionMD.cpp:412-448).  origin: per-axis coordinate subtracted before the phase
// (0 = the reference's absolute coordinates).  Terms in Real, sums in double.
template <class Real>
static void rhok_impl(int64_t n, const Real* pos, const double* charge, const double* box,
                      const double* origin, int P, const int32_t* m, double* rho) {
  const double twopi = 2.0 * M_PI;
  std::vector<Real> kx(P), ky(P), kz(P);
  for (int l = 0; l < P; ++l) {
    kx[l] = (Real)(twopi * (Real)m[3 * l] / (Real)box[0]);
    ky[l] = (Real)(twopi * (Real)m[3 * l + 1] / (Real)box[1]);
    kz[l] = (Real)(twopi * (Real)m[3 * l + 2] / (Real)box[2]);
  }
#pragma omp parallel for schedule(static)
  for (int l = 0; l < P; ++l) {
    double re = 0, im = 0;
    for (int64_t j = 0; j < n; ++j) {
      Real x = pos[3 * j] - (Real)origin[0], y = pos[3 * j + 1] - (Real)origin[1],
           z = pos[3 * j + 2] - (Real)origin[2];
      Real ph = kx[l] * x + ky[l] * y + kz[l] * z;
      Real q = (Real)charge[j];
      re += (double)(q * (Real)std::cos(ph));
      im += (double)(q * (Real)std::sin(ph));
    }
    rho[2 * l] = re;
    rho[2 * l + 1] = im;
  }
}

EXPORT void oracle_rhok_f32(int64_t n, const float* pos, const double* charge, const double* box,
                            const double* origin, int P, const int32_t* m, double* rho) {
  rhok_impl<float>(n, pos, charge, box, origin, P, m, rho);
}
EXPORT void oracle_rhok_f64(int64_t n, const double* pos, const double* charge, const double* box,
                            const double* origin, int P, const int32_t* m, double* rho) {
  rhok_impl<double>(n, pos, charge, box, origin, P, m, rho);
}

// RBE force: ComputeNewRBEForceWorklet + ComputeRBEForceSum + ComputeRBEForce
// (RunWorklet.cpp:1508-1548, ExecForceFunction.h:247-264), times qqr2e (UnitRescaleWorklet in
// ExecutionNVT::EleNewForce, rbmd/framework/run/ExecutionNVT.cpp:717-733).  weights (nullable)
// multiply each sample's term (importance weights of a non-Gaussian proposal).
template <class Real>
static void rbe_force_impl(int64_t n, const Real* pos, const double* charge, const double* box,
                           const double* origin, double alpha, double qqr2e, int P,
                           const int32_t* m, const double* rho, const double* weights,
                           double S_override, double* force_out) {
  const double twopi = 2.0 * M_PI;
  Real b[3] = {(Real)box[0], (Real)box[1], (Real)box[2]};
  Real volume = b[0] * b[1] * b[2];
  Real S = S_override > 0 ? (Real)S_override : compute_S<Real>((Real)alpha, b);
  std::vector<Real> kx(P), ky(P), kz(P), k2(P);
  for (int l = 0; l < P; ++l) {
    kx[l] = (Real)(twopi * (Real)m[3 * l] / b[0]);
    ky[l] = (Real)(twopi * (Real)m[3 * l + 1] / b[1]);
    kz[l] = (Real)(twopi * (Real)m[3 * l + 2] / b[2]);
    k2[l] = kx[l] * kx[l] + ky[l] * ky[l] + kz[l] * kz[l];
  }
  const Real fourpi = (Real)(4.0 * M_PI);
  if constexpr (sizeof(Real) == 4) {
    // The reference's FP32 operation order: per k, factor_a = (float)((-4 pi q) k_d) in double
    // (a Float64 scalar times a Vec3f), term = (factor_a / (V |k|^2)) * (cos(k.r) Im rho -
    // sin(k.r) Re rho), summed over k in float, then times S and divided by P in double
    // (ComputeRBEForceSum / ComputeRBEForce, ExecForceFunction.h:247-264).
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      const float x = pos[3 * i] - (float)origin[0], y = pos[3 * i + 1] - (float)origin[1],
                  z = pos[3 * i + 2] - (float)origin[2];
      const double a4 = -4.0 * M_PI * (double)(float)charge[i];
      float f[3] = {0, 0, 0};
      for (int l = 0; l < P; ++l) {
        const float k[3] = {kx[l], ky[l], kz[l]};
        const float ph = k[0] * x + k[1] * y + k[2] * z;
        const float fb = std::cos(ph) * (float)rho[2 * l + 1];
        const float fc = std::sin(ph) * (float)rho[2 * l];
        const float den = volume * k2[l];
        const float w = weights ? (float)weights[l] : 1.0f;
        for (int d = 0; d < 3; ++d) {
          const float fa = (float)(a4 * (double)k[d]);
          float t = fa / den * (fb - fc);
          if (weights) t *= w;
          f[d] += t;
        }
      }
      for (int d = 0; d < 3; ++d)
        force_out[3 * i + d] = (double)(float)((double)(f[d] * S) / (double)P) * qqr2e;
    }
    return;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    Real x = pos[3 * i] - (Real)origin[0], y = pos[3 * i + 1] - (Real)origin[1],
         z = pos[3 * i + 2] - (Real)origin[2];
    Real qi = (Real)charge[i];
    double acc[3] = {0, 0, 0};
    for (int l = 0; l < P; ++l) {
      Real ph = kx[l] * x + ky[l] * y + kz[l] * z;
      Real fb = (Real)std::cos(ph) * (Real)rho[2 * l + 1];
      Real fc = (Real)std::sin(ph) * (Real)rho[2 * l];
      Real s = -fourpi * qi / (volume * k2[l]) * (fb - fc);
      if (weights) s *= (Real)weights[l];
      acc[0] += (double)(s * kx[l]);
      acc[1] += (double)(s * ky[l]);
      acc[2] += (double)(s * kz[l]);
    }
    for (int d = 0; d < 3; ++d) force_out[3 * i + d] = acc[d] * (double)S / P * qqr2e;
  }
}

EXPORT void oracle_rbe_force_f32(int64_t n, const float* pos, const double* charge,
                                 const double* box, const double* origin, double alpha,
                                 double qqr2e, int P, const int32_t* m, const double* rho,
                                 const double* weights, double S_override, double* force_out) {
  rbe_force_impl<float>(n, pos, charge, box, origin, alpha, qqr2e, P, m, rho, weights, S_override,
                        force_out);
}
EXPORT void oracle_rbe_force_f64(int64_t n, const double* pos, const double* charge,
                                 const double* box, const double* origin, double alpha,
                                 double qqr2e, int P, const int32_t* m, const double* rho,
                                 const double* weights, double S_override, double* force_out) {
  rbe_force_impl<double>(n, pos, charge, box, origin, alpha, qqr2e, P, m, rho, weights,
                         S_override, force_out);
}

// FP64 full Ewald reciprocal-space force and energy over all m != 0 with |k| <= kcut (the
// converged version of ComputeFarEle, ExecForceFunction.h:226-245, whose reference loop is the
// cube [-Kmax, Kmax]^3, ExecPointLocator.h:127-145).  Uses the per-axis recurrence
// e^{i k.r} = e^{i kx x} e^{i ky y} e^{i kz z} with tabulated powers.  force x qqr2e.
EXPORT double oracle_ewald_kspace_f64(int64_t n, const double* pos, const double* charge,
                                      const double* box, double alpha, double kcut, double qqr2e,
                                      double* force_out) {
  int M[3];
  for (int d = 0; d < 3; ++d) M[d] = (int)std::floor(kcut * box[d] / (2 * M_PI));
  const double V = box[0] * box[1] * box[2];
  std::vector<double> F(3 * n, 0.0);
  double energy = 0;
  // powers: e^{i 2pi m x/L} for m in [0, M]
  std::vector<double> cx(n * (M[0] + 1)), sx(n * (M[0] + 1)), cy(n * (M[1] + 1)),
      sy(n * (M[1] + 1)), cz(n * (M[2] + 1)), sz(n * (M[2] + 1));
  auto fill = [&](int d, std::vector<double>& c, std::vector<double>& s) {
    int Md = M[d];
#pragma omp parallel for
    for (int64_t j = 0; j < n; ++j) {
      double t = 2 * M_PI * pos[3 * j + d] / box[d];
      for (int mm = 0; mm <= Md; ++mm) {
        c[j * (Md + 1) + mm] = std::cos(mm * t);
        s[j * (Md + 1) + mm] = std::sin(mm * t);
      }
    }
  };
  fill(0, cx, sx);
  fill(1, cy, sy);
  fill(2, cz, sz);
  // enumerate half space (m > 0 lexicographic) and double
  std::vector<int> ms;
  for (int a = 0; a <= M[0]; ++a)
    for (int b = -M[1]; b <= M[1]; ++b)
      for (int c = -M[2]; c <= M[2]; ++c) {
        if (a == 0 && (b < 0 || (b == 0 && c <= 0))) continue;
        double kx = 2 * M_PI * a / box[0], ky = 2 * M_PI * b / box[1], kz = 2 * M_PI * c / box[2];
        if (kx * kx + ky * ky + kz * kz > kcut * kcut) continue;
        ms.push_back(a); ms.push_back(b); ms.push_back(c);
      }
  int64_t nk = (int64_t)ms.size() / 3;
  auto phase = [&](int64_t j, int a, int b, int c, double& co, double& si) {
    double c1 = cx[j * (M[0] + 1) + a], s1 = sx[j * (M[0] + 1) + a];
    double c2 = cy[j * (M[1] + 1) + std::abs(b)], s2 = (b < 0 ? -1 : 1) * sy[j * (M[1] + 1) + std::abs(b)];
    double c3 = cz[j * (M[2] + 1) + std::abs(c)], s3 = (c < 0 ? -1 : 1) * sz[j * (M[2] + 1) + std::abs(c)];
    double c12 = c1 * c2 - s1 * s2, s12 = s1 * c2 + c1 * s2;
    co = c12 * c3 - s12 * s3;
    si = s12 * c3 + c12 * s3;
  };
#pragma omp parallel
  {
    std::vector<double> Fl(3 * n, 0.0);
    double el = 0;
#pragma omp for schedule(dynamic, 16)
    for (int64_t kk = 0; kk < nk; ++kk) {
      int a = ms[3 * kk], b = ms[3 * kk + 1], c = ms[3 * kk + 2];
      double kx = 2 * M_PI * a / box[0], ky = 2 * M_PI * b / box[1], kz = 2 * M_PI * c / box[2];
      double k2 = kx * kx + ky * ky + kz * kz;
      double re = 0, im = 0;
      for (int64_t j = 0; j < n; ++j) {
        double co, si;
        phase(j, a, b, c, co, si);
        re += charge[j] * co;
        im += charge[j] * si;
      }
      double g = std::exp(-k2 / (4 * alpha)) / k2;
      el += 2.0 * (2 * M_PI / V) * g * (re * re + im * im);
      for (int64_t j = 0; j < n; ++j) {
        double co, si;
        phase(j, a, b, c, co, si);
        // F_j = -(4 pi q_j / V) g k (cos Im - sin Re), doubled for -k
        double s = -2.0 * 4 * M_PI * charge[j] / V * g * (co * im - si * re);
        Fl[3 * j] += s * kx;
        Fl[3 * j + 1] += s * ky;
        Fl[3 * j + 2] += s * kz;
      }
    }
#pragma omp critical
    {
      for (int64_t t = 0; t < 3 * n; ++t) F[t] += Fl[t];
      energy += el;
    }
  }
  for (int64_t t = 0; t < 3 * n; ++t) force_out[t] = F[t] * qqr2e;
  return energy * qqr2e;
}

// FP64 real-space Ewald force and energy over the full list (erfc(sqrt(a) r)/r), x qqr2e.
EXPORT double oracle_ewald_real_f64(int64_t n, const double* pos, const double* lo,
                                    const double* hi, double cutoff, const double* charge,
                                    double alpha, double qqr2e, int64_t cap, const int32_t* counts,
                                    const int32_t* ids, const int32_t* codes, double* force_out) {
  Grid<double> g = make_grid<double>(lo, hi, cutoff, cutoff);
  double energy = 0;
#pragma omp parallel for reduction(+ : energy) schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    double f[3] = {0, 0, 0};
    for (int32_t p = 0; p < counts[i]; ++p) {
      int j = ids[i * cap + p];
      double off[3];
      shift_offset(g, codes[i * cap + p], off);
      double r[3];
      for (int d = 0; d < 3; ++d) r[d] = (pos[3 * i + d] - (pos[3 * j + d] - off[d]));
      double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      double d = std::sqrt(d2);
      if (d >= cutoff) continue;
      double qq = charge[i] * charge[j];
      double gg = std::erfc(std::sqrt(alpha) * d) / d2 +
                  2 * std::sqrt(alpha / M_PI) * std::exp(-alpha * d2) / d;
      for (int k = 0; k < 3; ++k) f[k] += qq * gg * r[k] / d;
      energy += 0.5 * qq * std::erfc(std::sqrt(alpha) * d) / d;
    }
    for (int k = 0; k < 3; ++k) force_out[3 * i + k] = f[k] * qqr2e;
  }
  return energy * qqr2e;
}

// ------------------------------------------------------------------------------------------
// EAM (funcfl): ExecutionNVT::ReadPotentialFile / file2array / interpolate / array2spline
// (rbmd/framework/run/ExecutionNVT.cpp:903-1107); the passes ComputeEAMfpVerletWorklet and
// ComputeEAMForceVerletWorklet (RunWorklet.cpp:305-417) with ComputeEAMrho / ComputeEAMfp /
// ComputeEAMforce (ExecForceFunction.h:333-481).  The reader stores the file arrays 0-based
// while file2array indexes them 1-based (k-1 .. k+2), and rho(r) is read with the nrho count;
// both are kept.
// ------------------------------------------------------------------------------------------
struct EamTables {
  int nrho, nr;
  float drho, dr, rhomax, cut;
  std::vector<float> frho_spl, rhor_spl, z2r_spl;   // 7 floats per entry, (n+1) entries
};

static void eam_interpolate(int n, float delta, const std::vector<float>& f, std::vector<float>& s) {
  auto S = [&](int m, int c) -> float& { return s[7 * m + c]; };
  for (int m = 1; m <= n; m++) S(m, 6) = f[m];
  S(1, 5) = S(2, 6) - S(1, 6);
  S(2, 5) = (float)(0.5 * (S(3, 6) - S(1, 6)));
  S(n - 1, 5) = (float)(0.5 * (S(n, 6) - S(n - 2, 6)));
  S(n, 5) = S(n, 6) - S(n - 1, 6);
  for (int m = 3; m <= n - 2; m++)
    S(m, 5) = (float)(((S(m - 2, 6) - S(m + 2, 6)) + 8.0 * (S(m + 1, 6) - S(m - 1, 6))) / 12.0);
  for (int m = 1; m <= n - 1; m++) {
    S(m, 4) = (float)(3.0 * (S(m + 1, 6) - S(m, 6)) - 2.0 * S(m, 5) - S(m + 1, 5));
    S(m, 3) = (float)(S(m, 5) + S(m + 1, 5) - 2.0 * (S(m + 1, 6) - S(m, 6)));
  }
  S(n, 4) = 0.0f;
  S(n, 3) = 0.0f;
  for (int m = 1; m <= n; m++) {
    S(m, 2) = S(m, 5) / delta;
    S(m, 1) = (float)(2.0 * S(m, 4) / delta);
    S(m, 0) = (float)(3.0 * S(m, 3) / delta);
  }
}

static int eam_load(const char* path, EamTables& t) {
  std::ifstream in(path);
  if (!in.is_open()) return 1;
  for (int i = 0; i < 2; ++i) in.ignore(std::numeric_limits<std::streamsize>::max(), '\n');
  int fnrho, fnr;
  float fdrho, fdr, fcut;
  in >> fnrho >> fdrho >> fnr >> fdr >> fcut;
  if (!in || fnrho < 5 || fnr < 5) return 2;
  std::vector<float> ffrho(fnrho + 1), fzr(fnr + 1), frhor(std::max(fnrho, fnr) + 1);
  for (int i = 0; i < fnrho; ++i) in >> ffrho[i];
  for (int i = 0; i < fnr; ++i) in >> fzr[i];
  for (int i = 0; i < fnrho; ++i) in >> frhor[i];
  if (!in) return 3;
  const float sixth = (float)(1.0 / 6.0);
  float dr = 0, drho = 0, rmax = 0, rhomax = 0;
  dr = std::max(dr, fdr);
  drho = std::max(drho, fdrho);
  rmax = std::max(rmax, (fnr - 1) * fdr);
  rhomax = std::max(rhomax, (fnrho - 1) * fdrho);
  int nr = (int)(rmax / dr + 0.5);
  int nrho = (int)(rhomax / drho + 0.5);
  std::vector<float> frho(nrho + 1), rhor(std::max(nrho, nr) + 1), z2r(nr + 1);
  auto cofs = [&](float p, float* c) {
    c[0] = (float)(-sixth * p * (p - 1.0) * (p - 2.0));
    c[1] = (float)(0.5 * (p * p - 1.0) * (p - 2.0));
    c[2] = (float)(-0.5 * p * (p + 1.0) * (p - 2.0));
    c[3] = (float)(sixth * p * (p * p - 1.0));
  };
  for (int m = 1; m <= nrho; m++) {
    float r = (float)(m - 1) * drho;
    float p = (float)(r / fdrho + 1.0);
    int k = (int)p;
    k = std::min(k, fnrho - 2);
    k = std::max(k, 2);
    p -= (float)k;
    p = std::min(p, 2.0f);
    float c[4];
    cofs(p, c);
    frho[m] = c[0] * ffrho[k - 1] + c[1] * ffrho[k] + c[2] * ffrho[k + 1] + c[3] * ffrho[k + 2];
  }
  for (int m = 1; m <= nr; m++) {
    float r = (float)(m - 1) * dr;
    float p = (float)(r / fdr + 1.0);
    int k = (int)p;
    k = std::min(k, fnr - 2);
    k = std::max(k, 2);
    p -= (float)k;
    p = std::min(p, 2.0f);
    // ExecutionNVT.cpp:1003-1006 declare these `auto`: the products are double
    double c0 = -sixth * p * (p - 1.0) * (p - 2.0);
    double c1 = 0.5 * (p * p - 1.0) * (p - 2.0);
    double c2 = -0.5 * p * (p + 1.0) * (p - 2.0);
    double c3 = sixth * p * (p * p - 1.0);
    if (m < (int)rhor.size())
      rhor[m] = (float)(c0 * frhor[k - 1] + c1 * frhor[k] + c2 * frhor[k + 1] + c3 * frhor[k + 2]);
  }
  for (int m = 1; m <= nr; m++) {
    float r = (float)(m - 1) * dr;
    float p = (float)(r / fdr + 1.0);
    int k = (int)p;
    k = std::min(k, fnr - 2);
    k = std::max(k, 2);
    p -= (float)k;
    p = std::min(p, 2.0f);
    float c[4];
    cofs(p, c);
    // Real cof1..cof4 times Real zr: a float sum stored into the double zri
    float zf = c[0] * fzr[k - 1] + c[1] * fzr[k] + c[2] * fzr[k + 1] + c[3] * fzr[k + 2];
    double zri = (double)zf;
    z2r[m] = (float)(27.2 * 0.529 * zri * zri);
  }
  t.nrho = nrho;
  t.nr = nr;
  t.drho = drho;
  t.dr = dr;
  t.rhomax = rhomax;
  t.cut = fcut;
  t.frho_spl.assign(7 * (nrho + 1), 0.f);
  t.rhor_spl.assign(7 * (std::max(nrho, nr) + 1), 0.f);
  t.z2r_spl.assign(7 * (nr + 1), 0.f);
  eam_interpolate(nrho, drho, frho, t.frho_spl);
  eam_interpolate(nr, dr, rhor, t.rhor_spl);
  eam_interpolate(nr, dr, z2r, t.z2r_spl);
  return 0;
}

// meta: nrho, nr, drho, dr, rhomax, cut
EXPORT int oracle_eam_tables(const char* path, double* meta, float* frho, float* rhor, float* z2r,
                             int64_t max_entries) {
  EamTables t;
  int rc = eam_load(path, t);
  if (rc) return rc;
  meta[0] = t.nrho; meta[1] = t.nr; meta[2] = t.drho; meta[3] = t.dr; meta[4] = t.rhomax;
  meta[5] = t.cut;
  if (frho && (int64_t)t.frho_spl.size() <= 7 * max_entries)
    std::copy(t.frho_spl.begin(), t.frho_spl.end(), frho);
  if (rhor && (int64_t)t.rhor_spl.size() <= 7 * max_entries)
    std::copy(t.rhor_spl.begin(), t.rhor_spl.end(), rhor);
  if (z2r && (int64_t)t.z2r_spl.size() <= 7 * max_entries)
    std::copy(t.z2r_spl.begin(), t.z2r_spl.end(), z2r);
  return 0;
}

template <class Real>
static int eam_force_impl(const char* path, int64_t n, const Real* pos, const double* lo,
                          const double* hi, double cutoff, int64_t cap, const int32_t* counts,
                          const int32_t* ids, const int32_t* codes, int sum_mode, double* fp_out,
                          double* force_out, int ref_sign) {
  EamTables t;
  int rc0 = eam_load(path, t);
  if (rc0) return rc0;
  Grid<Real> g = make_grid<Real>(lo, hi, cutoff, cutoff);
  const Real rc = (Real)cutoff;
  std::vector<Real> fp(n);
  const Real rdr = (Real)1 / (Real)t.dr, rdrho = (Real)1 / (Real)t.drho;
  auto C = [&](const std::vector<float>& s, int m, int c) -> Real { return (Real)s[7 * m + c]; };
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    Real rho = 0;
    double rhod = 0;
    for (int32_t p = 0; p < counts[i]; ++p) {
      int j = ids[i * cap + p];
      Real off[3];
      shift_offset(g, codes[i * cap + p], off);
      Real pj[3] = {pos[3 * j] - off[0], pos[3 * j + 1] - off[1], pos[3 * j + 2] - off[2]};
      Real r[3];
      min_dist(pos + 3 * i, pj, g.box, r);
      Real rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      Real cutsq = rc * rc;
      Real v = 0;
      if (rsq < cutsq && (double)rsq > 0.01) {
        double pp = (double)((Real)std::sqrt(rsq) * rdr) + 1.0;
        int64_t m = (int64_t)pp;
        m = std::min<int64_t>(m, t.nr - 1);
        pp -= (double)m;
        pp = std::min(pp, 1.0);
        v = (Real)(((C(t.rhor_spl, m, 3) * pp + C(t.rhor_spl, m, 4)) * pp + C(t.rhor_spl, m, 5)) * pp +
                   C(t.rhor_spl, m, 6));
      }
      if (sum_mode == 0) rho += v; else rhod += (double)v;
    }
    Real rr = sum_mode == 0 ? rho : (Real)rhod;
    double pp = (double)(rr * rdrho) + 1.0;
    int m = (int)pp;
    m = std::max(1, std::min(m, t.nrho - 1));
    pp -= m;
    pp = std::min(pp, 1.0);
    fp[i] = (Real)((C(t.frho_spl, m, 0) * pp + C(t.frho_spl, m, 1)) * pp + C(t.frho_spl, m, 2));
    if (fp_out) fp_out[i] = (double)fp[i];
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    Real acc[3] = {0, 0, 0};
    double accd[3] = {0, 0, 0};
    for (int32_t p = 0; p < counts[i]; ++p) {
      int j = ids[i * cap + p];
      Real off[3];
      shift_offset(g, codes[i * cap + p], off);
      Real pj[3] = {pos[3 * j] - off[0], pos[3 * j + 1] - off[1], pos[3 * j + 2] - off[2]};
      // ref_sign: the reference's MinDistanceVec(p_j, p_i) (RunWorklet.cpp:402), which reverses
      // the force; otherwise p_i - p_j as in LAMMPS' pair_eam and the reference's own RBL pass
      // (RunWorklet.cpp:1180), the sign for which F = -grad E.
      Real r[3];
      if (ref_sign) min_dist(pj, pos + 3 * i, g.box, r);
      else min_dist(pos + 3 * i, pj, g.box, r);
      Real rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      Real cutsq = rc * rc;
      Real f[3] = {0, 0, 0};
      if (rsq < cutsq && (double)rsq > 0.01) {
        Real rv = (Real)std::sqrt(rsq);
        double pp = (double)(rv * rdr) + 1.0;
        int m = (int)pp;
        m = std::min(m, t.nr - 1);
        pp -= m;
        pp = std::min(pp, 1.0);
        double rhoip = (C(t.rhor_spl, m, 0) * pp + C(t.rhor_spl, m, 1)) * pp + C(t.rhor_spl, m, 2);
        double rhojp = rhoip;
        double z2p = (C(t.z2r_spl, m, 0) * pp + C(t.z2r_spl, m, 1)) * pp + C(t.z2r_spl, m, 2);
        double z2 = ((C(t.z2r_spl, m, 3) * pp + C(t.z2r_spl, m, 4)) * pp + C(t.z2r_spl, m, 5)) * pp +
                    C(t.z2r_spl, m, 6);
        double recip = 1.0 / (double)rv;
        double phi = z2 * recip;
        double phip = z2p * recip - phi * recip;
        double psip = (double)fp[i] * rhojp + (double)fp[j] * rhoip + phip;
        double fpair = -psip * recip;
        for (int d = 0; d < 3; ++d) f[d] = (Real)((double)r[d] * fpair);
      }
      for (int d = 0; d < 3; ++d) {
        if (sum_mode == 0) acc[d] += f[d]; else accd[d] += (double)f[d];
      }
    }
    for (int d = 0; d < 3; ++d) force_out[3 * i + d] = sum_mode == 0 ? (double)acc[d] : accd[d];
  }
  return 0;
}

EXPORT int oracle_eam_force_f32(const char* path, int64_t n, const float* pos, const double* lo,
                                const double* hi, double cutoff, int64_t cap, const int32_t* counts,
                                const int32_t* ids, const int32_t* codes, int sum_mode,
                                double* fp_out, double* force_out, int ref_sign) {
  return eam_force_impl<float>(path, n, pos, lo, hi, cutoff, cap, counts, ids, codes, sum_mode,
                               fp_out, force_out, ref_sign);
}
EXPORT int oracle_eam_force_f64(const char* path, int64_t n, const double* pos, const double* lo,
                                const double* hi, double cutoff, int64_t cap,
                                const int32_t* counts, const int32_t* ids, const int32_t* codes,
                                int sum_mode, double* fp_out, double* force_out, int ref_sign) {
  return eam_force_impl<double>(path, n, pos, lo, hi, cutoff, cap, counts, ids, codes, sum_mode,
                                fp_out, force_out, ref_sign);
}

// EAM total energy sum_i F(rho_i) + 1/2 sum_ij phi(r_ij) in FP64 over a full list, with the
// value coefficients (3..6) of the same splines (ComputeEAMrhoOUT and the energy terms of
// ThermoOutput, rbmd/framework/forceFunction/ExecForceFunction.h:522-613); the finite-difference
// check of the force sign uses it.
EXPORT double oracle_eam_energy_f64(const char* path, int64_t n, const double* pos, const double* lo,
                                    const double* hi, double cutoff, int64_t cap,
                                    const int32_t* counts, const int32_t* ids, const int32_t* codes) {
  EamTables t;
  if (eam_load(path, t)) return NAN;
  Grid<double> g = make_grid<double>(lo, hi, cutoff, cutoff);
  auto C = [&](const std::vector<float>& s, int64_t m, int c) -> double { return (double)s[7 * m + c]; };
  double e = 0;
  for (int64_t i = 0; i < n; ++i) {
    double rho = 0, pair = 0;
    for (int32_t p = 0; p < counts[i]; ++p) {
      int j = ids[i * cap + p];
      double off[3];
      shift_offset(g, codes[i * cap + p], off);
      double pj[3] = {pos[3 * j] - off[0], pos[3 * j + 1] - off[1], pos[3 * j + 2] - off[2]};
      double r[3];
      min_dist(pos + 3 * i, pj, g.box, r);
      double rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      if (rsq < cutoff * cutoff && rsq > 0.01) {
        double rv = std::sqrt(rsq);
        double pp = rv / (double)t.dr + 1.0;
        int64_t m = std::min<int64_t>((int64_t)pp, t.nr - 1);
        pp -= (double)m;
        pp = std::min(pp, 1.0);
        rho += ((C(t.rhor_spl, m, 3) * pp + C(t.rhor_spl, m, 4)) * pp + C(t.rhor_spl, m, 5)) * pp +
               C(t.rhor_spl, m, 6);
        double z2 = ((C(t.z2r_spl, m, 3) * pp + C(t.z2r_spl, m, 4)) * pp + C(t.z2r_spl, m, 5)) * pp +
                    C(t.z2r_spl, m, 6);
        pair += z2 / rv;
      }
    }
    double pp = rho / (double)t.drho + 1.0;
    int m = std::max(1, std::min((int)pp, t.nrho - 1));
    pp -= m;
    pp = std::min(pp, 1.0);
    double F = ((C(t.frho_spl, m, 3) * pp + C(t.frho_spl, m, 4)) * pp + C(t.frho_spl, m, 5)) * pp +
               C(t.frho_spl, m, 6);
    if (rho > t.rhomax) {
      double fp = (C(t.frho_spl, m, 0) * pp + C(t.frho_spl, m, 1)) * pp + C(t.frho_spl, m, 2);
      F += fp * (rho - t.rhomax);
    }
    e += F + 0.5 * pair;
  }
  return e;
}

// ------------------------------------------------------------------------------------------
// SHAKE (positions) and RATTLE (velocities) for rigid 3-site water:
// NewConstraintAWaterBondAngleWorklet / NewConstraintBWaterBondAngleWorklet
// (rbmd/framework/run/worklet/MolecularWorklet.h:2209-2656).  Bond 1.0 and the H-H distance
// from 109.47 degrees are fixed as in the reference; tol and max_iter are arguments
// (the reference uses 1e-5 and 5000).  FP64.
// ------------------------------------------------------------------------------------------
static inline void md(const double* a, const double* b, const double* box, double* v) {
  for (int d = 0; d < 3; ++d) {
    v[d] = a[d] - b[d];
    if (std::fabs(v[d]) > box[d] * 0.5) v[d] -= (v[d] > 0 ? box[d] : -box[d]);
  }
}
static inline double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

EXPORT int oracle_shake_f64(int64_t n_mol, const int32_t* hoh, double* pos_old, double* vel_old,
                            const double* force, const double* mass, int32_t* image,
                            const double* lo, const double* hi, double dt, double fmt2v, double tol,
                            int max_iter, int32_t* iters_out) {
  double box[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  int nonconv = 0;
  for (int64_t w = 0; w < n_mol; ++w) {
    int id[3] = {hoh[3 * w], hoh[3 * w + 1], hoh[3 * w + 2]};
    double sp[3][3];
    for (int a = 0; a < 3; ++a)
      for (int d = 0; d < 3; ++d)
        sp[a][d] = pos_old[3 * id[a] + d] + vel_old[3 * id[a] + d] * dt +
                   0.5 * dt * dt * force[3 * id[a] + d] / mass[id[a]] * fmt2v;
    const double bond1 = 1.0, bond2 = 1.0;
    const double bond12 = std::sqrt(bond1 * bond1 + bond2 * bond2 -
                                    2.0 * bond1 * bond2 * std::cos((109.4700 / 180.0) * M_PI));
    double r01[3], r12[3], r20[3], s10[3], s21[3], s02[3];
    md(pos_old + 3 * id[1], pos_old + 3 * id[0], box, r01);
    md(pos_old + 3 * id[2], pos_old + 3 * id[1], box, r12);
    md(pos_old + 3 * id[0], pos_old + 3 * id[2], box, r20);
    md(sp[0], sp[1], box, s10);
    md(sp[1], sp[2], box, s21);
    md(sp[2], sp[0], box, s02);
    double r01sq = dot3(r01, r01), r02sq = dot3(r20, r20), r12sq = dot3(r12, r12);
    double s01sq = dot3(s10, s10), s02sq = dot3(s02, s02), s12sq = dot3(s21, s21);
    double im0 = 1.0 / mass[id[0]], im1 = 1.0 / mass[id[1]], im2 = 1.0 / mass[id[2]];
    double a11 = 2.0 * (im0 + im1) * dot3(s10, r01);
    double a12 = -2.0 * im1 * dot3(s10, r12);
    double a13 = -2.0 * im0 * dot3(s10, r20);
    double a21 = -2.0 * im1 * dot3(s21, r01);
    double a22 = 2.0 * (im1 + im2) * dot3(s21, r12);
    double a23 = -2.0 * im2 * dot3(s21, r20);
    double a31 = -2.0 * im0 * dot3(s02, r01);
    double a32 = -2.0 * im2 * dot3(s02, r12);
    double a33 = 2.0 * (im0 + im2) * dot3(s02, r20);
    double det = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a11 * a23 * a32 -
                 a12 * a21 * a33 - a13 * a22 * a31;
    double di = 1.0 / det;
    double b11 = di * (a22 * a33 - a23 * a32), b12 = -di * (a12 * a33 - a13 * a32),
           b13 = di * (a12 * a23 - a13 * a22), b21 = -di * (a21 * a33 - a23 * a31),
           b22 = di * (a11 * a33 - a13 * a31), b23 = -di * (a11 * a23 - a13 * a21),
           b31 = di * (a21 * a32 - a22 * a31), b32 = -di * (a11 * a32 - a12 * a31),
           b33 = di * (a11 * a22 - a12 * a21);
    double r0120 = dot3(r01, r20), r0112 = dot3(r01, r12), r2012 = dot3(r20, r12);
    double q1_0101 = (im0 + im1) * (im0 + im1) * r01sq, q1_1212 = im1 * im1 * r12sq,
           q1_2020 = im0 * im0 * r02sq, q1_0120 = -2.0 * (im0 + im1) * im0 * r0120,
           q1_0112 = -2.0 * (im0 + im1) * im1 * r0112, q1_2012 = 2.0 * im0 * im1 * r2012;
    double q2_0101 = im1 * im1 * r01sq, q2_1212 = (im1 + im2) * (im1 + im2) * r12sq,
           q2_2020 = im2 * im2 * r02sq, q2_0120 = 2.0 * im1 * im2 * r0120,
           q2_0112 = -2.0 * (im1 + im2) * im1 * r0112, q2_2012 = -2.0 * (im1 + im2) * im2 * r2012;
    double q3_0101 = im0 * im0 * r01sq, q3_1212 = im2 * im2 * r12sq,
           q3_2020 = (im0 + im2) * (im0 + im2) * r02sq, q3_0120 = -2.0 * (im0 + im2) * im0 * r0120,
           q3_0112 = 2.0 * im0 * im2 * r0112, q3_2012 = -2.0 * (im0 + im2) * im2 * r2012;
    double l01 = 0, l20 = 0, l12 = 0;
    int niter = 0, done = 0;
    while (!done && niter < max_iter) {
      double quad1 = q1_0101 * l01 * l01 + q1_2020 * l20 * l20 + q1_1212 * l12 * l12 +
                     q1_0120 * l01 * l20 + q1_0112 * l01 * l12 + q1_2012 * l20 * l12;
      double quad2 = q2_0101 * l01 * l01 + q2_2020 * l20 * l20 + q2_1212 * l12 * l12 +
                     q2_0120 * l01 * l20 + q2_0112 * l01 * l12 + q2_2012 * l20 * l12;
      double quad3 = q3_0101 * l01 * l01 + q3_2020 * l20 * l20 + q3_1212 * l12 * l12 +
                     q3_0120 * l01 * l20 + q3_0112 * l01 * l12 + q3_2012 * l20 * l12;
      double b1 = bond1 * bond1 - s01sq - quad1;
      double b2 = bond2 * bond2 - s12sq - quad2;
      double b3 = bond12 * bond12 - s02sq - quad3;
      double n01 = b11 * b1 + b12 * b2 + b13 * b3;
      double n12 = b21 * b1 + b22 * b2 + b23 * b3;
      double n20 = b31 * b1 + b32 * b2 + b33 * b3;
      done = 1;
      if (std::fabs(n01 - l01) > tol) done = 0;
      if (std::fabs(n20 - l20) > tol) done = 0;
      if (std::fabs(n12 - l12) > tol) done = 0;
      l01 = n01; l20 = n20; l12 = n12;
      if (std::isnan(l01) || std::isnan(l20) || std::isnan(l12) || std::fabs(l01) > 1e20 ||
          std::fabs(l20) > 1e20 || std::fabs(l12) > 1e20)
        done = 1;
      niter++;
    }
    if (!done) nonconv = 1;
    if (iters_out) iters_out[w] = niter;
    double pc[3][3], sv[3][3];
    for (int d = 0; d < 3; ++d) {
      pc[0][d] = l01 * r01[d] * im0 - l20 * r20[d] * im0;
      pc[1][d] = l12 * r12[d] * im1 - l01 * r01[d] * im1;
      pc[2][d] = l20 * r20[d] * im2 - l12 * r12[d] * im2;
    }
    for (int a = 0; a < 3; ++a)
      for (int d = 0; d < 3; ++d) {
        sv[a][d] = vel_old[3 * id[a] + d] + 0.5 * dt * force[3 * id[a] + d] / mass[id[a]] * fmt2v;
        vel_old[3 * id[a] + d] = sv[a][d] + pc[a][d] / dt;
        double x = sp[a][d] + pc[a][d];
        if (x < lo[d]) { x += hi[d] - lo[d]; if (image) image[3 * id[a] + d] -= 1; }
        if (x > hi[d]) { x -= hi[d] - lo[d]; if (image) image[3 * id[a] + d] += 1; }
        pos_old[3 * id[a] + d] = x;
      }
  }
  return nonconv;
}

EXPORT void oracle_rattle_f64(int64_t n_mol, const int32_t* hoh, const double* pos,
                              double* vel_old, const double* force, const double* mass,
                              const double* lo, const double* hi, double dt, double fmt2v) {
  double box[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  for (int64_t w = 0; w < n_mol; ++w) {
    int id[3] = {hoh[3 * w], hoh[3 * w + 1], hoh[3 * w + 2]};
    double sv[3][3];
    for (int a = 0; a < 3; ++a)
      for (int d = 0; d < 3; ++d)
        sv[a][d] = vel_old[3 * id[a] + d] + 0.5 * dt * force[3 * id[a] + d] / mass[id[a]] * fmt2v;
    double r01[3], r12[3], r20[3];
    md(pos + 3 * id[1], pos + 3 * id[0], box, r01);
    md(pos + 3 * id[2], pos + 3 * id[1], box, r12);
    md(pos + 3 * id[0], pos + 3 * id[2], box, r20);
    double sv10[3], sv21[3], sv02[3];
    for (int d = 0; d < 3; ++d) {
      sv10[d] = sv[0][d] - sv[1][d];
      sv21[d] = sv[1][d] - sv[2][d];
      sv02[d] = sv[2][d] - sv[0][d];
    }
    double im0 = 1.0 / mass[id[0]], im1 = 1.0 / mass[id[1]], im2 = 1.0 / mass[id[2]];
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
    double c[3] = {-dot3(sv10, r01), -dot3(sv21, r12), -dot3(sv02, r20)};
    double det = a[0][0] * a[1][1] * a[2][2] + a[0][1] * a[1][2] * a[2][0] +
                 a[0][2] * a[1][0] * a[2][1] - a[0][0] * a[1][2] * a[2][1] -
                 a[0][1] * a[1][0] * a[2][2] - a[0][2] * a[1][1] * a[2][0];
    double di = 1.0 / det;
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
      vel_old[3 * id[0] + d] = sv[0][d] + (l[0] * r01[d] * im0 - l[2] * r20[d] * im0);
      vel_old[3 * id[1] + d] = sv[1][d] + (l[1] * r12[d] * im1 - l[0] * r01[d] * im1);
      vel_old[3 * id[2] + d] = sv[2][d] + (l[2] * r20[d] * im2 - l[1] * r12[d] * im2);
    }
  }
}

// Intramolecular bare-Coulomb removal (ComputeSpecialCoulWorklet, RunWorklet.cpp:1386-1437) and
// harmonic bond / angle of each (H,O,H) triple (ComputeBondHarmonicWorklet /
// ComputeAngleHarmonicWorklet, MolecularWorklet.h:57-283): bonds (0,1), (2,1); angle 0-1-2.
EXPORT void oracle_water_extras_f64(int64_t n_mol, const int32_t* hoh, const double* pos,
                                    const double* charge, const double* lo, const double* hi,
                                    double bond_k, double bond_r0, double angle_k,
                                    double angle_theta0_deg, double* force_out, double* e_out) {
  double box[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  double eb = 0, ea = 0;
  for (int64_t w = 0; w < n_mol; ++w) {
    int id[3] = {hoh[3 * w], hoh[3 * w + 1], hoh[3 * w + 2]};
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        if (a == b) continue;
        double r[3];
        md(pos + 3 * id[a], pos + 3 * id[b], box, r);
        double d = std::sqrt(dot3(r, r));
        double fc = -332.06371 * charge[id[a]] * charge[id[b]] / (d * d * d);
        for (int k = 0; k < 3; ++k) force_out[3 * id[a] + k] += fc * r[k];
      }
    int bonds[2][2] = {{id[0], id[1]}, {id[2], id[1]}};
    for (auto& bd : bonds) {
      double r[3];
      md(pos + 3 * bd[0], pos + 3 * bd[1], box, r);
      double d = std::sqrt(dot3(r, r));
      double dr = d - bond_r0, rk = bond_k * dr;
      double fb = d > 0.01 ? -2.0 * rk / d : 0.0;
      for (int k = 0; k < 3; ++k) {
        force_out[3 * bd[0] + k] += fb * r[k];
        force_out[3 * bd[1] + k] -= fb * r[k];
      }
      eb += rk * dr;
    }
    double rij[3], rkj[3];
    md(pos + 3 * id[0], pos + 3 * id[1], box, rij);
    md(pos + 3 * id[2], pos + 3 * id[1], box, rkj);
    double dij2 = dot3(rij, rij), dij = std::sqrt(dij2), dkj2 = dot3(rkj, rkj), dkj = std::sqrt(dkj2);
    double c = dot3(rij, rkj) / (dij * dkj);
    c = std::min(1.0, std::max(-1.0, c));
    double s = std::sqrt(1.0 - c * c);
    if (s < 0.001) s = 0.001;
    s = 1.0 / s;
    double dth = std::acos(c) - angle_theta0_deg * M_PI / 180.0;
    double tk = angle_k * dth;
    ea += tk * dth;
    double aa = -2.0 * tk * s, a11 = aa * c / dij2, a12 = -aa / (dij * dkj), a22 = aa * c / dkj2;
    for (int k = 0; k < 3; ++k) {
      double fi = a11 * rij[k] + a12 * rkj[k], fk = a22 * rkj[k] + a12 * rij[k];
      force_out[3 * id[0] + k] += fi;
      force_out[3 * id[1] + k] += -fi - fk;
      force_out[3 * id[2] + k] += fk;
    }
  }
  if (e_out) { e_out[0] = eb; e_out[1] = ea; }
}

// Special-bond partner lists of ModelFileInitCondition::SetSpecialBonds
// (rbmd/framework/InitCondition/ModelFileInitCondition.cpp:850-910): the bond graph as a multimap
// filled in Bonds order (both directions, :509-511); for each atom in id order its 1-2 partners
// (weight w3[0]), through each of them the 1-3 partners other than the atom itself (w3[1]) and
// through those the 1-4 partners other than the 1-2 atom they came from (w3[2]); an atom without
// bonds gets the single entry (itself, 1.0).  Duplicates are kept, as in the reference.  Writes
// off[n+1], ids/wts up to cap entries; returns the number of entries.
EXPORT int64_t oracle_special_lists(int64_t n, int64_t nb, const int32_t* bonds, const double* w3, int64_t cap,
                                    int64_t* off, int32_t* ids, double* wts) {
  std::vector<std::vector<int32_t>> adj(n);
  for (int64_t b = 0; b < nb; ++b) {
    adj[bonds[2 * b]].push_back(bonds[2 * b + 1]);
    adj[bonds[2 * b + 1]].push_back(bonds[2 * b]);
  }
  int64_t m = 0;
  auto put = [&](int32_t id, double w) {
    if (m < cap) { ids[m] = id; wts[m] = w; }
    ++m;
  };
  for (int64_t a = 0; a < n; ++a) {
    off[a] = m;
    if (adj[a].empty()) { put((int32_t)a, 1.0); continue; }
    for (int32_t k1 : adj[a]) {
      put(k1, w3[0]);
      for (int32_t k2 : adj[k1]) {
        if (k2 == a) continue;
        put(k2, w3[1]);
        for (int32_t k3 : adj[k2]) {
          if (k3 == k1) continue;
          put(k3, w3[2]);
        }
      }
    }
  }
  off[n] = m;
  return m;
}

// Harmonic dihedral of ComputeDihedralHarmonicWorklet::ComputeijDihedralHarmonicEnergyForce
// (rbmd/framework/run/worklet/MolecularWorklet.h:555-818): E = K [1 + d cos(n phi)] with
// cos_shift = d = +-1, sin_shift = 0, cos(n phi) by the angle-addition recursion.
static double dihedral_harmonic(const double* pi, const double* pj, const double* pk, const double* pw,
                                const double* box, double K, int sign, int mult, double f[4][3]) {
  double vb1[3], vb2[3], vb3[3], vb2m[3];
  md(pi, pj, box, vb1);
  md(pk, pj, box, vb2);
  for (int d = 0; d < 3; ++d) vb2m[d] = -vb2[d];
  md(pw, pk, box, vb3);
  const double ax = vb1[1] * vb2m[2] - vb1[2] * vb2m[1];
  const double ay = vb1[2] * vb2m[0] - vb1[0] * vb2m[2];
  const double az = vb1[0] * vb2m[1] - vb1[1] * vb2m[0];
  const double bx = vb3[1] * vb2m[2] - vb3[2] * vb2m[1];
  const double by = vb3[2] * vb2m[0] - vb3[0] * vb2m[2];
  const double bz = vb3[0] * vb2m[1] - vb3[1] * vb2m[0];
  const double rasq = ax * ax + ay * ay + az * az;
  const double rbsq = bx * bx + by * by + bz * bz;
  const double rgsq = vb2m[0] * vb2m[0] + vb2m[1] * vb2m[1] + vb2m[2] * vb2m[2];
  const double rg = std::sqrt(rgsq);
  const double rginv = rg > 0 ? 1.0 / rg : 0.0;
  const double ra2inv = rasq > 0 ? 1.0 / rasq : 0.0;
  const double rb2inv = rbsq > 0 ? 1.0 / rbsq : 0.0;
  const double rabinv = std::sqrt(ra2inv * rb2inv);
  double c = (ax * bx + ay * by + az * bz) * rabinv;
  const double s = rg * rabinv * (ax * vb3[0] + ay * vb3[1] + az * vb3[2]);
  c = std::min(1.0, std::max(-1.0, c));
  const double cos_shift = sign == 1 ? 1.0 : -1.0, sin_shift = 0.0;
  double p = 1.0, ddf1 = 0.0, df1 = 0.0;
  for (int i = 0; i < mult; ++i) {
    ddf1 = p * c - df1 * s;
    df1 = p * s + df1 * c;
    p = ddf1;
  }
  p = p * cos_shift + df1 * sin_shift;
  df1 = df1 * cos_shift - ddf1 * sin_shift;
  df1 *= -mult;
  p += 1.0;
  if (mult == 0) { p = 1.0 + cos_shift; df1 = 0.0; }
  const double fg = vb1[0] * vb2m[0] + vb1[1] * vb2m[1] + vb1[2] * vb2m[2];
  const double hg = vb3[0] * vb2m[0] + vb3[1] * vb2m[1] + vb3[2] * vb2m[2];
  const double fga = fg * ra2inv * rginv, hgb = hg * rb2inv * rginv;
  const double gaa = -ra2inv * rg, gbb = rb2inv * rg;
  const double dtf[3] = {gaa * ax, gaa * ay, gaa * az};
  const double dtg[3] = {fga * ax - hgb * bx, fga * ay - hgb * by, fga * az - hgb * bz};
  const double dth[3] = {gbb * bx, gbb * by, gbb * bz};
  const double df = -K * df1;
  for (int d = 0; d < 3; ++d) {
    const double s2 = df * dtg[d];
    f[0][d] = df * dtf[d];
    f[1][d] = s2 - f[0][d];
    f[3][d] = df * dth[d];
    f[2][d] = -s2 - f[3][d];
  }
  return K * p;
}

// CVFF intramolecular terms of ExecutionNVT::ComputeAllForce (ExecutionNVT.cpp:199-215), added to
// force_out in the reference's order: special Coulomb (ComputeSpecialCoulWorklet /
// ComputeSpecialCoulGeneralWorklet, RunWorklet.cpp:1386-1511: for every other member j of the
// atom's molecule when the molecule has >= 3 atoms, -332.06371 q_i q_j r_ij / r^3 times 1, or
// times (1 - w_ij) with special lists), harmonic bonds k (r - r0)^2 (ComputeBondHarmonicWorklet),
// harmonic angles k (theta - theta0)^2 (ComputeAngleHarmonicWorklet), and, with special lists,
// harmonic dihedrals.  Coefficients per type: bonds (k, r0), angles (k, theta0 in degrees),
// dihedrals (K, sign, multiplicity).  e_out = {bond, angle, dihedral, special Coulomb} sums.
EXPORT void oracle_cvff_terms_f64(int64_t n, const double* pos, const double* lo, const double* hi,
                                  const double* charge, const int32_t* mol, int64_t nb, const int32_t* bonds,
                                  const int32_t* btype, const double* bcoef, int64_t na, const int32_t* angles,
                                  const int32_t* atype, const double* acoef, int64_t nd, const int32_t* dih,
                                  const int32_t* dtype, const double* dcoef, const int64_t* sp_off,
                                  const int32_t* sp_ids, const double* sp_w, double* force_out, double* e_out) {
  const double box[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  double eb = 0, ea = 0, ed = 0, es = 0;
  // molecule groups
  int32_t mmax = 0;
  for (int64_t i = 0; i < n; ++i) mmax = std::max(mmax, mol[i]);
  std::vector<std::vector<int32_t>> group((size_t)mmax + 1);
  for (int64_t i = 0; i < n; ++i) group[mol[i]].push_back((int32_t)i);
  std::vector<double> fsc(3 * n, 0.0), fb(3 * n, 0.0), fa(3 * n, 0.0), fd(3 * n, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    const auto& g = group[mol[i]];
    if (g.size() < 3) continue;
    for (int32_t j : g) {
      if (j == i) continue;
      double r[3];
      md(pos + 3 * i, pos + 3 * j, box, r);
      const double d = std::sqrt(dot3(r, r));
      const double fac = sp_off ? 1.0 - special_weight(sp_off, sp_ids, sp_w, i, j) : 1.0;
      const double fc = -332.06371 * charge[i] * charge[j] / (d * d * d);
      for (int k = 0; k < 3; ++k) fsc[3 * i + k] += fac * fc * r[k];
      es += -0.5 * fac * 332.06371 * charge[i] * charge[j] / d;
    }
  }
  for (int64_t b = 0; b < nb; ++b) {
    const int32_t i = bonds[2 * b], j = bonds[2 * b + 1];
    const double k = bcoef[2 * btype[b]], r0 = bcoef[2 * btype[b] + 1];
    double r[3];
    md(pos + 3 * i, pos + 3 * j, box, r);
    const double d = std::sqrt(dot3(r, r));
    const double dr = d - r0, rk = k * dr;
    const double f = d > 0.01 ? -2.0 * rk / d : 0.0;
    for (int c = 0; c < 3; ++c) { fb[3 * i + c] += f * r[c]; fb[3 * j + c] -= f * r[c]; }
    eb += rk * dr;
  }
  for (int64_t a = 0; a < na; ++a) {
    const int32_t i = angles[3 * a], j = angles[3 * a + 1], l = angles[3 * a + 2];
    const double k = acoef[2 * atype[a]], t0 = acoef[2 * atype[a] + 1] * M_PI / 180.0;
    double rij[3], rkj[3];
    md(pos + 3 * i, pos + 3 * j, box, rij);
    md(pos + 3 * l, pos + 3 * j, box, rkj);
    const double dij2 = dot3(rij, rij), dij = std::sqrt(dij2), dkj2 = dot3(rkj, rkj), dkj = std::sqrt(dkj2);
    double c = dot3(rij, rkj) / (dij * dkj);
    c = std::min(1.0, std::max(-1.0, c));
    double s = std::sqrt(1.0 - c * c);
    if (s < 0.001) s = 0.001;
    s = 1.0 / s;
    const double dth = std::acos(c) - t0, tk = k * dth;
    ea += tk * dth;
    const double aa = -2.0 * tk * s, a11 = aa * c / dij2, a12 = -aa / (dij * dkj), a22 = aa * c / dkj2;
    for (int q = 0; q < 3; ++q) {
      const double fi = a11 * rij[q] + a12 * rkj[q], fk = a22 * rkj[q] + a12 * rij[q];
      fa[3 * i + q] += fi;
      fa[3 * j + q] += -fi - fk;
      fa[3 * l + q] += fk;
    }
  }
  if (sp_off)
    for (int64_t t = 0; t < nd; ++t) {
      const int32_t* q = dih + 4 * t;
      const double* cf = dcoef + 3 * dtype[t];
      double f[4][3];
      ed += dihedral_harmonic(pos + 3 * q[0], pos + 3 * q[1], pos + 3 * q[2], pos + 3 * q[3], box, cf[0],
                              (int)cf[1], (int)cf[2], f);
      for (int a = 0; a < 4; ++a)
        for (int d = 0; d < 3; ++d) fd[3 * q[a] + d] += f[a][d];
    }
  for (int64_t i = 0; i < 3 * n; ++i) {
    force_out[i] += fsc[i];
    force_out[i] += fb[i];
    force_out[i] += fa[i];
    force_out[i] += fd[i];
  }
  if (e_out) { e_out[0] = eb; e_out[1] = ea; e_out[2] = ed; e_out[3] = es; }
}

EXPORT int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

EXPORT void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// ==========================================================================================
// RBL (random batch list) near field.
//   * list sizes: ExecutionMD::ComputeRBLNearForce / ComputeRBLLJForce / ComputeRBLEAMForce
//     (rbmd/framework/run/ExecutionMD.cpp:460-801): rho_system = N / (Lx Ly Lz) in Real,
//     rs_num = round(1 + 0.05/rho - 0.05) * rho * ceil(4/3 pi rs^3) + 1 (no round factor for
//     EAM), rc_num likewise, pice_num = ceil(1 / (sample_num / (rc_num - rs_num)));
//   * list: ComputeRBLNeighboursOnceWorklet (rbmd/framework/run/worklet/RunWorklet.cpp:634-708):
//     stencil x offset outermost, z innermost, points of a cell in sorted order; a candidate is a
//     shell pair when rc^2 - d^2 > 1e-4 && d^2 - rs^2 > 1e-4 and is kept when its running shell
//     index is a multiple of pice_num; otherwise a core pair when rs^2 - d^2 > 1e-4 && d^2 > 1e-4;
//   * forces: ComputeNearForceRBLERFWorklet (:710-814) and ComputeLJForceRBLWorklet
//     (:1218-1302): core Coulomb -q_i q_j G(d) r/d for 1e-4 < d^2 < rc^2 on p_j' - p_i (G from the
//     ERF table at |MinDistanceVec|), core LJ (ComputeLJForce), shell LJ x pice_num
//     (ComputeLJForceRcs: rs^2 < d^2 < rc^2), LJ skipped within a molecule; corr = LJ + qqr2e * Coul;
//   * EAM: ComputeEAMfp_Worklet / ComputeEAMRBLWorklet (:1052-1216) with ComputeEAMrhoRs and
//     ComputeEAMforceRBL (rbmd/framework/forceFunction/ExecForceFunction.h:358-381,484-520);
//   * mean removal: F_i = corr_i - (sum_j corr_j) / N (SumRBLCorrForceWorklet, RunWorklet.cpp:1304-1321).
// Reference quirks kept behind switches: table_mode 1 takes G from the reference's ERF table
// (alpha fixed at 0.1, one value per distance bucket, rbmd/framework/staticTable/
// ExecStaticTable.h:37-39,96-135); shell_coul 0 drops the shell Coulomb term, whose value the
// reference computes and discards (RunWorklet.cpp:782).  Defaults of the library: table_mode 0
// (G at the configured alpha and the exact distance) and shell_coul 1 (shell Coulomb x pice_num).
// ==========================================================================================
struct RblSizes { int64_t rs_num, rc_num, pice_num; };

template <class Real>
RblSizes rbl_sizes(int64_t n, const Real* box, double rs, double rc, double sample_num, bool eam) {
  const Real rho = (Real)n / (box[0] * box[1] * box[2]);
  const float pif = 3.14159265358979323846f;
  const Real rs_r = (Real)rs, rc_r = (Real)rc;
  int64_t coeff = 1;
  if (!eam) {
    const Real c = (Real)(1.0 + (0.05 / (double)rho - 0.05));
    coeff = (int64_t)std::round(c);
  }
  const double cs = std::ceil(4.0 / 3.0 * (double)pif * (double)rs_r * (double)rs_r * (double)rs_r);
  const double cc = std::ceil(4.0 / 3.0 * (double)pif * (double)rc_r * (double)rc_r * (double)rc_r);
  RblSizes z;
  z.rs_num = (int64_t)((double)(eam ? rho : (Real)coeff * rho) * cs + 1);
  z.rc_num = (int64_t)((double)(eam ? rho : (Real)coeff * rho) * cc + 1);
  const Real rate = (Real)sample_num / (Real)(z.rc_num - z.rs_num);
  z.pice_num = (int64_t)std::ceil(1.0 / (double)rate);
  return z;
}

template <class Real>
void rbl_list(const Grid<Real>& g, const Cells<Real>& c, int64_t n, const Real* pos, double cutoff,
              double rs, int64_t pice, int64_t core_cap, int64_t shell_cap, int32_t* ncore,
              int32_t* nshell, int32_t* ids, int32_t* codes) {
  const Real rc = (Real)cutoff, r_s = (Real)rs;
  const Real rc_2 = rc * rc, rs_2 = r_s * r_s;
  const int nc = g.num_cycles;
  const int64_t row = core_cap + shell_cap;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t a = 0; a < n; ++a) {
    const Real* pi = pos + 3 * a;
    int ci[3];
    for (int d = 0; d < 3; ++d) ci[d] = (int)((pi[d] - g.lo[d]) / g.dx[d]);
    int64_t index_shell = 0, index_random = 0, index_rs = 0;
    for (int i = -nc; i <= nc; ++i)
      for (int j = -nc; j <= nc; ++j)
        for (int k = -nc; k <= nc; ++k) {
          int nb[3] = {ci[0] + i, ci[1] + j, ci[2] + k};
          Real off[3];
          int code = 0, w[3];
          for (int d = 0; d < 3; ++d) {
            w[d] = ((nb[d] % g.dims[d]) + g.dims[d]) % g.dims[d];
            int delta = w[d] - nb[d];
            off[d] = g.dx[d] * (Real)delta;             // PeriodicCoordOffset
            int cd = delta > 0 ? 1 : (delta < 0 ? 2 : 0);
            code |= cd << (2 * d);
          }
          int cell = w[0] + w[1] * g.dims[0] + w[2] * g.dims[0] * g.dims[1];
          for (int s = c.lower[cell]; s < c.upper[cell]; ++s) {
            int jd = c.point_ids[s];
            const Real* pj = pos + 3 * jd;
            Real r0 = (pj[0] - off[0]) - pi[0];
            Real r1 = (pj[1] - off[1]) - pi[1];
            Real r2 = (pj[2] - off[2]) - pi[2];
            const Real dis_2 = r0 * r0 + r1 * r1 + r2 * r2;
            if ((double)(rc_2 - dis_2) > 0.0001 && (double)(dis_2 - rs_2) > 0.0001) {
              if (index_shell % pice == 0) {
                if (index_random < shell_cap) {
                  ids[a * row + core_cap + index_random] = jd;
                  codes[a * row + core_cap + index_random] = code;
                }
                ++index_random;
              }
              ++index_shell;
            } else if ((double)(rs_2 - dis_2) > 0.0001 && (double)dis_2 > 0.0001) {
              if (index_rs < core_cap) {
                ids[a * row + index_rs] = jd;
                codes[a * row + index_rs] = code;
              }
              ++index_rs;
            }
          }
        }
    ncore[a] = (int32_t)index_rs;
    nshell[a] = (int32_t)index_random;
  }
}

// The reference's ERF table (rbmd/framework/model/ERFTable.h via ExecStaticTable::Extract /
// TableGnearValue, rbmd/framework/staticTable/ExecStaticTable.h:37-39,96-135): the entry of a
// float distance is its bits 15..25; the entry's value is the reference's float Gnear(0.1, d_k)
// with d_k the entry's lower bucket edge rounded up to 4 decimals (d < 2) or 3 decimals (d >= 2),
// and at least 0.1, rounded to the 6 significant digits of the table's literals (1734 of the
// 1766 entries exact, the others within one unit of the sixth digit).  The reference's tables hold entries for 0.1 <= d < 12 only; outside, this
// evaluates G(0.1, d) in FP64 (the reference would read past its arrays).
inline float rbl_table_g(float dis) {
  if (!(dis >= 0.1f && dis < 12.0f)) {
    const double d = dis;
    return (float)gnear_fp64<double>(0.1, d);
  }
  uint32_t full;
  std::memcpy(&full, &dis, 4);
  const uint32_t edge_bits = full & ~0x7FFFu;
  float edge;
  std::memcpy(&edge, &edge_bits, 4);
  const int dec = dis < 2.0f ? 4 : 3;
  const double sc = std::pow(10.0, dec);
  const double v = (double)edge * sc, rv = std::nearbyint(v);
  double d = (std::fabs(v - rv) < 1e-6 ? rv : std::ceil(v)) / sc;
  if (d < 0.1) d = 0.1;
  // the table's literals carry 6 significant decimal digits
  char buf[32];
  std::snprintf(buf, sizeof buf, "%.6g", (double)gnear<float>(0.1f, (float)d));
  return (float)std::strtod(buf, nullptr);
}

template <class Real>
static void rbl_near_impl(int64_t n, const Real* pos, const double* lo, const double* hi,
                          double cutoff, double rs, int64_t pice, const int32_t* type,
                          const int32_t* mol, const double* charge, const double* eps,
                          const double* sig, int64_t core_cap, int64_t shell_cap,
                          const int32_t* ncore, const int32_t* nshell, const int32_t* ids,
                          const int32_t* codes, int with_coul, double alpha, double qqr2e,
                          int table_mode, int shell_coul, int remove_mean, double* force_out,
                          const int64_t* sp_off = nullptr, const int32_t* sp_ids = nullptr,
                          const double* sp_w = nullptr, int sum_mode = 1) {
  Grid<Real> g = make_grid<Real>(lo, hi, cutoff, rs);
  const Real rc = (Real)cutoff, r_s = (Real)rs, a = (Real)alpha;
  const int64_t row = core_cap + shell_cap;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    const Real* pi = pos + 3 * i;
    int ti = type ? type[i] : 0;
    int64_t mi = mol ? mol[i] : i;
    const Real eps_i = (Real)eps[ti], sig_i = (Real)sig[ti];
    const Real qi = charge ? (Real)charge[i] : (Real)0;
    double lj[3] = {0, 0, 0}, el[3] = {0, 0, 0};
    // sum_mode 0: the reference's accumulators in Real (core LJ, shell LJ, core Coulomb, shell
    // Coulomb), combined as (core + shell LJ) + qqr2e (core + shell Coulomb)
    // (ComputeNearForceRBLERFWorklet, RunWorklet.cpp:754-812)
    Real acc[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    auto pair = [&](int64_t slot, bool shell) {
      const int j = ids[i * row + slot];
      Real off[3];
      shift_offset(g, codes[i * row + slot], off);
      Real pj[3] = {pos[3 * j] - off[0], pos[3 * j + 1] - off[1], pos[3 * j + 2] - off[2]};
      const int tj = type ? type[j] : 0;
      const int64_t mj = mol ? mol[j] : j;
      Real rm[3];
      min_dist(pj, pi, g.box, rm);
      if (with_coul && (!shell || shell_coul)) {
        const Real qj = charge ? (Real)charge[j] : (Real)0;
        Real r[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
        const Real d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        const Real dis = (Real)std::sqrt(d2);
        const Real dism = (Real)std::sqrt(rm[0] * rm[0] + rm[1] * rm[1] + rm[2] * rm[2]);
        bool ok = shell ? (d2 < rc * rc && d2 > r_s * r_s) : (d2 < rc * rc && (double)d2 > 0.0001);
        if (ok) {
          Real gv;
          if (table_mode) gv = (Real)rbl_table_g((float)dism);
          else gv = sizeof(Real) == 4 ? gnear<Real>(a, dism) : gnear_fp64<Real>(a, dism);
          const Real sc = -qi * qj * gv;
          const Real w = shell ? (Real)pice : (Real)1;
          for (int d = 0; d < 3; ++d) {
            if (sum_mode == 0) acc[shell ? 3 : 2][d] += w * (sc * r[d] / dis);
            else el[d] += (double)(w * (sc * r[d] / dis));
          }
        }
      }
      if (!sp_off && mi == mj) return;
      Real f[3] = {0, 0, 0};
      if (!shell) {
        lj_force(rm, eps_i, (Real)eps[tj], sig_i, (Real)sig[tj], rc, f);
      } else {
        const Real d2 = rm[0] * rm[0] + rm[1] * rm[1] + rm[2] * rm[2];
        if (d2 < rc * rc && d2 > r_s * r_s) {
          Real sg = (sig_i + (Real)sig[tj]) / 2;
          Real s6 = sg * sg * sg * sg * sg * sg;
          Real d6 = d2 * d2 * d2;
          Real sd6 = s6 / d6;
          Real scal = (Real)(-24) * (Real)std::sqrt(eps_i * (Real)eps[tj]) * (((Real)2 * sd6 - (Real)1) * sd6) / d2;
          for (int d = 0; d < 3; ++d) f[d] = (Real)pice * (scal * rm[d]);
        }
      }
      if (sp_off) {
        const Real w = (Real)special_weight(sp_off, sp_ids, sp_w, i, j);
        for (int d = 0; d < 3; ++d) f[d] = w * f[d];
      }
      for (int d = 0; d < 3; ++d) {
        if (sum_mode == 0) acc[shell ? 1 : 0][d] += f[d];
        else lj[d] += (double)f[d];
      }
    };
    for (int32_t p = 0; p < std::min<int64_t>(ncore[i], core_cap); ++p) pair(p, false);
    for (int32_t p = 0; p < std::min<int64_t>(nshell[i], shell_cap); ++p) pair(core_cap + p, true);
    for (int d = 0; d < 3; ++d)
      force_out[3 * i + d] = sum_mode == 0
          ? (double)((acc[0][d] + acc[1][d]) + (Real)qqr2e * (acc[2][d] + acc[3][d]))
          : lj[d] + qqr2e * el[d];
  }
  if (remove_mean) {
    double m[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) m[d] += force_out[3 * i + d];
    for (int64_t i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) force_out[3 * i + d] -= m[d] / (double)n;
  }
}

template <class Real>
static int rbl_eam_impl(const char* path, int64_t n, const Real* pos, const double* lo, const double* hi,
                        double cutoff, double rs, int64_t pice, int64_t core_cap, int64_t shell_cap,
                        const int32_t* ncore, const int32_t* nshell, const int32_t* ids,
                        const int32_t* codes, int remove_mean, double* fp_out, double* force_out) {
  EamTables t;
  int rc0 = eam_load(path, t);
  if (rc0) return rc0;
  Grid<Real> g = make_grid<Real>(lo, hi, cutoff, rs);
  const Real rc = (Real)cutoff, r_s = (Real)rs;
  const int64_t row = core_cap + shell_cap;
  std::vector<Real> fp(n);
  const Real rdr = (Real)1 / (Real)t.dr, rdrho = (Real)1 / (Real)t.drho;
  auto C = [&](const std::vector<float>& s, int64_t m, int c) -> Real { return (Real)s[7 * m + c]; };
  auto pj_of = [&](int64_t i, int64_t slot, Real* pj) {
    const int j = ids[i * row + slot];
    Real off[3];
    shift_offset(g, codes[i * row + slot], off);
    for (int d = 0; d < 3; ++d) pj[d] = pos[3 * j + d] - off[d];
    return j;
  };
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    double rhod = 0;
    for (int pass = 0; pass < 2; ++pass) {
      const int64_t cnt = pass == 0 ? std::min<int64_t>(ncore[i], core_cap) : std::min<int64_t>(nshell[i], shell_cap);
      for (int64_t p = 0; p < cnt; ++p) {
        Real pj[3];
        pj_of(i, pass == 0 ? p : core_cap + p, pj);
        Real r[3];
        min_dist(pos + 3 * i, pj, g.box, r);
        const Real rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        const bool ok = pass == 0 ? (rsq < rc * rc && (double)rsq > 0.01) : (rsq < rc * rc && rsq > r_s * r_s);
        if (!ok) continue;
        double pp = (double)((Real)std::sqrt(rsq) * rdr) + 1.0;
        int64_t m = std::min<int64_t>((int64_t)pp, t.nr - 1);
        pp -= (double)m;
        pp = std::min(pp, 1.0);
        Real v = (Real)(((C(t.rhor_spl, m, 3) * pp + C(t.rhor_spl, m, 4)) * pp + C(t.rhor_spl, m, 5)) * pp +
                        C(t.rhor_spl, m, 6));
        rhod += pass == 0 ? (double)v : (double)((Real)pice * v);
      }
    }
    const Real rr = (Real)rhod;
    double pp = (double)(rr * rdrho) + 1.0;
    int m = std::max(1, std::min((int)pp, t.nrho - 1));
    pp -= m;
    pp = std::min(pp, 1.0);
    fp[i] = (Real)((C(t.frho_spl, m, 0) * pp + C(t.frho_spl, m, 1)) * pp + C(t.frho_spl, m, 2));
    if (fp_out) fp_out[i] = (double)fp[i];
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    double acc[3] = {0, 0, 0};
    for (int pass = 0; pass < 2; ++pass) {
      const int64_t cnt = pass == 0 ? std::min<int64_t>(ncore[i], core_cap) : std::min<int64_t>(nshell[i], shell_cap);
      for (int64_t p = 0; p < cnt; ++p) {
        Real pj[3];
        const int j = pj_of(i, pass == 0 ? p : core_cap + p, pj);
        Real r[3];
        min_dist(pos + 3 * i, pj, g.box, r);   // MinDistanceVec(p_i, p_j) (RunWorklet.cpp:1180)
        const Real rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        const bool ok = pass == 0 ? (rsq < rc * rc && (double)rsq > 0.01) : (rsq < rc * rc && rsq > r_s * r_s);
        if (!ok) continue;
        Real rv = (Real)std::sqrt(rsq);
        double pp = (double)(rv * rdr) + 1.0;
        int m = std::min((int)pp, t.nr - 1);
        pp -= m;
        pp = std::min(pp, 1.0);
        double rhop = (C(t.rhor_spl, m, 0) * pp + C(t.rhor_spl, m, 1)) * pp + C(t.rhor_spl, m, 2);
        double z2p = (C(t.z2r_spl, m, 0) * pp + C(t.z2r_spl, m, 1)) * pp + C(t.z2r_spl, m, 2);
        double z2 = ((C(t.z2r_spl, m, 3) * pp + C(t.z2r_spl, m, 4)) * pp + C(t.z2r_spl, m, 5)) * pp +
                    C(t.z2r_spl, m, 6);
        double recip = 1.0 / (double)rv;
        double phi = z2 * recip;
        double phip = z2p * recip - phi * recip;
        double psip = (double)fp[i] * rhop + (double)fp[j] * rhop + phip;
        double fpair = -psip * recip;
        for (int d = 0; d < 3; ++d) {
          Real f = (Real)((double)r[d] * fpair);
          acc[d] += pass == 0 ? (double)f : (double)((Real)pice * f);
        }
      }
    }
    for (int d = 0; d < 3; ++d) force_out[3 * i + d] = acc[d];
  }
  if (remove_mean) {
    double mm[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) mm[d] += force_out[3 * i + d];
    for (int64_t i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) force_out[3 * i + d] -= mm[d] / (double)n;
  }
  return 0;
}

template <class Real>
static void rbl_list_impl(int64_t n, const Real* pos, const double* lo, const double* hi, double cutoff,
                          double rs, int64_t pice, int64_t core_cap, int64_t shell_cap, int32_t* ncore,
                          int32_t* nshell, int32_t* ids, int32_t* codes) {
  Grid<Real> g = make_grid<Real>(lo, hi, cutoff, rs);
  Cells<Real> c = build_cells(g, n, pos);
  rbl_list(g, c, n, pos, cutoff, rs, pice, core_cap, shell_cap, ncore, nshell, ids, codes);
}

EXPORT void oracle_rbl_sizes(int64_t n, const double* lo, const double* hi, double rs, double rc,
                             double sample_num, int eam, int fp64, int64_t* out) {
  RblSizes z;
  if (fp64) {
    double box[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    z = rbl_sizes<double>(n, box, rs, rc, sample_num, eam != 0);
  } else {
    float box[3] = {(float)hi[0] - (float)lo[0], (float)hi[1] - (float)lo[1], (float)hi[2] - (float)lo[2]};
    z = rbl_sizes<float>(n, box, rs, rc, sample_num, eam != 0);
  }
  out[0] = z.rs_num; out[1] = z.rc_num; out[2] = z.pice_num;
}
EXPORT void oracle_rbl_list_f32(int64_t n, const float* pos, const double* lo, const double* hi, double cutoff,
                                double rs, int64_t pice, int64_t core_cap, int64_t shell_cap, int32_t* ncore,
                                int32_t* nshell, int32_t* ids, int32_t* codes) {
  rbl_list_impl<float>(n, pos, lo, hi, cutoff, rs, pice, core_cap, shell_cap, ncore, nshell, ids, codes);
}
EXPORT void oracle_rbl_list_f64(int64_t n, const double* pos, const double* lo, const double* hi, double cutoff,
                                double rs, int64_t pice, int64_t core_cap, int64_t shell_cap, int32_t* ncore,
                                int32_t* nshell, int32_t* ids, int32_t* codes) {
  rbl_list_impl<double>(n, pos, lo, hi, cutoff, rs, pice, core_cap, shell_cap, ncore, nshell, ids, codes);
}
EXPORT float oracle_rbl_table_g(float dis) { return rbl_table_g(dis); }
EXPORT void oracle_rbl_near_f32(int64_t n, const float* pos, const double* lo, const double* hi, double cutoff,
                                double rs, int64_t pice, const int32_t* type, const int32_t* mol,
                                const double* charge, const double* eps, const double* sig, int64_t core_cap,
                                int64_t shell_cap, const int32_t* ncore, const int32_t* nshell,
                                const int32_t* ids, const int32_t* codes, int with_coul, double alpha,
                                double qqr2e, int table_mode, int shell_coul, int remove_mean, double* out) {
  rbl_near_impl<float>(n, pos, lo, hi, cutoff, rs, pice, type, mol, charge, eps, sig, core_cap, shell_cap,
                       ncore, nshell, ids, codes, with_coul, alpha, qqr2e, table_mode, shell_coul,
                       remove_mean, out);
}
// The same in the reference's float accumulation order (the worklet's four accumulators).
EXPORT void oracle_rbl_near_ref_f32(int64_t n, const float* pos, const double* lo, const double* hi, double cutoff,
                                    double rs, int64_t pice, const int32_t* type, const int32_t* mol,
                                    const double* charge, const double* eps, const double* sig, int64_t core_cap,
                                    int64_t shell_cap, const int32_t* ncore, const int32_t* nshell,
                                    const int32_t* ids, const int32_t* codes, int with_coul, double alpha,
                                    double qqr2e, int table_mode, int shell_coul, int remove_mean, double* out) {
  rbl_near_impl<float>(n, pos, lo, hi, cutoff, rs, pice, type, mol, charge, eps, sig, core_cap, shell_cap,
                       ncore, nshell, ids, codes, with_coul, alpha, qqr2e, table_mode, shell_coul,
                       remove_mean, out, nullptr, nullptr, nullptr, 0);
}
EXPORT void oracle_rbl_near_f64(int64_t n, const double* pos, const double* lo, const double* hi, double cutoff,
                                double rs, int64_t pice, const int32_t* type, const int32_t* mol,
                                const double* charge, const double* eps, const double* sig, int64_t core_cap,
                                int64_t shell_cap, const int32_t* ncore, const int32_t* nshell,
                                const int32_t* ids, const int32_t* codes, int with_coul, double alpha,
                                double qqr2e, int table_mode, int shell_coul, int remove_mean, double* out) {
  rbl_near_impl<double>(n, pos, lo, hi, cutoff, rs, pice, type, mol, charge, eps, sig, core_cap, shell_cap,
                        ncore, nshell, ids, codes, with_coul, alpha, qqr2e, table_mode, shell_coul,
                        remove_mean, out);
}
// RBL near force with special-bond LJ weights (ComputeNearForceRBLERFSpecialBondsWorklet,
// RunWorklet.cpp:816-933): no same-molecule exclusion, the LJ pair force times its weight.
EXPORT void oracle_rbl_near_sp_f32(int64_t n, const float* pos, const double* lo, const double* hi, double cutoff,
                                   double rs, int64_t pice, const int32_t* type, const double* charge,
                                   const double* eps, const double* sig, int64_t core_cap, int64_t shell_cap,
                                   const int32_t* ncore, const int32_t* nshell, const int32_t* ids,
                                   const int32_t* codes, int with_coul, double alpha, double qqr2e, int table_mode,
                                   int shell_coul, int remove_mean, const int64_t* sp_off, const int32_t* sp_ids,
                                   const double* sp_w, double* out) {
  rbl_near_impl<float>(n, pos, lo, hi, cutoff, rs, pice, type, nullptr, charge, eps, sig, core_cap, shell_cap,
                       ncore, nshell, ids, codes, with_coul, alpha, qqr2e, table_mode, shell_coul, remove_mean,
                       out, sp_off, sp_ids, sp_w);
}
EXPORT void oracle_rbl_near_sp_f64(int64_t n, const double* pos, const double* lo, const double* hi, double cutoff,
                                   double rs, int64_t pice, const int32_t* type, const double* charge,
                                   const double* eps, const double* sig, int64_t core_cap, int64_t shell_cap,
                                   const int32_t* ncore, const int32_t* nshell, const int32_t* ids,
                                   const int32_t* codes, int with_coul, double alpha, double qqr2e, int table_mode,
                                   int shell_coul, int remove_mean, const int64_t* sp_off, const int32_t* sp_ids,
                                   const double* sp_w, double* out) {
  rbl_near_impl<double>(n, pos, lo, hi, cutoff, rs, pice, type, nullptr, charge, eps, sig, core_cap, shell_cap,
                        ncore, nshell, ids, codes, with_coul, alpha, qqr2e, table_mode, shell_coul, remove_mean,
                        out, sp_off, sp_ids, sp_w);
}

EXPORT int oracle_rbl_eam_f32(const char* path, int64_t n, const float* pos, const double* lo, const double* hi,
                              double cutoff, double rs, int64_t pice, int64_t core_cap, int64_t shell_cap,
                              const int32_t* ncore, const int32_t* nshell, const int32_t* ids,
                              const int32_t* codes, int remove_mean, double* fp_out, double* force_out) {
  return rbl_eam_impl<float>(path, n, pos, lo, hi, cutoff, rs, pice, core_cap, shell_cap, ncore, nshell, ids,
                             codes, remove_mean, fp_out, force_out);
}
EXPORT int oracle_rbl_eam_f64(const char* path, int64_t n, const double* pos, const double* lo, const double* hi,
                              double cutoff, double rs, int64_t pice, int64_t core_cap, int64_t shell_cap,
                              const int32_t* ncore, const int32_t* nshell, const int32_t* ids,
                              const int32_t* codes, int remove_mean, double* fp_out, double* force_out) {
  return rbl_eam_impl<double>(path, n, pos, lo, hi, cutoff, rs, pice, core_cap, shell_cap, ncore, nshell, ids,
                              codes, remove_mean, fp_out, force_out);
}
