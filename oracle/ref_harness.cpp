// ref_harness.cpp -- RBMD's own force-path code, compiled from the reference tree on the host,
// behind a C ABI, so that the oracle's restatement can be checked against the reference's code
// on identical inputs.  Test infrastructure only: nothing in the library links or loads it.
//
// What is compiled from the reference (rbmd/framework, by oracle/build_ref.sh, against the
// VTK-m stand-in in oracle/ref_shim):
//   * ExecForceFunction (forceFunction/ExecForceFunction.h): LJ, erfc Coulomb, RBE terms and
//     normaliser, EAM spline terms;
//   * ExecPointLocator (locator/ExecPointLocator.h): cells, periodic offsets, MinDistanceVec;
//   * ContPointLocator's grid setters (locator/ContPointLocator.h:44-73) and its
//     BinPointsWorklet (locator/ContPointLocator.cxx:38-66);
//   * ExecTopology (topology/ExecTopology.h), ExecStaticTable (staticTable/ExecStaticTable.h)
//     with the ERF table arrays of model/ERFTable.h, loaded as ExecutionMD::InitERF does;
//   * RBEPSAMPLE (model/RBEPSample.h) with its uniforms injected (RandomValue below replaces
//     math/Utiles.h's std::random_device draw);
//   * every worklet struct of run/worklet/RunWorklet.cpp (lines 40-1913), called here through
//     operator() with the arguments their ExecutionSignature lists.
// What is written here (VTK-m's control-side algorithms, which are not in the reference tree):
// the stable SortByKey of points by cell id (points of a cell in ascending id), Lower/Upper
// bounds per cell, the ReduceByKey of the structure-factor terms (summed per k in FP64 in atom
// order), and the loops that map a worklet over atoms.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <vector>

#include "Types.h"   // rbmd/framework/Types.h: Real = vtkm::FloatDefault (float), Id = int32

// Injected uniform stream for RBEPSAMPLE: every RandomValue<T>(0, 1) call takes the next value.
namespace ref_rng {
thread_local const double* stream = nullptr;
thread_local int64_t next = 0;
thread_local int64_t size = 0;
}  // namespace ref_rng
template <typename T>
T RandomValue(const Real& lo, const Real& hi) {
  const double u = ref_rng::next < ref_rng::size ? ref_rng::stream[ref_rng::next] : 0.5;
  ++ref_rng::next;
  return static_cast<T>(lo + (hi - lo) * u);
}

#include "forceFunction/ExecForceFunction.h"
#include "locator/ExecPointLocator.h"
#include "model/RBEPSample.h"
#include "staticTable/ExecStaticTable.h"
#include "topology/ExecTopology.h"
#include "model/ERFTable.h"   // the RBL Coulomb table arrays (ExecutionMD::InitERF loads them)
// ContPointLocator's members are private; its setters hold the reference's grid formula
#define private public
#include "locator/ContPointLocator.h"
#undef private
#include <vtkm/worklet/WorkletMapField.h>

namespace ref_bin {
#include "bin_points.inc"   // class BinPointsWorklet (ContPointLocator.cxx:38-66)
}
#include "run_worklets.inc"  // namespace RunWorklet { every worklet struct }

#define EXPORT extern "C" __attribute__((visibility("default")))

namespace {

using IdPortal = vtkm::cont::ArrayHandle<vtkm::Id>::ReadPortalType;

template <typename T>
typename vtkm::cont::ArrayHandle<T>::ReadPortalType portal(const std::vector<T>& v) {
  return {v.data(), (vtkm::Id)v.size()};
}

// a list row handed to a worklet: ids or offsets of one atom (FieldIn / FieldInOut groups)
template <typename T>
struct Row {
  T* p;
  T& operator[](vtkm::Id i) const { return p[i]; }
};

struct Grid {
  vtkm::Vec3f lo, hi;
  Real cut, rs;
  vtkm::Id3 dims;
  vtkm::Id num_cycles;
};

// ContPointLocator::SetRs / SetCutOff / SetRange (ContPointLocator.h:44-73), in that order
Grid make_grid(const double* lo, const double* hi, double cut, double rs) {
  ContPointLocator c;
  c.SetRs((Real)rs);
  c.SetCutOff((Real)cut);
  c.SetRange(vtkm::Vec3f((Real)lo[0], (Real)lo[1], (Real)lo[2]), vtkm::Vec3f((Real)hi[0], (Real)hi[1], (Real)hi[2]));
  Grid g;
  g.lo = c._left_bottom;
  g.hi = c._right_top;
  g.cut = c._cut_off;
  g.rs = c._rs;
  g.dims = c._dims;
  g.num_cycles = c._num_cycles;
  return g;
}

struct Cells {
  std::vector<vtkm::Id> point_ids, lower, upper;
};

// ContPointLocator::Build (ContPointLocator.cxx:68-92): BinPointsWorklet per point, then
// SortByKey (stable here), Lower/UpperBounds per cell id
Cells build_cells(const Grid& g, const std::vector<vtkm::Vec3f>& pos) {
  const vtkm::Id n = (vtkm::Id)pos.size();
  ref_bin::internal::BinPointsWorklet bin(g.lo, g.hi, g.dims);
  std::vector<vtkm::Id> key(n);
  for (vtkm::Id i = 0; i < n; ++i) bin(pos[i], key[i]);
  Cells c;
  c.point_ids.resize(n);
  std::iota(c.point_ids.begin(), c.point_ids.end(), 0);
  std::stable_sort(c.point_ids.begin(), c.point_ids.end(), [&](vtkm::Id a, vtkm::Id b) { return key[a] < key[b]; });
  std::vector<vtkm::Id> sorted(n);
  for (vtkm::Id i = 0; i < n; ++i) sorted[i] = key[c.point_ids[i]];
  const vtkm::Id ncell = g.dims[0] * g.dims[1] * g.dims[2];
  c.lower.resize(ncell);
  c.upper.resize(ncell);
  for (vtkm::Id k = 0; k < ncell; ++k) {
    c.lower[k] = (vtkm::Id)(std::lower_bound(sorted.begin(), sorted.end(), k) - sorted.begin());
    c.upper[k] = (vtkm::Id)(std::upper_bound(sorted.begin(), sorted.end(), k) - sorted.begin());
  }
  return c;
}

ExecPointLocator make_locator(const Grid& g, const Cells& c, const std::vector<vtkm::Vec3f>& pos) {
  return ExecPointLocator(g.lo, g.hi, g.cut, g.rs, g.dims, g.num_cycles, 0, portal(c.point_ids), portal(pos),
                          portal(c.lower), portal(c.upper), IdPortal{}, ExecPointLocator::GroupVecPortalType{},
                          ExecPointLocator::CoordOffsetPortalType{});
}

std::vector<vtkm::Vec3f> to_vec3(int64_t n, const float* x) {
  std::vector<vtkm::Vec3f> v((size_t)n);
  for (int64_t i = 0; i < n; ++i) v[i] = vtkm::Vec3f(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
  return v;
}

// ExecForceFunction with the arguments ExecutionMD passes (volume = Lx Ly Lz, vlength = Lx)
ExecForceFunction make_force_function(const Grid& g, double cut, double alpha, int P, double rhomax = 0, int nrho = 0,
                                      double drho = 1, int nr = 0, double dr = 1) {
  const vtkm::Vec3f box = g.hi - g.lo;
  const Real volume = box[0] * box[1] * box[2];
  return ExecForceFunction((Real)cut, (Real)alpha, volume, box[0], box, 0, P, (Real)rhomax, nrho, (Real)drho, nr,
                           (Real)dr);
}

}  // namespace

// Grid of ContPointLocator: dims[3], num_cycles.
EXPORT void ref_grid(const double* lo, const double* hi, double cut, double rs, int32_t* dims, int32_t* num_cycles) {
  Grid g = make_grid(lo, hi, cut, rs);
  for (int d = 0; d < 3; ++d) dims[d] = g.dims[d];
  *num_cycles = g.num_cycles;
}

// Cells of ContPointLocator::Build: point_ids[n], lower/upper[ncell].
EXPORT void ref_cells(int64_t n, const float* pos, const double* lo, const double* hi, double cut, double rs,
                      int32_t* point_ids, int32_t* lower, int32_t* upper) {
  Grid g = make_grid(lo, hi, cut, rs);
  auto p = to_vec3(n, pos);
  Cells c = build_cells(g, p);
  std::copy(c.point_ids.begin(), c.point_ids.end(), point_ids);
  std::copy(c.lower.begin(), c.lower.end(), lower);
  std::copy(c.upper.begin(), c.upper.end(), upper);
}

// ComputeNeighboursWorklet (RunWorklet.cpp:40-96) over every atom: counts[n], ids[n*cap] and the
// periodic coordinate offsets off[n*cap*3] in the reference's traversal order.  Returns the
// largest count (rows beyond cap are truncated).
EXPORT int32_t ref_neighbors(int64_t n, const float* pos, const double* lo, const double* hi, double cut, double rs,
                             int64_t cap, int32_t* counts, int32_t* ids, float* off) {
  Grid g = make_grid(lo, hi, cut, rs);
  auto p = to_vec3(n, pos);
  Cells c = build_cells(g, p);
  ExecPointLocator loc = make_locator(g, c, p);
  RunWorklet::ComputeNeighboursWorklet w((Real)cut);
  int32_t mx = 0;
#pragma omp parallel
  {
    std::vector<vtkm::Id> row_ids((size_t)n);
    std::vector<vtkm::Vec3f> row_off((size_t)n);
#pragma omp for schedule(dynamic, 64) reduction(max : mx)
    for (int64_t i = 0; i < n; ++i) {
      Row<vtkm::Id> ri{row_ids.data()};
      Row<vtkm::Vec3f> ro{row_off.data()};
      vtkm::Id num = 0;
      w((vtkm::Id)i, loc, ri, num, ro);
      counts[i] = num;
      mx = std::max<int32_t>(mx, num);
      for (vtkm::Id k = 0; k < num && k < cap; ++k) {
        ids[i * cap + k] = row_ids[k];
        for (int d = 0; d < 3; ++d) off[(i * cap + k) * 3 + d] = row_off[k][d];
      }
    }
  }
  return mx;
}

// Near force over the lists of ref_neighbors: ComputeNearForceVerletWorklet (with_coul, LJ plus
// erfc Coulomb, RunWorklet.cpp:170-237) or ComputeLJForceVerletWorklet (LJ only, :239-303).
// mol: molecule id per atom (the reference skips LJ within a molecule); eps/sigma per type.
EXPORT void ref_near_force(int64_t n, const float* pos, const double* lo, const double* hi, double cut,
                           const int32_t* type, const int32_t* mol, const float* charge, int ntypes, const float* eps,
                           const float* sigma, double alpha, int with_coul, int64_t cap, const int32_t* counts,
                           const int32_t* ids, const float* off, float* force) {
  Grid g = make_grid(lo, hi, cut, cut);
  auto p = to_vec3(n, pos);
  Cells c = build_cells(g, p);
  ExecPointLocator loc = make_locator(g, c, p);
  std::vector<vtkm::Id> molv(mol, mol + n), typev(type, type + n);
  std::vector<Real> qv(charge, charge + n), ev(eps, eps + ntypes), sv(sigma, sigma + ntypes);
  ExecTopology topo(ExecTopology::GroupIdPortalTypeId{}, portal(molv), portal(typev), portal(qv), portal(ev),
                    portal(sv));
  ExecForceFunction ff = make_force_function(g, cut, alpha, 0);
  const vtkm::Vec3f box = g.hi - g.lo;
  RunWorklet::ComputeNearForceVerletWorklet wc((Real)cut, box);
  RunWorklet::ComputeLJForceVerletWorklet wl((Real)cut, box);
#pragma omp parallel
  {
    std::vector<vtkm::Id> rid((size_t)cap);
    std::vector<vtkm::Vec3f> roff((size_t)cap);
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
      const vtkm::Id num = counts[i];
      for (vtkm::Id k = 0; k < num; ++k) {
        rid[k] = ids[i * cap + k];
        roff[k] = vtkm::Vec3f(off[(i * cap + k) * 3], off[(i * cap + k) * 3 + 1], off[(i * cap + k) * 3 + 2]);
      }
      Row<vtkm::Id> gj{rid.data()};
      Row<vtkm::Vec3f> oj{roff.data()};
      vtkm::Vec3f f;
      if (with_coul)
        wc((vtkm::Id)i, loc, topo, ff, gj, num, oj, f);
      else
        wl((vtkm::Id)i, loc, topo, ff, gj, num, oj, f);
      for (int d = 0; d < 3; ++d) force[3 * i + d] = f[d];
    }
  }
}

// RBE structure factors: ComputePnumberChargeStructureFactorWorklet (RunWorklet.cpp:1616-1677)
// gives the N x P terms q cos(k.r), q sin(k.r); the reduction by key is a sum per k in FP64 in
// atom order.  m[P*3] integer vectors.  rho[P*2] (Re, Im).
EXPORT void ref_rhok(int64_t n, const float* pos, const float* charge, const double* box, int P, const int32_t* m,
                     double* rho) {
  const vtkm::Vec3f b((Real)box[0], (Real)box[1], (Real)box[2]);
  std::vector<vtkm::Vec3f> ps(P);
  for (int l = 0; l < P; ++l) ps[l] = vtkm::Vec3f((Real)m[3 * l], (Real)m[3 * l + 1], (Real)m[3 * l + 2]);
  std::vector<Real> re((size_t)n * P), im((size_t)n * P);
  vtkm::cont::WritePortalT<Real> wre{re.data(), (vtkm::Id)re.size()}, wim{im.data(), (vtkm::Id)im.size()};
  RunWorklet::ComputePnumberChargeStructureFactorWorklet w(b, P, (vtkm::Id)n);
  const auto psp = portal(ps);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const vtkm::Vec3f x(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    w((vtkm::Id)i, x, (Real)charge[i], psp, wre, wim);
  }
  for (int l = 0; l < P; ++l) {
    double a = 0, c = 0;
    for (int64_t i = 0; i < n; ++i) {
      a += (double)re[i + (size_t)l * n];
      c += (double)im[i + (size_t)l * n];
    }
    rho[2 * l] = a;
    rho[2 * l + 1] = c;
  }
}

// RBE force: ComputeNewRBEForceWorklet (RunWorklet.cpp:1508-1548) with ComputeRBEForceSum,
// ComputeRBEForce and Compute_S (ExecForceFunction.h:247-294), before the qqr2e rescale; rho is
// handed in as the reference's Vec2f.  Also returns S.
EXPORT double ref_rbe_force(int64_t n, const float* pos, const float* charge, const double* lo, const double* hi,
                            double alpha, int P, const int32_t* m, const float* rho, float* force) {
  Grid g = make_grid(lo, hi, 1.0, 1.0);
  auto p = to_vec3(n, pos);
  Cells c;   // the worklet reads positions only
  ExecPointLocator loc = make_locator(g, c, p);
  std::vector<vtkm::Id> zi((size_t)n, 0);
  std::vector<Real> qv(charge, charge + n), one(1, 1.0f);
  ExecTopology topo(ExecTopology::GroupIdPortalTypeId{}, portal(zi), portal(zi), portal(qv), portal(one), portal(one));
  ExecForceFunction ff = make_force_function(g, 1.0, alpha, P);
  std::vector<vtkm::Vec3f> ps(P);
  std::vector<vtkm::Vec2f> rk(P);
  for (int l = 0; l < P; ++l) {
    ps[l] = vtkm::Vec3f((Real)m[3 * l], (Real)m[3 * l + 1], (Real)m[3 * l + 2]);
    rk[l] = vtkm::Vec2f(rho[2 * l], rho[2 * l + 1]);
  }
  RunWorklet::ComputeNewRBEForceWorklet w(P);
  const auto psp = portal(ps);
  const auto rkp = portal(rk);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    ExecForceFunction f = ff;
    ExecPointLocator l = loc;
    vtkm::Vec3f out;
    w((vtkm::Id)i, psp, rkp, f, topo, l, out);
    for (int d = 0; d < 3; ++d) force[3 * i + d] = out[d];
  }
  return (double)ff.Compute_S();
}

// EAM over the lists of ref_neighbors: ComputeEAMfpVerletWorklet then
// ComputeEAMForceVerletWorklet (RunWorklet.cpp:305-417) with the spline tables frho/rhor/z2r
// ([rows][7] float, as ExecutionNVT::SetEAM builds them).  fp[n], force[n*3].
EXPORT void ref_eam(int64_t n, const float* pos, const double* lo, const double* hi, double cut, int nrho, double drho,
                    int nr, double dr, double rhomax, const float* frho, int64_t frho_rows, const float* rhor,
                    int64_t rhor_rows, const float* z2r, int64_t z2r_rows, int64_t cap, const int32_t* counts,
                    const int32_t* ids, const float* off, float* fp_out, float* force) {
  Grid g = make_grid(lo, hi, cut, cut);
  auto p = to_vec3(n, pos);
  Cells c = build_cells(g, p);
  ExecPointLocator loc = make_locator(g, c, p);
  ExecForceFunction ff = make_force_function(g, cut, 0.0, 0, rhomax, nrho, drho, nr, dr);
  auto tab = [](const float* t, int64_t rows) {
    std::vector<Vec7f> v((size_t)rows);
    for (int64_t r = 0; r < rows; ++r)
      for (int k = 0; k < 7; ++k) v[r][k] = t[r * 7 + k];
    return v;
  };
  const auto tf = tab(frho, frho_rows), tr = tab(rhor, rhor_rows), tz = tab(z2r, z2r_rows);
  const vtkm::Vec3f box = g.hi - g.lo;
  RunWorklet::ComputeEAMfpVerletWorklet wfp((Real)cut, box);
  RunWorklet::ComputeEAMForceVerletWorklet wf((Real)cut, box);
  std::vector<Real> fp((size_t)n);
  auto run = [&](auto&& body) {
#pragma omp parallel
    {
      std::vector<vtkm::Id> rid((size_t)cap);
      std::vector<vtkm::Vec3f> roff((size_t)cap);
#pragma omp for schedule(dynamic, 64)
      for (int64_t i = 0; i < n; ++i) {
        const vtkm::Id num = counts[i];
        for (vtkm::Id k = 0; k < num; ++k) {
          rid[k] = ids[i * cap + k];
          roff[k] = vtkm::Vec3f(off[(i * cap + k) * 3], off[(i * cap + k) * 3 + 1], off[(i * cap + k) * 3 + 2]);
        }
        body(i, num, Row<vtkm::Id>{rid.data()}, Row<vtkm::Vec3f>{roff.data()});
      }
    }
  };
  const auto tfp = portal(tf), trp = portal(tr), tzp = portal(tz);
  run([&](int64_t i, vtkm::Id num, Row<vtkm::Id> gj, Row<vtkm::Vec3f> oj) {
    Real v;
    wfp((vtkm::Id)i, trp, tfp, loc, ff, gj, num, oj, v);
    fp[i] = v;
  });
  const auto fpp = portal(fp);
  run([&](int64_t i, vtkm::Id num, Row<vtkm::Id> gj, Row<vtkm::Vec3f> oj) {
    vtkm::Vec3f f;
    wf((vtkm::Id)i, trp, tzp, fpp, loc, ff, gj, num, oj, f);
    for (int d = 0; d < 3; ++d) force[3 * i + d] = f[d];
  });
  for (int64_t i = 0; i < n; ++i) fp_out[i] = fp[i];
}

// RBEPSAMPLE::Fetch_P_Sample (model/RBEPSample.h:144-173) with mu = 0 and
// sigma_d = sqrt(alpha / 2) L_d / pi (ExecutionNVT::PreForce), drawing its uniforms from
// `uniforms` in call order (0.5 once exhausted).  random = 0 is the reference's TEST mode
// (U = 0.5 throughout).  m_out[P*3]; returns the number of uniforms consumed.
EXPORT int64_t ref_rbe_sample(double alpha, const double* L, int P, int random, const double* uniforms,
                              int64_t n_uniforms, float* m_out) {
  RBEPSAMPLE s;
  s._alpha = (Real)alpha;
  s._box = vtkm::Vec3f((Real)L[0], (Real)L[1], (Real)L[2]);
  s._Length = (Real)L[0];
  s._P = P;
  s._RBE_random = random != 0;
  vtkm::Vec3f sigma;
  for (int d = 0; d < 3; ++d) sigma[d] = (Real)(std::sqrt(alpha / 2.0) * L[d] / M_PI);
  ref_rng::stream = uniforms;
  ref_rng::size = n_uniforms;
  ref_rng::next = 0;
  auto out = s.Fetch_P_Sample(0.0f, sigma);
  auto rp = out.ReadPortal();
  for (int l = 0; l < P; ++l)
    for (int d = 0; d < 3; ++d) m_out[3 * l + d] = rp.Get(l)[d];
  ref_rng::stream = nullptr;
  return ref_rng::next;
}

// ExecForceFunction::Gnear (ExecForceFunction.h:217-224) on an array of distances (the erfc
// Coulomb kernel of the near pass).
EXPORT void ref_gnear(int64_t n, double alpha, const float* dis, float* g) {
  const double lo[3] = {0, 0, 0}, hi[3] = {10, 10, 10};
  ExecForceFunction ff = make_force_function(make_grid(lo, hi, 1.0, 1.0), 1.0, alpha, 0);
  for (int64_t i = 0; i < n; ++i) g[i] = ff.Gnear((Real)alpha, dis[i]);
}

// RBL list: ComputeRBLNeighboursOnceWorklet (RunWorklet.cpp:634-708) with the reference's row
// layout: core pairs at [0, ncore), every pice-th shell pair at [rs_num, rs_num + nshell).
// ids[n*cap], off[n*cap*3] with cap >= rs_num + the largest nshell; returns the largest
// rs_num + nshell (and ncore) so that the caller can regrow.
EXPORT int32_t ref_rbl_list(int64_t n, const float* pos, const double* lo, const double* hi, double rc, double rs,
                            int32_t rs_num, int32_t pice_num, int64_t cap, int32_t* ncore, int32_t* nshell,
                            int32_t* ids, float* off) {
  Grid g = make_grid(lo, hi, rc, rs);
  auto p = to_vec3(n, pos);
  Cells c = build_cells(g, p);
  ExecPointLocator loc = make_locator(g, c, p);
  RunWorklet::ComputeRBLNeighboursOnceWorklet w(rs_num, pice_num);
  int32_t mx = 0;
#pragma omp parallel
  {
    std::vector<vtkm::Id> rid((size_t)(n + rs_num));
    std::vector<vtkm::Vec3f> roff((size_t)(n + rs_num));
#pragma omp for schedule(dynamic, 64) reduction(max : mx)
    for (int64_t i = 0; i < n; ++i) {
      Row<vtkm::Id> ri{rid.data()};
      Row<vtkm::Vec3f> ro{roff.data()};
      vtkm::Id2 num(0, 0);
      w((vtkm::Id)i, loc, ri, num, ro);
      ncore[i] = num[0];
      nshell[i] = num[1];
      mx = std::max<int32_t>(mx, std::max<int32_t>(num[0], rs_num + num[1]));
      auto put = [&](int64_t k) {
        if (k >= cap) return;
        ids[i * cap + k] = rid[k];
        for (int d = 0; d < 3; ++d) off[(i * cap + k) * 3 + d] = roff[k][d];
      };
      for (vtkm::Id k = 0; k < num[0]; ++k) put(k);
      for (vtkm::Id k = 0; k < num[1]; ++k) put(rs_num + k);
    }
  }
  return mx;
}

// RBL near force over the lists of ref_rbl_list, before the mean removal:
// ComputeNearForceRBLERFWorklet (with_coul; RunWorklet.cpp:710-814, the ERF table G and the
// shell Coulomb term computed and dropped, as the reference) or ComputeLJForceRBLWorklet
// (:1218-1302).
EXPORT void ref_rbl_near(int64_t n, const float* pos, const double* lo, const double* hi, double rc, double rs,
                         int32_t rs_num, int32_t pice_num, double qqr2e, const int32_t* type, const int32_t* mol,
                         const float* charge, int ntypes, const float* eps, const float* sigma, double alpha,
                         int with_coul, int64_t cap, const int32_t* ncore, const int32_t* nshell, const int32_t* ids,
                         const float* off, float* force) {
  Grid g = make_grid(lo, hi, rc, rs);
  auto p = to_vec3(n, pos);
  Cells c = build_cells(g, p);
  ExecPointLocator loc = make_locator(g, c, p);
  std::vector<vtkm::Id> molv(mol, mol + n), typev(type, type + n);
  std::vector<Real> qv(charge, charge + n), ev(eps, eps + ntypes), sv(sigma, sigma + ntypes);
  ExecTopology topo(ExecTopology::GroupIdPortalTypeId{}, portal(molv), portal(typev), portal(qv), portal(ev),
                    portal(sv));
  ExecForceFunction ff = make_force_function(g, rc, alpha, 0);
  ExecStaticTable table(portal(erf_index_leq2_v), portal(erf_dis_leq2_v), portal(erf_dis_dif_leq2_v),
                        portal(erf_gnear_leq2_v), portal(erf_gnear_der_leq2_v), portal(erf_index_geq2_v),
                        portal(erf_dis_geq2_v), portal(erf_dis_dif_geq2_v), portal(erf_gnear_geq2_v),
                        portal(erf_gnear_der_geq2_v));
  const vtkm::Vec3f box = g.hi - g.lo;
  RunWorklet::ComputeNearForceRBLERFWorklet we(rs_num, pice_num, (Real)qqr2e, box);
  RunWorklet::ComputeLJForceRBLWorklet wl(rs_num, pice_num, box);
#pragma omp parallel
  {
    std::vector<vtkm::Id> rid((size_t)cap);
    std::vector<vtkm::Vec3f> roff((size_t)cap);
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
      for (int64_t k = 0; k < cap; ++k) {
        rid[k] = ids[i * cap + k];
        roff[k] = vtkm::Vec3f(off[(i * cap + k) * 3], off[(i * cap + k) * 3 + 1], off[(i * cap + k) * 3 + 2]);
      }
      Row<vtkm::Id> gj{rid.data()};
      Row<vtkm::Vec3f> oj{roff.data()};
      const vtkm::Id2 num(ncore[i], nshell[i]);
      vtkm::Vec3f f;
      if (with_coul)
        we((vtkm::Id)i, loc, topo, ff, table, gj, num, oj, f);
      else
        wl((vtkm::Id)i, loc, topo, ff, gj, num, oj, f);
      for (int d = 0; d < 3; ++d) force[3 * i + d] = f[d];
    }
  }
}

// The RBL Coulomb table lookup: ExecStaticTable::Extract + TableGnearValue (ExecStaticTable.h:
// 96-135) over the arrays of model/ERFTable.h, for each float distance.
EXPORT void ref_erf_table(int64_t n, const float* dis, float* g) {
  ExecStaticTable table(portal(erf_index_leq2_v), portal(erf_dis_leq2_v), portal(erf_dis_dif_leq2_v),
                        portal(erf_gnear_leq2_v), portal(erf_gnear_der_leq2_v), portal(erf_index_geq2_v),
                        portal(erf_dis_geq2_v), portal(erf_dis_dif_geq2_v), portal(erf_gnear_geq2_v),
                        portal(erf_gnear_der_geq2_v));
  for (int64_t i = 0; i < n; ++i) {
    IdComponent k = table.Extract(dis[i]);
    g[i] = table.TableGnearValue(dis[i], k);
  }
}

// The ORIGINAL neighbour type's EAM (ExecutionMD::ComputeOriginalEAMForce,
// rbmd/framework/run/ExecutionMD.cpp:863-893): ComputeEAMrhoWorklet, ComputeEAMfpWorklet and
// ComputeEAMforceWorklet (RunWorklet.cpp:419-524), each walking the cells on the fly
// (ExecPointLocator::ExecuteOnNeighbor).  fp[n], force[n*3].
EXPORT void ref_eam_original(int64_t n, const float* pos, const double* lo, const double* hi, double cut, int nrho,
                             double drho, int nr, double dr, double rhomax, const float* frho, int64_t frho_rows,
                             const float* rhor, int64_t rhor_rows, const float* z2r, int64_t z2r_rows, float* fp_out,
                             float* force) {
  Grid g = make_grid(lo, hi, cut, cut);
  auto p = to_vec3(n, pos);
  Cells c = build_cells(g, p);
  ExecPointLocator loc = make_locator(g, c, p);
  std::vector<vtkm::Id> zi((size_t)n, 0);
  std::vector<Real> zr((size_t)n, 0.0f), one(1, 1.0f);
  ExecTopology topo(ExecTopology::GroupIdPortalTypeId{}, portal(zi), portal(zi), portal(zr), portal(one), portal(one));
  ExecForceFunction ff = make_force_function(g, cut, 0.0, 0, rhomax, nrho, drho, nr, dr);
  auto tab = [](const float* t, int64_t rows) {
    std::vector<Vec7f> v((size_t)rows);
    for (int64_t r = 0; r < rows; ++r)
      for (int k = 0; k < 7; ++k) v[r][k] = t[r * 7 + k];
    return v;
  };
  const auto tf = tab(frho, frho_rows), tr = tab(rhor, rhor_rows), tz = tab(z2r, z2r_rows);
  const auto tfp = portal(tf), trp = portal(tr), tzp = portal(tz);
  const vtkm::Vec3f box = g.hi - g.lo;
  RunWorklet::ComputeEAMrhoWorklet wr((Real)cut, box);
  RunWorklet::ComputeEAMfpWorklet wfp;
  RunWorklet::ComputeEAMforceWorklet wf((Real)cut, box);
  std::vector<Real> rho((size_t)n), fp((size_t)n);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) wr((vtkm::Id)i, trp, loc, topo, ff, rho[i]);
  const auto rhop = portal(rho);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) wfp((vtkm::Id)i, rhop, tfp, loc, topo, ff, fp[i]);
  const auto fpp = portal(fp);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    vtkm::Vec3f f;
    wf((vtkm::Id)i, fpp, trp, tzp, loc, topo, ff, f);
    for (int d = 0; d < 3; ++d) force[3 * i + d] = f[d];
  }
  for (int64_t i = 0; i < n; ++i) fp_out[i] = fp[i];
}
