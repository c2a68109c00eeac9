// eam_funcfl.hpp -- host-side funcfl and setfl readers and the 7-coefficient spline build.
//
// Follows ExecutionNVT::ReadPotentialFile / file2array / interpolate / array2spline
// (rbmd/framework/run/ExecutionNVT.cpp:903-1107), which is LAMMPS pair_eam's published
// funcfl procedure with two reference-specific details kept for parity: the file arrays are
// read 0-based but interpolated with 1-based indices (k-1 .. k+2), and rho(r) is read with the
// nrho count.  Arithmetic mirrors the reference's float storage (Real = float).
#pragma once
#include <algorithm>
#include <fstream>
#include <limits>
#include <string>
#include <vector>

namespace rbmd {

struct FuncflTables {
  int nrho = 0, nr = 0;
  float drho = 0, dr = 0, rhomax = 0, cut = 0;
  std::vector<float> frho, rhor, z2r;   // 7 floats per row, rows 0..n
};

inline void funcfl_interpolate(int n, float delta, const std::vector<float>& f, std::vector<float>& s) {
  s.assign(7 * (size_t)(n + 1), 0.0f);
  auto S = [&](int m, int c) -> float& { return s[7 * (size_t)m + c]; };
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

// returns 0 on success
inline int funcfl_load(const std::string& path, FuncflTables& t) {
  std::ifstream in(path);
  if (!in.is_open()) return 1;
  for (int i = 0; i < 2; ++i) in.ignore(std::numeric_limits<std::streamsize>::max(), '\n');
  int fnrho = 0, fnr = 0;
  float fdrho = 0, fdr = 0, fcut = 0;
  in >> fnrho >> fdrho >> fnr >> fdr >> fcut;
  if (!in || fnrho < 5 || fnr < 5) return 2;
  std::vector<float> ffrho(fnrho + 1), fzr(fnr + 1), frhor(std::max(fnrho, fnr) + 1);
  for (int i = 0; i < fnrho; ++i) in >> ffrho[i];
  for (int i = 0; i < fnr; ++i) in >> fzr[i];
  for (int i = 0; i < fnrho; ++i) in >> frhor[i];
  if (!in) return 3;
  const float sixth = (float)(1.0 / 6.0);
  const float dr = std::max(0.0f, fdr), drho = std::max(0.0f, fdrho);
  const float rmax = std::max(0.0f, (float)(fnr - 1) * fdr);
  const float rhomax = std::max(0.0f, (float)(fnrho - 1) * fdrho);
  const int nr = (int)(rmax / dr + 0.5);
  const int nrho = (int)(rhomax / drho + 0.5);
  std::vector<float> frho(nrho + 1, 0.f), rhor(std::max(nrho, nr) + 1, 0.f), z2r(nr + 1, 0.f);
  auto lagrange = [&](float p, float* c) {
    c[0] = (float)(-sixth * p * (p - 1.0) * (p - 2.0));
    c[1] = (float)(0.5 * (p * p - 1.0) * (p - 2.0));
    c[2] = (float)(-0.5 * p * (p + 1.0) * (p - 2.0));
    c[3] = (float)(sixth * p * (p * p - 1.0));
  };
  auto knot = [](float r, float step, int nfile, float& p) {
    p = (float)(r / step + 1.0);
    int k = (int)p;
    k = std::min(k, nfile - 2);
    k = std::max(k, 2);
    p -= (float)k;
    p = std::min(p, 2.0f);
    return k;
  };
  for (int m = 1; m <= nrho; m++) {
    float p;
    const int k = knot((float)(m - 1) * drho, fdrho, fnrho, p);
    float c[4];
    lagrange(p, c);
    frho[m] = c[0] * ffrho[k - 1] + c[1] * ffrho[k] + c[2] * ffrho[k + 1] + c[3] * ffrho[k + 2];
  }
  for (int m = 1; m <= nr; m++) {
    float p;
    const int k = knot((float)(m - 1) * dr, fdr, fnr, p);
    // the rho(r) loop declares its coefficients `auto`, which makes them double
    const double d0 = -sixth * p * (p - 1.0) * (p - 2.0);   // (-sixth * p) is a float product
    const double d1 = 0.5 * (p * p - 1.0) * (p - 2.0);
    const double d2 = -0.5 * p * (p + 1.0) * (p - 2.0);
    const double d3 = sixth * p * (p * p - 1.0);
    rhor[m] = (float)(d0 * frhor[k - 1] + d1 * frhor[k] + d2 * frhor[k + 1] + d3 * frhor[k + 2]);
  }
  for (int m = 1; m <= nr; m++) {
    float p;
    const int k = knot((float)(m - 1) * dr, fdr, fnr, p);
    float c[4];
    lagrange(p, c);
    // float coefficients times float data, summed in float, then widened
    const float zf = c[0] * fzr[k - 1] + c[1] * fzr[k] + c[2] * fzr[k + 1] + c[3] * fzr[k + 2];
    const double zri = (double)zf;
    z2r[m] = (float)(27.2 * 0.529 * zri * zri);
  }
  t.nrho = nrho;
  t.nr = nr;
  t.drho = drho;
  t.dr = dr;
  t.rhomax = rhomax;
  t.cut = fcut;
  funcfl_interpolate(nrho, drho, frho, t.frho);
  funcfl_interpolate(nr, dr, rhor, t.rhor);
  funcfl_interpolate(nr, dr, z2r, t.z2r);
  return 0;
}

// setfl (LAMMPS eam/alloy) reader for the single-element EAM path: header of three comment lines,
// "N el_1 .. el_N", "nrho drho nr dr cut", per element a line (number, mass, lattice constant,
// lattice) then F(rho)[nrho] and rho(r)[nr], then r*phi_ij(r)[nr] for i >= j.  The tables are
// used on the file's own grids (LAMMPS' file2array copies setfl arrays without resampling), with
// z2r = r*phi of the first element's self pair; `element` picks another element (0-based).
// The reference reads funcfl files only (ExecutionNVT.cpp:903-1107): this reader widens the
// inputs a drop-in user can bring, and shares funcfl_interpolate and the device path.
inline int setfl_load(const std::string& path, FuncflTables& t, int element = 0) {
  std::ifstream in(path);
  if (!in.is_open()) return 1;
  for (int i = 0; i < 3; ++i) in.ignore(std::numeric_limits<std::streamsize>::max(), '\n');
  int nel = 0;
  in >> nel;
  if (!in || nel < 1 || element < 0 || element >= nel) return 2;
  in.ignore(std::numeric_limits<std::streamsize>::max(), '\n');   // element names
  int nrho = 0, nr = 0;
  float drho = 0, dr = 0, cut = 0;
  in >> nrho >> drho >> nr >> dr >> cut;
  if (!in || nrho < 5 || nr < 5 || !(drho > 0) || !(dr > 0)) return 2;
  std::vector<float> frho(nrho + 1, 0.f), rhor(nr + 1, 0.f), z2r(nr + 1, 0.f);
  for (int e = 0; e < nel; ++e) {
    double num, mass, lat;
    std::string lattice;
    in >> num >> mass >> lat >> lattice;
    for (int m = 1; m <= nrho; ++m) {
      float v;
      in >> v;
      if (e == element) frho[m] = v;
    }
    for (int m = 1; m <= nr; ++m) {
      float v;
      in >> v;
      if (e == element) rhor[m] = v;
    }
    if (!in) return 3;
  }
  for (int i = 0; i < nel; ++i)
    for (int j = 0; j <= i; ++j)
      for (int m = 1; m <= nr; ++m) {
        float v;
        in >> v;
        if (i == element && j == element) z2r[m] = v;
      }
  if (!in) return 3;
  t.nrho = nrho;
  t.nr = nr;
  t.drho = drho;
  t.dr = dr;
  t.rhomax = (float)(nrho - 1) * drho;
  t.cut = cut;
  funcfl_interpolate(nrho, drho, frho, t.frho);
  funcfl_interpolate(nr, dr, rhor, t.rhor);
  funcfl_interpolate(nr, dr, z2r, t.z2r);
  return 0;
}

// funcfl unless the name ends in ".alloy" or ".setfl" (or format == "setfl")
inline int eam_load(const std::string& path, FuncflTables& t, const std::string& format = "") {
  auto ends = [&](const char* suf) {
    const std::string s(suf);
    return path.size() >= s.size() && path.compare(path.size() - s.size(), s.size(), s) == 0;
  };
  if (format == "setfl" || (format.empty() && (ends(".alloy") || ends(".setfl")))) return setfl_load(path, t);
  return funcfl_load(path, t);
}

}  // namespace rbmd
