// data_io.cpp -- LAMMPS data files, the reference's model input (read_data), for a drop-in
// host driver: read atoms, velocities, per-type coefficients and bond/angle topology into host
// arrays (the caller copies them to the device and binds them), and write the same format back
// (checkpoints that double as inputs).
//
// Reader semantics follow ModelFileInitCondition (rbmd/framework/InitCondition/
// ModelFileInitCondition.cpp:120-605): header counts by keyword ("atoms", "bonds", "angles",
// "dihedrals", "atom types", "bond types", "angle types", "xlo xhi" .. "zlo zhi"), then the
// sections Masses, Pair Coeffs, Bond Coeffs, Angle Coeffs, Atoms (styles atomic: id type x y z;
// charge: id type q x y z; full: id mol type q x y z), Bonds, Angles, Dihedrals, Velocities, each
// reading its count of non-empty lines; ids, types and molecules become 0-based and atoms are
// stored by id; in LJ units every mass is 1 (:293-298).  Beyond the reference: the optional image
// flags after the coordinates are kept, ids outside [1, N] and short lines are errors.
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/rbmd_force.h"

namespace rbmd_internal {
extern char g_last_error[512];
}

struct rbmd_data {
  rbmd_data_info info{};
  std::string style;
  std::vector<double> pos, vel, charge, mass_type, eps, sig, bond_k, bond_r0, angle_k, angle_t0, dih_coeffs;
  std::vector<int32_t> type, mol, image, bonds, bond_type, angles, angle_type, dihedrals, dihedral_type;
};

namespace {

using rbmd_internal::g_last_error;

rbmd_status fail(const char* what, const std::string& detail) {
  std::snprintf(g_last_error, sizeof g_last_error, "data file: %s %s", what, detail.c_str());
  return RBMD_ERR_FILE;
}

bool blank(const std::string& s) {
  for (char c : s)
    if (!std::isspace((unsigned char)c)) return false;
  return true;
}

// next non-empty line of the section body
bool next_line(std::vector<std::string>& lines, size_t& i, std::string& out) {
  while (i < lines.size()) {
    const std::string& l = lines[i++];
    if (!blank(l)) {
      out = l;
      return true;
    }
  }
  return false;
}

}  // namespace

extern "C" {

RBMD_API rbmd_status rbmd_data_read(const char* path, const char* atom_style, const char* unit, rbmd_data** out,
                                    rbmd_data_info* info) {
  if (!path || !atom_style || !out) return RBMD_ERR_ARG;
  *out = nullptr;
  const std::string style = atom_style;
  if (style != "atomic" && style != "charge" && style != "full") return RBMD_ERR_ARG;
  std::ifstream in(path);
  if (!in) return fail("cannot open", path);
  std::vector<std::string> lines;
  for (std::string l; std::getline(in, l);) {
    if (!l.empty() && l.back() == '\r') l.pop_back();
    lines.push_back(l);
  }
  if (!lines.empty() && lines[0].size() >= 3 && (unsigned char)lines[0][0] == 0xEF) lines[0].erase(0, 3);
  auto d = new rbmd_data();
  d->style = style;
  rbmd_data_info& h = d->info;
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  size_t i = 1;   // the first line is the title
  int64_t n_dih = 0;
  for (; i < lines.size(); ++i) {
    const std::string& l = lines[i];
    if (blank(l)) continue;
    std::istringstream ss(l);
    if (l.find("xlo xhi") != std::string::npos) ss >> lo[0] >> hi[0];
    else if (l.find("ylo yhi") != std::string::npos) ss >> lo[1] >> hi[1];
    else if (l.find("zlo zhi") != std::string::npos) { ss >> lo[2] >> hi[2]; ++i; break; }
    else if (l.find("atom types") != std::string::npos) ss >> h.n_atom_types;
    else if (l.find("bond types") != std::string::npos) ss >> h.n_bond_types;
    else if (l.find("angle types") != std::string::npos) ss >> h.n_angle_types;
    else if (l.find("dihedral types") != std::string::npos) ss >> h.n_dihedral_types;
    else if (l.find("atoms") != std::string::npos) ss >> h.n_atoms;
    else if (l.find("bonds") != std::string::npos) ss >> h.n_bonds;
    else if (l.find("angles") != std::string::npos) ss >> h.n_angles;
    else if (l.find("dihedrals") != std::string::npos) ss >> n_dih;
  }
  for (int k = 0; k < 3; ++k) { h.box.lo[k] = lo[k]; h.box.hi[k] = hi[k]; }
  h.n_dihedrals = n_dih;
  if (h.n_atoms < 1 || h.n_atom_types < 1 || !(hi[0] > lo[0] && hi[1] > lo[1] && hi[2] > lo[2])) {
    delete d;
    return fail("bad header in", path);
  }
  const int64_t n = h.n_atoms;
  const int nt = h.n_atom_types;
  d->pos.assign(3 * n, 0.0);
  d->vel.assign(3 * n, 0.0);
  d->charge.assign(n, 0.0);
  d->type.assign(n, -1);
  d->mol.assign(n, 0);
  d->image.assign(3 * n, 0);
  d->mass_type.assign(nt, 1.0);
  std::string l;
  auto bad = [&](const char* what) {
    delete d;
    return fail(what, std::string("in ") + path);
  };
  for (; i < lines.size(); ++i) {
    const std::string& sec = lines[i];
    if (blank(sec)) continue;
    size_t j = i + 1;
    if (sec.find("Masses") != std::string::npos) {
      for (int k = 0; k < nt; ++k) {
        if (!next_line(lines, j, l)) return bad("short Masses");
        std::istringstream ss(l);
        int t; double m;
        if (!(ss >> t >> m) || t < 1 || t > nt) return bad("bad Masses line");
        d->mass_type[t - 1] = m;
      }
    } else if (sec.find("Pair Coeffs") != std::string::npos) {
      d->eps.assign(nt, 0.0);
      d->sig.assign(nt, 0.0);
      for (int k = 0; k < nt; ++k) {
        if (!next_line(lines, j, l)) return bad("short Pair Coeffs");
        std::istringstream ss(l);
        int t; double e, s;
        if (!(ss >> t >> e >> s) || t < 1 || t > nt) return bad("bad Pair Coeffs line");
        d->eps[t - 1] = e;
        d->sig[t - 1] = s;
      }
      h.has_pair_coeffs = 1;
    } else if (sec.find("Bond Coeffs") != std::string::npos) {
      d->bond_k.assign(h.n_bond_types, 0.0);
      d->bond_r0.assign(h.n_bond_types, 0.0);
      for (int k = 0; k < h.n_bond_types; ++k) {
        if (!next_line(lines, j, l)) return bad("short Bond Coeffs");
        std::istringstream ss(l);
        int t; double a, b;
        if (!(ss >> t >> a >> b) || t < 1 || t > h.n_bond_types) return bad("bad Bond Coeffs line");
        d->bond_k[t - 1] = a;
        d->bond_r0[t - 1] = b;
      }
    } else if (sec.find("Angle Coeffs") != std::string::npos) {
      d->angle_k.assign(h.n_angle_types, 0.0);
      d->angle_t0.assign(h.n_angle_types, 0.0);
      for (int k = 0; k < h.n_angle_types; ++k) {
        if (!next_line(lines, j, l)) return bad("short Angle Coeffs");
        std::istringstream ss(l);
        int t; double a, b;
        if (!(ss >> t >> a >> b) || t < 1 || t > h.n_angle_types) return bad("bad Angle Coeffs line");
        d->angle_k[t - 1] = a;
        d->angle_t0[t - 1] = b;
      }
    } else if (sec.find("Dihedral Coeffs") != std::string::npos) {
      // ModelFileInitCondition::DihedralsCoeffs (ModelFileInitCondition.cpp:359-380): type K d n
      d->dih_coeffs.assign(3 * (size_t)std::max(h.n_dihedral_types, 0), 0.0);
      for (int k = 0; k < h.n_dihedral_types; ++k) {
        if (!next_line(lines, j, l)) return bad("short Dihedral Coeffs");
        std::istringstream ss(l);
        int t, sg, m; double kk;
        if (!(ss >> t >> kk >> sg >> m) || t < 1 || t > h.n_dihedral_types) return bad("bad Dihedral Coeffs line");
        d->dih_coeffs[3 * (t - 1)] = kk;
        d->dih_coeffs[3 * (t - 1) + 1] = sg;
        d->dih_coeffs[3 * (t - 1) + 2] = m;
      }
    } else if (sec.find("group") != std::string::npos) {
      j = i + 1;   // not used by the force path: the body is skipped as unknown lines
      continue;
    } else if (sec.find("Atoms") != std::string::npos) {
      for (int64_t k = 0; k < n; ++k) {
        if (!next_line(lines, j, l)) return bad("short Atoms");
        std::istringstream ss(l);
        int64_t id; int t = 0, m = 0; double q = 0, x, y, z;
        bool ok;
        if (style == "atomic") ok = (bool)(ss >> id >> t >> x >> y >> z);
        else if (style == "charge") ok = (bool)(ss >> id >> t >> q >> x >> y >> z);
        else ok = (bool)(ss >> id >> m >> t >> q >> x >> y >> z);
        if (!ok || id < 1 || id > n || t < 1 || t > nt) return bad("bad Atoms line");
        const int64_t a = id - 1;
        d->pos[3 * a] = x; d->pos[3 * a + 1] = y; d->pos[3 * a + 2] = z;
        d->charge[a] = q;
        d->type[a] = t - 1;
        d->mol[a] = m - 1;
        int ix = 0, iy = 0, iz = 0;
        if (ss >> ix >> iy >> iz) { d->image[3 * a] = ix; d->image[3 * a + 1] = iy; d->image[3 * a + 2] = iz; }
      }
      for (int64_t a = 0; a < n; ++a)
        if (d->type[a] < 0) return bad("missing atom ids");
    } else if (sec.find("Velocities") != std::string::npos) {
      for (int64_t k = 0; k < n; ++k) {
        if (!next_line(lines, j, l)) return bad("short Velocities");
        std::istringstream ss(l);
        int64_t id; double vx, vy, vz;
        if (!(ss >> id >> vx >> vy >> vz) || id < 1 || id > n) return bad("bad Velocities line");
        d->vel[3 * (id - 1)] = vx; d->vel[3 * (id - 1) + 1] = vy; d->vel[3 * (id - 1) + 2] = vz;
      }
      h.has_velocities = 1;
    } else if (sec.find("Bonds") != std::string::npos) {
      d->bonds.assign(2 * h.n_bonds, 0);
      d->bond_type.assign(h.n_bonds, 0);
      for (int64_t k = 0; k < h.n_bonds; ++k) {
        if (!next_line(lines, j, l)) return bad("short Bonds");
        std::istringstream ss(l);
        int64_t id, a, b; int t;
        if (!(ss >> id >> t >> a >> b) || a < 1 || a > n || b < 1 || b > n) return bad("bad Bonds line");
        d->bond_type[k] = t - 1;
        d->bonds[2 * k] = (int32_t)(a - 1);
        d->bonds[2 * k + 1] = (int32_t)(b - 1);
      }
    } else if (sec.find("Angles") != std::string::npos) {
      d->angles.assign(3 * h.n_angles, 0);
      d->angle_type.assign(h.n_angles, 0);
      for (int64_t k = 0; k < h.n_angles; ++k) {
        if (!next_line(lines, j, l)) return bad("short Angles");
        std::istringstream ss(l);
        int64_t id, a, b, c; int t;
        if (!(ss >> id >> t >> a >> b >> c) || a < 1 || a > n || b < 1 || b > n || c < 1 || c > n)
          return bad("bad Angles line");
        d->angle_type[k] = t - 1;
        d->angles[3 * k] = (int32_t)(a - 1);
        d->angles[3 * k + 1] = (int32_t)(b - 1);
        d->angles[3 * k + 2] = (int32_t)(c - 1);
      }
    } else if (sec.find("Dihedrals") != std::string::npos) {
      // ModelFileInitCondition::Dihedrals (ModelFileInitCondition.cpp:551-585): id type i j k l
      d->dihedrals.assign(4 * n_dih, 0);
      d->dihedral_type.assign(n_dih, 0);
      for (int64_t k = 0; k < n_dih; ++k) {
        if (!next_line(lines, j, l)) return bad("short Dihedrals");
        std::istringstream ss(l);
        int64_t id, q[4]; int t;
        if (!(ss >> id >> t >> q[0] >> q[1] >> q[2] >> q[3]) || t < 1 || t > std::max(h.n_dihedral_types, 1))
          return bad("bad Dihedrals line");
        for (int c = 0; c < 4; ++c) {
          if (q[c] < 1 || q[c] > n) return bad("bad Dihedrals line");
          d->dihedrals[4 * k + c] = (int32_t)(q[c] - 1);
        }
        d->dihedral_type[k] = t - 1;
      }
    } else {
      continue;
    }
    i = j - 1;
  }
  if (unit && std::string(unit) == "LJ") d->mass_type.assign(nt, 1.0);
  h.has_masses = 1;
  *out = d;
  if (info) *info = h;
  return RBMD_OK;
}

RBMD_API rbmd_status rbmd_data_atoms(const rbmd_data* d, double* pos, double* vel, double* charge, int32_t* type,
                                     int32_t* molecule, double* mass, int32_t* image) {
  if (!d) return RBMD_ERR_ARG;
  const int64_t n = d->info.n_atoms;
  if (pos) std::memcpy(pos, d->pos.data(), sizeof(double) * 3 * n);
  if (vel) std::memcpy(vel, d->vel.data(), sizeof(double) * 3 * n);
  if (charge) std::memcpy(charge, d->charge.data(), sizeof(double) * n);
  if (type) std::memcpy(type, d->type.data(), sizeof(int32_t) * n);
  if (molecule) std::memcpy(molecule, d->mol.data(), sizeof(int32_t) * n);
  if (image) std::memcpy(image, d->image.data(), sizeof(int32_t) * 3 * n);
  if (mass)
    for (int64_t a = 0; a < n; ++a) mass[a] = d->mass_type[d->type[a]];
  return RBMD_OK;
}

RBMD_API rbmd_status rbmd_data_types(const rbmd_data* d, double* mass_by_type, double* epsilon, double* sigma) {
  if (!d) return RBMD_ERR_ARG;
  const int nt = d->info.n_atom_types;
  if (mass_by_type) std::memcpy(mass_by_type, d->mass_type.data(), sizeof(double) * nt);
  if ((epsilon || sigma) && !d->info.has_pair_coeffs) return RBMD_ERR_STATE;
  if (epsilon) std::memcpy(epsilon, d->eps.data(), sizeof(double) * nt);
  if (sigma) std::memcpy(sigma, d->sig.data(), sizeof(double) * nt);
  return RBMD_OK;
}

RBMD_API rbmd_status rbmd_data_topology(const rbmd_data* d, int32_t* bonds, int32_t* bond_type, int32_t* angles,
                                        int32_t* angle_type, double* bond_coeffs, double* angle_coeffs) {
  if (!d) return RBMD_ERR_ARG;
  const rbmd_data_info& h = d->info;
  if (bonds && !d->bonds.empty()) std::memcpy(bonds, d->bonds.data(), sizeof(int32_t) * 2 * h.n_bonds);
  if (bond_type && !d->bond_type.empty()) std::memcpy(bond_type, d->bond_type.data(), sizeof(int32_t) * h.n_bonds);
  if (angles && !d->angles.empty()) std::memcpy(angles, d->angles.data(), sizeof(int32_t) * 3 * h.n_angles);
  if (angle_type && !d->angle_type.empty())
    std::memcpy(angle_type, d->angle_type.data(), sizeof(int32_t) * h.n_angles);
  if (bond_coeffs)
    for (size_t t = 0; t < d->bond_k.size(); ++t) { bond_coeffs[2 * t] = d->bond_k[t]; bond_coeffs[2 * t + 1] = d->bond_r0[t]; }
  if (angle_coeffs)
    for (size_t t = 0; t < d->angle_k.size(); ++t) {
      angle_coeffs[2 * t] = d->angle_k[t];
      angle_coeffs[2 * t + 1] = d->angle_t0[t];
    }
  return RBMD_OK;
}

RBMD_API rbmd_status rbmd_data_dihedrals(const rbmd_data* d, int32_t* dihedrals, int32_t* dihedral_type,
                                         double* dihedral_coeffs) {
  if (!d) return RBMD_ERR_ARG;
  if (dihedrals && !d->dihedrals.empty())
    std::memcpy(dihedrals, d->dihedrals.data(), sizeof(int32_t) * d->dihedrals.size());
  if (dihedral_type && !d->dihedral_type.empty())
    std::memcpy(dihedral_type, d->dihedral_type.data(), sizeof(int32_t) * d->dihedral_type.size());
  if (dihedral_coeffs && !d->dih_coeffs.empty())
    std::memcpy(dihedral_coeffs, d->dih_coeffs.data(), sizeof(double) * d->dih_coeffs.size());
  return RBMD_OK;
}

RBMD_API void rbmd_data_free(rbmd_data* d) { delete d; }

RBMD_API rbmd_status rbmd_data_write_arrays(const char* path, const char* atom_style, const rbmd_data_info* h,
                                            const rbmd_data_arrays* a) {
  if (!path || !atom_style || !h || !a || !a->pos || !a->type || h->n_atoms < 1 || h->n_atom_types < 1)
    return RBMD_ERR_ARG;
  const std::string style = atom_style;
  if (style != "atomic" && style != "charge" && style != "full") return RBMD_ERR_ARG;
  if (style != "atomic" && !a->charge) return RBMD_ERR_ARG;
  FILE* fp = std::fopen(path, "w");
  if (!fp) return fail("cannot write", path);
  const int64_t n = h->n_atoms;
  const int nt = h->n_atom_types;
  const int64_t nb = a->bonds ? h->n_bonds : 0, na = a->angles ? h->n_angles : 0;
  const int64_t nd = a->dihedrals ? h->n_dihedrals : 0;
  const int nbt = h->n_bond_types > 0 ? h->n_bond_types : 1, nat = h->n_angle_types > 0 ? h->n_angle_types : 1;
  const int ndt = h->n_dihedral_types > 0 ? h->n_dihedral_types : 1;
  std::fprintf(fp, "LAMMPS data file written by the B200 force library\n\n");
  std::fprintf(fp, "%lld atoms\n%d atom types\n", (long long)n, nt);
  if (nb) std::fprintf(fp, "%lld bonds\n%d bond types\n", (long long)nb, nbt);
  if (na) std::fprintf(fp, "%lld angles\n%d angle types\n", (long long)na, nat);
  if (nd) std::fprintf(fp, "%lld dihedrals\n%d dihedral types\n", (long long)nd, ndt);
  const char* ax[3] = {"xlo xhi", "ylo yhi", "zlo zhi"};
  std::fprintf(fp, "\n");
  for (int k = 0; k < 3; ++k) std::fprintf(fp, "%.17g %.17g %s\n", h->box.lo[k], h->box.hi[k], ax[k]);
  if (a->mass_by_type) {
    std::fprintf(fp, "\nMasses\n\n");
    for (int t = 0; t < nt; ++t) std::fprintf(fp, "%d %.17g\n", t + 1, a->mass_by_type[t]);
  }
  if (a->epsilon && a->sigma) {
    std::fprintf(fp, "\nPair Coeffs\n\n");
    for (int t = 0; t < nt; ++t) std::fprintf(fp, "%d %.17g %.17g\n", t + 1, a->epsilon[t], a->sigma[t]);
  }
  if (nb && a->bond_coeffs) {
    std::fprintf(fp, "\nBond Coeffs # harmonic\n\n");
    for (int t = 0; t < nbt; ++t)
      std::fprintf(fp, "%d %.17g %.17g\n", t + 1, a->bond_coeffs[2 * t], a->bond_coeffs[2 * t + 1]);
  }
  if (na && a->angle_coeffs) {
    std::fprintf(fp, "\nAngle Coeffs # harmonic\n\n");
    for (int t = 0; t < nat; ++t)
      std::fprintf(fp, "%d %.17g %.17g\n", t + 1, a->angle_coeffs[2 * t], a->angle_coeffs[2 * t + 1]);
  }
  if (nd && a->dihedral_coeffs) {
    std::fprintf(fp, "\nDihedral Coeffs # harmonic\n\n");
    for (int t = 0; t < ndt; ++t)
      std::fprintf(fp, "%d %.17g %d %d\n", t + 1, a->dihedral_coeffs[3 * t], (int)a->dihedral_coeffs[3 * t + 1],
                   (int)a->dihedral_coeffs[3 * t + 2]);
  }
  std::fprintf(fp, "\nAtoms # %s\n\n", style.c_str());
  const double* pos = a->pos;
  for (int64_t i = 0; i < n; ++i) {
    const int32_t* im = a->image;
    const int ix = im ? im[3 * i] : 0, iy = im ? im[3 * i + 1] : 0, iz = im ? im[3 * i + 2] : 0;
    if (style == "atomic")
      std::fprintf(fp, "%lld %d %.17g %.17g %.17g %d %d %d\n", (long long)i + 1, a->type[i] + 1, pos[3 * i],
                   pos[3 * i + 1], pos[3 * i + 2], ix, iy, iz);
    else if (style == "charge")
      std::fprintf(fp, "%lld %d %.17g %.17g %.17g %.17g %d %d %d\n", (long long)i + 1, a->type[i] + 1,
                   a->charge[i], pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], ix, iy, iz);
    else
      std::fprintf(fp, "%lld %d %d %.17g %.17g %.17g %.17g %d %d %d\n", (long long)i + 1,
                   (a->molecule ? a->molecule[i] : (int32_t)i) + 1, a->type[i] + 1, a->charge[i], pos[3 * i],
                   pos[3 * i + 1], pos[3 * i + 2], ix, iy, iz);
  }
  if (a->vel) {
    std::fprintf(fp, "\nVelocities\n\n");
    for (int64_t i = 0; i < n; ++i)
      std::fprintf(fp, "%lld %.17g %.17g %.17g\n", (long long)i + 1, a->vel[3 * i], a->vel[3 * i + 1],
                   a->vel[3 * i + 2]);
  }
  if (nb) {
    std::fprintf(fp, "\nBonds\n\n");
    for (int64_t b = 0; b < nb; ++b)
      std::fprintf(fp, "%lld %d %d %d\n", (long long)b + 1, a->bond_type ? a->bond_type[b] + 1 : 1,
                   a->bonds[2 * b] + 1, a->bonds[2 * b + 1] + 1);
  }
  if (na) {
    std::fprintf(fp, "\nAngles\n\n");
    for (int64_t b = 0; b < na; ++b)
      std::fprintf(fp, "%lld %d %d %d %d\n", (long long)b + 1, a->angle_type ? a->angle_type[b] + 1 : 1,
                   a->angles[3 * b] + 1, a->angles[3 * b + 1] + 1, a->angles[3 * b + 2] + 1);
  }
  if (nd) {
    std::fprintf(fp, "\nDihedrals\n\n");
    for (int64_t b = 0; b < nd; ++b)
      std::fprintf(fp, "%lld %d %d %d %d %d\n", (long long)b + 1, a->dihedral_type ? a->dihedral_type[b] + 1 : 1,
                   a->dihedrals[4 * b] + 1, a->dihedrals[4 * b + 1] + 1, a->dihedrals[4 * b + 2] + 1,
                   a->dihedrals[4 * b + 3] + 1);
  }
  const bool ok = std::fclose(fp) == 0;
  return ok ? RBMD_OK : fail("error writing", path);
}

RBMD_API rbmd_status rbmd_data_write(const char* path, const char* atom_style, const rbmd_data_info* h,
                                     const double* pos, const double* vel, const double* charge,
                                     const int32_t* type, const int32_t* molecule, const int32_t* image,
                                     const double* mass_by_type, const double* epsilon, const double* sigma,
                                     const int32_t* bonds, const int32_t* angles) {
  rbmd_data_arrays a{};
  a.pos = pos; a.vel = vel; a.charge = charge; a.type = type; a.molecule = molecule; a.image = image;
  a.mass_by_type = mass_by_type; a.epsilon = epsilon; a.sigma = sigma; a.bonds = bonds; a.angles = angles;
  return rbmd_data_write_arrays(path, atom_style, h, &a);
}

}  // extern "C"
