// ocfd_sc.cpp -- host driver over the C ABI, in place of the reference's
// Fortran program (opencfd.f90:14-31 -> NS_solver, OCFD_NS_Solver.f90:5-88).
//
//   ocfd_sc [--deck opencfd2.in] [--device N] [--steps K]
//   ocfd_sc --io-selftest DIR        (file-format round trip, no GPU work)
//   ocfd_sc --print-params [--deck F] (deck + set_parameters, printed as JSON, no GPU work)
//
// Flow of the reference, one rank owning the whole grid:
//   read_parameter (OCFD_readpara.f90:3-200)   -> read_deck()
//   set_parameters (:261-341)                  -> ocfd_set_parameters()
//   init_mesh      (OCFD_mesh.f90:1-58)        -> OCFD-grid.dat reader + ocfd_gpu_init_mesh()
//   read_flow_data (OCFD_IO.f90:5-41)          -> opencfd.dat reader, else flowfield_init('TGV')
//   init3d + OCFD_bc                           -> ocfd_gpu_init3d()
//   time loop      (OCFD_NS_Solver.f90:21-78)  -> ocfd_gpu_step() in blocks of Istep_show,
//                                                 show_flow_msg, save_flow_data at Istep_Save
//   save_flow_data (OCFD_IO.f90:45-65)         -> OCFD%08d.dat writer
//   OCFD_analysis  (OCFD_ANA.f90:3-31)         -> run_analysis(): the ANA_Para schedule
//                                                 (codes 100-104) over the device analyses
// Files use the reference's Fortran unformatted sequential records (4-byte
// length markers): record 1 = (Istep:int32, tt:real64), then for each of
// d,u,v,w,T nz records of nx*ny real64 (OCFD_IO_mpi.f90:132-282).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "ocfd_gpu.h"

namespace {

// ------------------------------------------------------------------ Fortran records
bool write_record(std::ofstream& os, const void* data, uint32_t bytes) {
  os.write(reinterpret_cast<const char*>(&bytes), 4);
  os.write(reinterpret_cast<const char*>(data), bytes);
  os.write(reinterpret_cast<const char*>(&bytes), 4);
  return bool(os);
}
bool read_record(std::ifstream& is, void* data, uint32_t bytes) {
  uint32_t a = 0, b = 0;
  is.read(reinterpret_cast<char*>(&a), 4);
  if (!is || a != bytes) return false;
  is.read(reinterpret_cast<char*>(data), bytes);
  is.read(reinterpret_cast<char*>(&b), 4);
  return bool(is) && a == b;
}

// save_flow_data / read_flow_data layout for 5 interior fields
bool write_flow(const std::string& path, int istep, double tt, int nx, int ny, int nz,
                const std::vector<std::vector<double>>& q) {
  std::ofstream os(path, std::ios::binary);
  if (!os) return false;
  char rec1[12];
  std::memcpy(rec1, &istep, 4);
  std::memcpy(rec1 + 4, &tt, 8);
  if (!write_record(os, rec1, 12)) return false;
  const size_t plane = (size_t)nx * ny;
  for (int v = 0; v < 5; v++)
    for (int k = 0; k < nz; k++)
      if (!write_record(os, q[v].data() + plane * k, (uint32_t)(plane * 8))) return false;
  return true;
}
bool read_flow(const std::string& path, int& istep, double& tt, int nx, int ny, int nz,
               std::vector<std::vector<double>>& q) {
  std::ifstream is(path, std::ios::binary);
  if (!is) return false;
  char rec1[12];
  if (!read_record(is, rec1, 12)) return false;
  std::memcpy(&istep, rec1, 4);
  std::memcpy(&tt, rec1 + 4, 8);
  const size_t plane = (size_t)nx * ny;
  q.assign(5, std::vector<double>(plane * nz));
  for (int v = 0; v < 5; v++)
    for (int k = 0; k < nz; k++)
      if (!read_record(is, q[v].data() + plane * k, (uint32_t)(plane * 8))) return false;
  return true;
}

// OCFD-grid.dat: read_mesh1d / read_mesh2d_plane / read_mesh2d_AxialSymm /
// read_mesh3d (OCFD_mesh.f90:187-317).  Iflag_Gridtype 31 also reads the ten
// metric / Jacobian arrays into jac (Akx, Aky, Akz, Aix, Aiy, Aiz, Asx, Asy,
// Asz, Ajac).
bool read_grid(const std::string& path, int type, int nx, int ny, int nz, std::vector<double>& X,
               std::vector<double>& Y, std::vector<double>& Z, std::vector<std::vector<double>>& jac) {
  std::ifstream is(path, std::ios::binary);
  if (!is) return false;
  const size_t n = (size_t)nx * ny * nz, plane = (size_t)nx * ny;
  X.resize(n);
  Y.resize(n);
  Z.resize(n);
  if (type == OCFD_GRID1D) {
    std::vector<double> x(nx), y(ny), z(nz);
    if (!read_record(is, x.data(), nx * 8) || !read_record(is, y.data(), ny * 8) ||
        !read_record(is, z.data(), nz * 8))
      return false;
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          const size_t c = i + plane * k + (size_t)nx * j;
          X[c] = x[i];
          Y[c] = y[j];
          Z[c] = z[k];
        }
    return true;
  }
  if (type == OCFD_GRID2D_PLANE || type == OCFD_GRID2D_AXIAL_SYMM) {
    std::vector<double> x2(plane), y2(plane), z1(nz);
    if (!read_record(is, x2.data(), (uint32_t)(plane * 8)) || !read_record(is, y2.data(), (uint32_t)(plane * 8)) ||
        !read_record(is, z1.data(), nz * 8))
      return false;
    for (int k = 0; k < nz; k++)
      for (size_t c = 0; c < plane; c++) {
        X[c + plane * k] = x2[c];
        if (type == OCFD_GRID2D_PLANE) {
          Y[c + plane * k] = y2[c];
          Z[c + plane * k] = z1[k];
        } else {
          // read_mesh2d_AxialSymm (OCFD_mesh.f90:286-317): y2 is R, z1 the angle seta
          Y[c + plane * k] = y2[c] * std::cos(z1[k]);
          Z[c + plane * k] = y2[c] * std::sin(z1[k]);
        }
      }
    return true;
  }
  if (type == OCFD_GRID3D || type == OCFD_GRID_AND_JACOBIAN3D) {
    std::vector<double>* A[3] = {&X, &Y, &Z};
    for (int a = 0; a < 3; a++)
      for (int k = 0; k < nz; k++)
        if (!read_record(is, A[a]->data() + plane * k, (uint32_t)(plane * 8))) return false;
    if (type == OCFD_GRID_AND_JACOBIAN3D) {
      jac.assign(10, std::vector<double>(n));
      for (int a = 0; a < 10; a++)
        for (int k = 0; k < nz; k++)
          if (!read_record(is, jac[a].data() + plane * k, (uint32_t)(plane * 8))) return false;
    }
    return true;
  }
  return false;
}

// ------------------------------------------------------------------ namelist
std::string upper(std::string s) {
  for (auto& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}
std::vector<std::string> split_values(const std::string& s) {
  std::vector<std::string> out;
  std::string cur;
  bool q = false;
  for (char c : s) {
    if (c == '"' || c == '\'') {
      q = !q;
      continue;
    }
    if (!q && (c == ',' || std::isspace((unsigned char)c))) {
      if (!cur.empty()) out.push_back(cur);
      cur.clear();
    } else {
      cur += c;
    }
  }
  if (!cur.empty()) out.push_back(cur);
  return out;
}
double num(std::string s) {
  for (auto& c : s)
    if (c == 'd' || c == 'D') c = 'e';
  return std::strtod(s.c_str(), nullptr);
}

// read_parameter (OCFD_readpara.f90:3-200): namelist /control_opencfd/
// ANA_Number and ANA_Para(100, 10) of /control_opencfd/ (OCFD_readpara.f90:12,21,58-59),
// column-major like the Fortran array: entry m is para[100*m .. 100*m+99] =
// (code, step interval, data(1:50), ...).
struct AnaDeck {
  int number = 0;
  std::vector<double> para = std::vector<double>(1000, 0.0);
};

bool read_deck(const std::string& path, ocfd_params& p, std::string& err, AnaDeck* ana = nullptr) {
  std::ifstream is(path);
  if (!is) {
    err = "cannot open " + path;
    return false;
  }
  std::stringstream ss;
  std::string line;
  bool in = false;
  while (std::getline(is, line)) {
    const size_t bang = line.find('!');
    if (bang != std::string::npos) line = line.substr(0, bang);
    const std::string u = upper(line);
    if (!in) {
      if (u.find("CONTROL_OPENCFD") != std::string::npos) in = true;
      continue;
    }
    if (u.find("$END") != std::string::npos || u.find("&END") != std::string::npos ||
        (u.find('/') != std::string::npos && u.find('=') == std::string::npos))
      break;
    ss << line << "\n";
  }
  const std::string body = ss.str();
  // split "KEY = values" assignments
  std::vector<std::pair<std::string, std::string>> kv;
  size_t pos = 0;
  while (true) {
    size_t eq = body.find('=', pos);
    if (eq == std::string::npos) break;
    size_t ks = body.find_last_not_of(" \t\n", eq - 1);
    size_t kb = ks;
    while (kb > 0 && (std::isalnum((unsigned char)body[kb - 1]) || body[kb - 1] == '_' || body[kb - 1] == '(' ||
                      body[kb - 1] == ')' || body[kb - 1] == ':' || body[kb - 1] == ','))
      kb--;
    if (!kv.empty()) kv.back().second = body.substr(pos, kb - pos);
    kv.push_back({upper(body.substr(kb, ks - kb + 1)), ""});
    pos = eq + 1;
  }
  if (!kv.empty()) kv.back().second = body.substr(pos);
  std::map<std::string, int> schemes = {{"WENO5", 1}, {"WENO7", 2}, {"OMP6", 3}, {"UD7L", 4},
                                        {"CD6", 5},   {"CD8", 6},   {"HYBRID", 10}, {"SCHEME_USER", 99}};
  std::map<std::string, int> bcs = {{"BC_NONE", 0}, {"BC_BLUNT2D", 1}, {"BC_BOUNDARYLAYER", 2},
                                    {"BC_SWEPTCORNER", 3}, {"BC_USER_DEF", 99}};
  for (auto& [key0, val] : kv) {
    std::string key = key0;
    std::string sub;
    const size_t par = key.find('(');
    if (par != std::string::npos) {
      sub = key.substr(par + 1, key.find(')') - par - 1);
      key = key.substr(0, par);
    }
    auto v = split_values(val);
    if (v.empty()) continue;
    auto I = [&](int32_t& x) { x = (int32_t)num(v[0]); };
    auto D = [&](double& x) { x = num(v[0]); };
    if (key == "NX_GLOBAL") I(p.nx);
    else if (key == "NY_GLOBAL") I(p.ny);
    else if (key == "NZ_GLOBAL") I(p.nz);
    else if (key == "LAP") I(p.lap);
    else if (key == "MA") D(p.ma);
    else if (key == "RE") D(p.re);
    else if (key == "GAMMA") D(p.gamma);
    else if (key == "PR") D(p.pr);
    else if (key == "REF_AMU_T0") D(p.ref_amu_t0);
    else if (key == "DT") D(p.dt);
    else if (key == "END_TIME") D(p.end_time);
    else if (key == "AOA") p.aoa = num(v[0]) * 3.1415926535897932 / 180.0;
    else if (key == "IPERIODIC_X") I(p.iperiodic[0]);
    else if (key == "IPERIODIC_Y") I(p.iperiodic[1]);
    else if (key == "IPERIODIC_Z") I(p.iperiodic[2]);
    else if (key == "PERIODIC_ISPAN" || key == "PERIODIC_JSPAN" || key == "PERIODIC_KSPAN") {
      const int d = key[9] == 'I' ? 0 : (key[9] == 'J' ? 1 : 2);
      for (size_t c = 0; c < 3 && c < v.size(); c++) p.periodic_span[d][c] = num(v[c]);
    } else if (key == "SCHEME_INVIS" || key == "SCHEME_VIS") {
      auto it = schemes.find(upper(v[0]));
      if (it == schemes.end()) {
        err = "This Scheme  is not supported !! " + v[0];
        return false;
      }
      (key == "SCHEME_INVIS" ? p.scheme_invis : p.scheme_vis) = it->second;
    } else if (key == "BOUNDARYCONDITION") {
      auto it = bcs.find(upper(v[0]));
      if (it == bcs.end()) {
        err = "This Boundary Condition  is not supported !! " + v[0];
        return false;
      }
      p.ibc = it->second;
    } else if (key == "IF_SCHEME_CHARACTER") I(p.if_scheme_character);
    else if (key == "IF_VISCOUS") I(p.if_viscous);
    else if (key == "ISTEP_SHOW") I(p.istep_show);
    else if (key == "ISTEP_SAVE") I(p.istep_save);
    else if (key == "IFLAG_GRIDTYPE") I(p.iflag_gridtype);
    else if (key == "IF_MASS_FORCE") I(p.if_mass_force);
    else if (key == "NFILTERING") I(p.nfiltering);
    else if (key == "FLUX_SPLITTING") I(p.flux_splitting);
    else if (key == "UD7L_DISS") D(p.ud7l_diss);
    else if (key == "SCHEME_BOUNDARY" || key == "GHOST_CELL") {
      int32_t* a = key == "SCHEME_BOUNDARY" ? p.scheme_boundary : p.ghost_cell;
      int st = sub.empty() ? 0 : std::atoi(sub.c_str()) - 1;
      for (size_t c = 0; c < v.size() && st + (int)c < 6; c++) a[st + c] = (int32_t)num(v[c]);
    } else if (key == "MASS_FORCE" || key == "BC_PARA" || key == "HYBRID_PARA") {
      double* a = key == "MASS_FORCE" ? p.mass_force : (key == "BC_PARA" ? p.bc_para : p.hybrid_para);
      const int cap = key == "MASS_FORCE" ? 3 : 100;
      int st = sub.empty() ? 0 : std::atoi(sub.c_str()) - 1;
      for (size_t c = 0; c < v.size() && st + (int)c < cap; c++) a[st + c] = num(v[c]);
    } else if (key == "FILTER_PARA") {
      int col = 0;
      const size_t comma = sub.find(',');
      if (comma != std::string::npos) col = std::atoi(sub.substr(comma + 1).c_str()) - 1;
      for (size_t c = 0; c < v.size() && c < 100; c++) p.filter_para[col][c] = num(v[c]);
    }
    else if (key == "ANA_NUMBER" && ana) {
      ana->number = (int)num(v[0]);
    } else if (key == "ANA_PARA" && ana) {
      int r0 = 0, c0 = 0;
      if (!sub.empty()) {
        const size_t comma = sub.find(',');
        const std::string a = sub.substr(0, comma), b = comma == std::string::npos ? "" : sub.substr(comma + 1);
        if (!a.empty() && a != ":") r0 = std::atoi(a.c_str()) - 1;
        if (!b.empty() && b != ":") c0 = std::atoi(b.c_str()) - 1;
      }
      const int st = r0 + 100 * c0;
      for (size_t c = 0; c < v.size() && st + (int)c < 1000; c++) ana->para[st + c] = num(v[c]);
    }
    // npx0/npy0/npz0: one rank here
  }
  if (ana && ana->number > 10) {
    err = "ANA_Number and NFiltering should <=10";
    return false;
  }
  return true;
}

// Fortran Ew.dE2 edit descriptor: 0.ddd...E+xx, right-aligned in w columns.
std::string fortran_e(double x, int w = 20, int d = 13) {
  std::string body;
  if (x == 0.0) {
    body = "0." + std::string(d, '0') + "E+00";
  } else {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.*E", d - 1, std::fabs(x));
    std::string m(buf);
    const size_t e = m.find('E');
    std::string digits = m.substr(0, e);
    digits.erase(std::remove(digits.begin(), digits.end(), '.'), digits.end());
    const int ex = std::atoi(m.c_str() + e + 1) + 1;
    char eb[16];
    std::snprintf(eb, sizeof(eb), "E%c%02d", ex >= 0 ? '+' : '-', std::abs(ex));
    body = "0." + digits + eb;
    if (x < 0) body = "-" + body;
  }
  if ((int)body.size() < w) body = std::string(w - body.size(), ' ') + body;
  return body;
}

// OCFD_analysis after a step: every entry whose interval divides Istep, with
// the reference's files (OCFD_ANA.f90:3-31; codes OCFD_parameters.f90:36-37):
//   100 ana_time_average  means of d,u,v,w,T (restart from opencfd.dat.average);
//                         every data(1) steps OCFD%08d.dat.average
//   101 ana_getQ          Q-%07d.dat, nz records of nx*ny
//   102 ana_box           a row of statistics.dat, '(20(E20.13E2))'
//   103 ana_savedata      planes (1 YZ, 2 XZ, 3 XY), points (4), a block (5)
//   104 Ana_corner        WallUtp-log.dat: (Istep, tt), then u_t, T, p_w
struct Analysis {
  ocfd_handle* h;
  int nx, ny, nz;
  const AnaDeck& deck;
  bool avg_started = false;

  static void rec(std::ofstream& os, const void* p, size_t bytes) { write_record(os, p, (uint32_t)bytes); }
  static std::string head(int istep, double tt) {
    std::string b(12, '\0');
    std::memcpy(&b[0], &istep, 4);
    std::memcpy(&b[4], &tt, 8);
    return b;
  }
  bool block(int ib, int ie, int jb, int je, int kb, int ke, std::vector<std::vector<double>>& out) {
    const size_t m = (size_t)(ie - ib + 1) * (je - jb + 1) * (ke - kb + 1);
    out.assign(5, std::vector<double>(m));
    double* o[5] = {out[0].data(), out[1].data(), out[2].data(), out[3].data(), out[4].data()};
    return ocfd_gpu_download_block(h, ib, ie, jb, je, kb, ke, o) == OCFD_OK;
  }
  int run(int istep, double tt) {
    for (int e = 0; e < deck.number; e++) {
      const double* P = &deck.para[100 * e];
      const int code = (int)std::lround(P[0]), every = (int)std::lround(P[1]);
      const double* data = P + 2;
      if (every <= 0 || istep % every != 0) continue;
      if (code == 100) {
        if (!time_average(istep, tt, data)) return 1;
      } else if (code == 101) {
        std::vector<double> q((size_t)nx * ny * nz);
        if (ocfd_gpu_ana_q(h, q.data()) != OCFD_OK) return 1;
        char name[32];
        std::snprintf(name, sizeof(name), "Q-%07d.dat", istep);
        std::ofstream os(name, std::ios::binary);
        for (int k = 0; k < nz; k++) rec(os, q.data() + (size_t)k * nx * ny, (size_t)nx * ny * 8);
      } else if (code == 102) {
        double row[20];
        if (ocfd_gpu_ana_box(h, row) != OCFD_OK) return 1;
        std::ofstream os("statistics.dat", std::ios::app);
        for (int c = 0; c < 20; c++) os << fortran_e(row[c]);
        os << "\n";
      } else if (code == 103) {
        if (!savedata(istep, tt, data)) return 1;
      } else if (code == 104) {
        std::vector<double> out(3 * (size_t)nx);
        if (ocfd_gpu_ana_corner(h, out.data()) != OCFD_OK) return 1;
        std::ofstream os("WallUtp-log.dat", std::ios::binary | std::ios::app);
        const std::string hd = head(istep, tt);
        rec(os, hd.data(), 12);
        rec(os, out.data(), out.size() * 8);
      } else {
        std::fprintf(stderr, "analysis code %d is not supported\n", code);
        return 1;
      }
    }
    return 0;
  }
  bool time_average(int istep, double tt, const double* data) {
    const size_t plane = (size_t)nx * ny, n = plane * nz;
    if (!avg_started) {
      avg_started = true;
      std::ifstream is("opencfd.dat.average", std::ios::binary);
      if (is) {
        char r1[12];
        if (!read_record(is, r1, 12)) return false;
        int k_avg;
        double t_avg;
        std::memcpy(&k_avg, r1, 4);
        std::memcpy(&t_avg, r1 + 4, 8);
        std::vector<std::vector<double>> m(5, std::vector<double>(n));
        for (int v = 0; v < 5; v++)
          for (int k = 0; k < nz; k++)
            if (!read_record(is, m[v].data() + k * plane, (uint32_t)(plane * 8))) return false;
        const double* mp[5] = {m[0].data(), m[1].data(), m[2].data(), m[3].data(), m[4].data()};
        if (ocfd_gpu_upload_average(h, mp, k_avg, t_avg) != OCFD_OK) return false;
      }
    }
    if (ocfd_gpu_ana_time_average(h) != OCFD_OK) return false;
    const int every_save = (int)std::lround(data[0]);
    if (every_save > 0 && istep % every_save == 0) {
      std::vector<std::vector<double>> m(5, std::vector<double>(n));
      double* mp[5] = {m[0].data(), m[1].data(), m[2].data(), m[3].data(), m[4].data()};
      int k_avg = 0;
      double t_avg = 0;
      if (ocfd_gpu_download_average(h, mp, &k_avg, &t_avg) != OCFD_OK) return false;
      char name[40];
      std::snprintf(name, sizeof(name), "OCFD%08d.dat.average", istep);
      std::ofstream os(name, std::ios::binary);
      const std::string hd = head(k_avg, t_avg);
      rec(os, hd.data(), 12);
      for (int v = 0; v < 5; v++)
        for (int k = 0; k < nz; k++) rec(os, m[v].data() + k * plane, plane * 8);
    }
    (void)tt;
    return true;
  }
  // ana_savedata (OCFD_ANA_savedata.f90:3-196)
  bool savedata(int istep, double tt, const double* data) {
    const int kind = (int)std::lround(data[0]);
    const std::string hd = head(istep, tt);
    std::vector<std::vector<double>> b;
    if (kind >= 1 && kind <= 3) {
      const int points = (int)std::lround(data[1]), band = (int)std::lround(data[2]);
      const char* tag = kind == 1 ? "YZ" : (kind == 2 ? "XZ" : "XY");
      for (int ka = 1; ka <= points; ka++) {
        const int at = (int)std::lround(data[2 + ka]);
        char name[40];
        std::snprintf(name, sizeof(name), "savedata-%s%03d.dat", tag, ka);
        std::ofstream os(name, std::ios::binary | std::ios::app);
        rec(os, hd.data(), 12);
        for (int q = at; q < at + band; q++) {
          const bool ok = kind == 1 ? block(q, q, 1, ny, 1, nz, b)
                                    : (kind == 2 ? block(1, nx, q, q, 1, nz, b) : block(1, nx, 1, ny, q, q, b));
          if (!ok) return false;
          for (auto& v : b) rec(os, v.data(), v.size() * 8);
        }
      }
    } else if (kind == 4) {
      std::ifstream is("save_points_locations.dat");
      int m = 0;
      if (!(is >> m)) return false;
      std::string rest;
      std::getline(is, rest);
      std::vector<std::vector<double>> vals(5, std::vector<double>(m));
      for (int c = 0; c < m; c++) {
        std::string line;
        std::getline(is, line);
        std::istringstream ls(line);
        int i = 0, j = 0, k = 0;
        ls >> i >> j >> k;
        if (!block(i, i, j, j, k, k, b)) return false;
        for (int q = 0; q < 5; q++) vals[q][c] = b[q][0];
      }
      std::ofstream os("save_points.dat", std::ios::binary | std::ios::app);
      rec(os, &tt, 8);
      for (int q = 0; q < 5; q++) rec(os, vals[q].data(), (size_t)m * 8);
    } else if (kind == 5) {
      int r[7];
      for (int c = 0; c < 7; c++) r[c] = (int)std::lround(data[1 + c]);
      if (!block(r[0], r[1], r[2], r[3], r[4], r[5], b)) return false;
      char name[40];
      std::snprintf(name, sizeof(name), "savedata-block%03d.dat", r[6]);
      std::ofstream os(name, std::ios::binary | std::ios::app);
      rec(os, hd.data(), 12);
      for (auto& v : b) rec(os, v.data(), v.size() * 8);
    }
    return true;
  }
  // steps until the next step at which some entry runs
  int next_due(int istep) const {
    int best = 1 << 30;
    for (int e = 0; e < deck.number; e++) {
      const int every = (int)std::lround(deck.para[100 * e + 1]);
      if (every > 0) best = std::min(best, every - istep % every);
    }
    return best;
  }
};

int fail(const char* what, int rc, ocfd_handle* h = nullptr) {
  std::fprintf(stderr, "%s failed (%d)%s%s\n", what, rc, h ? ": " : "", h ? ocfd_gpu_last_error(h) : "");
  return 1;
}

int io_selftest(const std::string& dir) {
  const int nx = 5, ny = 4, nz = 3;
  std::vector<std::vector<double>> q(5, std::vector<double>(nx * ny * nz));
  for (int v = 0; v < 5; v++)
    for (size_t c = 0; c < q[v].size(); c++) q[v][c] = 0.25 * v + 1e-3 * (double)c;
  const std::string f = dir + "/OCFD00000007.dat";
  if (!write_flow(f, 7, 0.035, nx, ny, nz, q)) return 2;
  std::vector<std::vector<double>> r;
  int istep = 0;
  double tt = 0;
  if (!read_flow(f, istep, tt, nx, ny, nz, r)) return 3;
  if (istep != 7 || tt != 0.035 || r != q) return 4;
  std::printf("io selftest ok\n");
  return 0;
}

// Reads OCFD-grid.dat as init_mesh would and writes the expanded coordinates
// (and, for Iflag_Gridtype 31, the ten metric arrays) as raw float64 to out:
// a check of the readers that needs no GPU.
int grid_dump(int type, int nx, int ny, int nz, const std::string& in, const std::string& out) {
  std::vector<double> X, Y, Z;
  std::vector<std::vector<double>> jac;
  if (!read_grid(in, type, nx, ny, nz, X, Y, Z, jac)) return 2;
  std::ofstream os(out, std::ios::binary);
  for (const std::vector<double>* a : {&X, &Y, &Z}) os.write((const char*)a->data(), a->size() * 8);
  for (const auto& a : jac) os.write((const char*)a.data(), a.size() * 8);
  return os ? 0 : 3;
}

}  // namespace

int main(int argc, char** argv) {
  std::string deck = "opencfd2.in";
  int device = 0;
  long max_steps = -1;
  bool print_only = false;
  for (int a = 1; a < argc; a++) {
    std::string s = argv[a];
    if (s == "--io-selftest" && a + 1 < argc) return io_selftest(argv[++a]);
    if (s == "--grid-dump" && a + 6 < argc)
      return grid_dump(std::atoi(argv[a + 1]), std::atoi(argv[a + 2]), std::atoi(argv[a + 3]),
                       std::atoi(argv[a + 4]), argv[a + 5], argv[a + 6]);
    if (s == "--print-params") print_only = true;
    else if (s == "--deck" && a + 1 < argc) deck = argv[++a];
    else if (s == "--device" && a + 1 < argc) device = std::atoi(argv[++a]);
    else if (s == "--steps" && a + 1 < argc) max_steps = std::atol(argv[++a]);
  }
  ocfd_params p;
  ocfd_default_params(&p);
  std::string err;
  AnaDeck ana;
  if (!read_deck(deck, p, err, &ana)) {
    std::fprintf(stderr, "%s\n", err.c_str());
    return 1;
  }
  int rc = ocfd_set_parameters(&p);
  if (rc) return fail("set_parameters", rc);
  if (print_only) {
    std::printf("{\"nx\": %d, \"ny\": %d, \"nz\": %d, \"iperiodic\": [%d, %d, %d], \"iflag_gridtype\": %d, "
                "\"scheme_invis\": %d, \"scheme_vis\": %d, \"if_scheme_character\": %d, \"flux_splitting\": %d, "
                "\"ibc\": %d, \"if_viscous\": %d, \"nfiltering\": %d, \"istep_show\": %d, \"istep_save\": %d, "
                "\"ma\": %.17g, \"re\": %.17g, \"gamma\": %.17g, \"pr\": %.17g, \"dt\": %.17g, "
                "\"end_time\": %.17g, \"hx\": %.17g, \"cv\": %.17g, \"cp\": %.17g, "
                "\"scheme_boundary\": [%d, %d, %d, %d, %d, %d], \"ghost_cell\": [%d, %d, %d, %d, %d, %d], "
                "\"hybrid_para\": [%.17g, %.17g, %.17g], \"bc_para0\": %.17g}\n",
                p.nx, p.ny, p.nz, p.iperiodic[0], p.iperiodic[1], p.iperiodic[2], p.iflag_gridtype, p.scheme_invis,
                p.scheme_vis, p.if_scheme_character, p.flux_splitting, p.ibc, p.if_viscous, p.nfiltering,
                p.istep_show, p.istep_save, p.ma, p.re, p.gamma, p.pr, p.dt, p.end_time, p.hx, p.cv, p.cp,
                p.scheme_boundary[0], p.scheme_boundary[1], p.scheme_boundary[2], p.scheme_boundary[3],
                p.scheme_boundary[4], p.scheme_boundary[5], p.ghost_cell[0], p.ghost_cell[1], p.ghost_cell[2],
                p.ghost_cell[3], p.ghost_cell[4], p.ghost_cell[5], p.hybrid_para[0], p.hybrid_para[1],
                p.hybrid_para[2], p.bc_para[0]);
    return 0;
  }
  std::printf("Re= %g  Ma= %g  Scheme_Invis= %d  Scheme_Vis= %d  Flux_Splitting= %d  IF_Scheme_Character= %d\n",
              p.re, p.ma, p.scheme_invis, p.scheme_vis, p.flux_splitting, p.if_scheme_character);
  ocfd_handle* h = nullptr;
  rc = ocfd_gpu_create(&p, device, &h);
  if (rc) return fail("ocfd_gpu_create", rc);
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const size_t n = (size_t)nx * ny * nz;
  // ---- init_mesh
  if (p.iflag_gridtype == OCFD_GRIDGEN) {
    rc = ocfd_gpu_init_mesh(h, nullptr, nullptr, nullptr);
  } else {
    std::vector<double> X, Y, Z;
    std::vector<std::vector<double>> jac;
    if (!read_grid("OCFD-grid.dat", p.iflag_gridtype, nx, ny, nz, X, Y, Z, jac)) {
      std::fprintf(stderr, "cannot read OCFD-grid.dat for Iflag_Gridtype %d\n", p.iflag_gridtype);
      return 1;
    }
    if (jac.empty()) {
      rc = ocfd_gpu_init_mesh(h, X.data(), Y.data(), Z.data());
    } else {
      const double* J[10];
      for (int a = 0; a < 10; a++) J[a] = jac[a].data();
      rc = ocfd_gpu_init_mesh_jacobian(h, X.data(), Y.data(), Z.data(), J);
    }
  }
  if (rc) return fail("init_mesh", rc, h);
  // ---- read_flow_data, or flowfield_init('TGV') (OCFD_flowinit.f90:18-28)
  std::vector<std::vector<double>> q;
  int istep = 0;
  double tt = 0.0;
  if (!read_flow("opencfd.dat", istep, tt, nx, ny, nz, q)) {
    std::vector<double> Xh((size_t)(nx + 8) * (ny + 8) * (nz + 8));
    double* mets[OCFD_N_METRICS] = {};
    mets[OCFD_M_AXX] = Xh.data();
    std::vector<double> Yh(Xh.size()), Zh(Xh.size());
    mets[OCFD_M_AYY] = Yh.data();
    mets[OCFD_M_AZZ] = Zh.data();
    rc = ocfd_gpu_download_metrics(h, mets);
    if (rc) return fail("download_metrics", rc, h);
    q.assign(5, std::vector<double>(n));
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          const size_t c = i + (size_t)nx * (j + (size_t)ny * k);
          const size_t hc = (i + 4) + (size_t)(nx + 8) * ((j + 4) + (size_t)(ny + 8) * (k + 4));
          const double x = Xh[hc], y = Yh[hc], z = Zh[hc];
          q[0][c] = 1.0;
          q[1][c] = std::sin(x) * std::cos(y) * std::cos(z);
          q[2][c] = -std::cos(x) * std::sin(y) * std::cos(z);
          q[3][c] = 0.0;
          q[4][c] = 1.0;
        }
    istep = 0;
    tt = 0.0;
  }
  const double* pr[5] = {q[0].data(), q[1].data(), q[2].data(), q[3].data(), q[4].data()};
  rc = ocfd_gpu_init3d(h, pr, istep, tt);
  if (rc) return fail("init3d", rc, h);
  std::printf("init ok\n");
  // ---- time loop
  auto t0 = std::chrono::steady_clock::now();
  long done = 0;
  const int show = p.istep_show > 0 ? p.istep_show : 1;
  Analysis an{h, nx, ny, nz, ana};
  while (tt < p.end_time - p.dt * 1e-4 && (max_steps < 0 || done < max_steps)) {
    int k = std::min(show - (istep % show), an.next_due(istep));
    const long left_t = (long)std::ceil((p.end_time - p.dt * 1e-4 - tt) / p.dt);
    if (k > left_t) k = (int)left_t;
    if (max_steps >= 0 && k > max_steps - done) k = (int)(max_steps - done);
    if (k <= 0) break;
    rc = ocfd_gpu_step(h, k, 1);
    if (rc == OCFD_E_NEGT) {
      std::printf("Number of Negative Temperature Points >  Limit, STOP !\n");
      ocfd_gpu_destroy(h);
      return 2;
    }
    if (rc) return fail("step", rc, h);
    done += k;
    ocfd_gpu_get_time(h, &istep, &tt);
    if (an.run(istep, tt)) return fail("analysis", 1, h);
    if (istep % show == 0) {
      double E0[3];
      ocfd_gpu_show_flow_msg(h, E0);
      std::printf("Istep= %d tt= %.10g\n%25s%25s%25s\n%25.15E%25.15E%25.15E\n", istep, tt, "Averaged Total-energy E",
                  "Kinetic-energy K", "Entropy S", E0[0], E0[1], E0[2]);
    }
    if (p.istep_save > 0 && istep % p.istep_save == 0) {
      // save_flow_data: primitives d,u,v,w,T
      std::vector<std::vector<double>> hal(5, std::vector<double>((size_t)(nx + 8) * (ny + 8) * (nz + 8)));
      double* hp[5] = {hal[0].data(), hal[1].data(), hal[2].data(), hal[3].data(), hal[4].data()};
      ocfd_gpu_download_state(h, nullptr, hp);
      std::vector<std::vector<double>> out(5, std::vector<double>(n));
      for (int v = 0; v < 5; v++)
        for (int kk = 0; kk < nz; kk++)
          for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++)
              out[v][i + (size_t)nx * (j + (size_t)ny * kk)] =
                  hal[v][(i + 4) + (size_t)(nx + 8) * ((j + 4) + (size_t)(ny + 8) * (kk + 4))];
      char name[64];
      std::snprintf(name, sizeof(name), "OCFD%08d.dat", istep);
      if (!write_flow(name, istep, tt, nx, ny, nz, out)) std::fprintf(stderr, "cannot write %s\n", name);
    }
  }
  const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::printf("total wtime cost: %.6f  (%ld steps, %.4f GPts/s)\n", wall, done, (double)n * done / wall / 1e9);
  ocfd_gpu_destroy(h);
  std::printf("OK The END of opencfd\n");
  return 0;
}
