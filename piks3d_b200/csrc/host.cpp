// Host-side set-up of libpiks3d_b200: para.in namelists, the discrete velocity set and the
// image preprocessing that turns a raw voxel image into the compact device geometry.
//
// The preprocessing must give voxel labels identical to PIKS3D's setupPhysicalGrid
// (physicalGrid.F90:217-1625): the drill / thin passes are in-place raster scans whose
// result depends on scan order, so they are run here in the same order. Everything after
// the labels (node compaction, wall programs, switch resolution, dependency levels) is
// this library's own layout for the device kernels.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <thread>

#include "piks_internal.h"

namespace piks {

namespace {
struct GHRow { int half, n; double xi[16]; double w[16]; };
const GHRow kGH[] = {
#include "gh_tables.inc"
};
const WProg kWall[] = {
#include "wall_table.inc"
};
struct SwitchRow { int o, axis, label, src; };
const SwitchRow kSwitch[] = {
#include "switch_table.inc"
};
const double kPi = std::atan(1.0) * 4.0;  // velocityGrid.F90:78
}  // namespace

const int kIncoming[6][4] = {{2, 3, 6, 7}, {1, 4, 5, 8}, {3, 4, 7, 8},
                             {1, 2, 5, 6}, {5, 6, 7, 8}, {1, 2, 3, 4}};

const WProg *wall_program(int label) {
  for (const WProg &p : kWall)
    if (p.label == label) return &p;
  return nullptr;
}

bool make_wall_plan(const WProg &p, WPlan &out) {
  out = WPlan{};
  out.nface = p.nface;
  out.nwr = p.nwr;
  if (p.nface < 1 || p.nface > 3 || p.nwr > 12) return false;
  for (int f = 0; f < p.nface; ++f) {
    out.dir[f] = p.face[f].dir;
    out.store[f] = p.face[f].store;
    out.keep[f] = p.face[f].store == ST_Z ? 0 : 0xf;
  }
  for (int k = 0; k < p.nwr; ++k) {
    const WWrite &w = p.wr[k];
    int src = -1;
    for (int f = 0; f < p.nface; ++f)
      for (int m = 0; m < 4; ++m)
        if (p.face[f].store == w.src_store && kIncoming[p.face[f].dir][m] == w.src_o) {
          if (src >= 0) return false;  // two faces produce the value
          src = f * 4 + m;
        }
    if (src < 0) return false;
    for (int j = 0; j < k; ++j)  // an earlier write replaced the source slot
      if (p.wr[j].dst_store == w.src_store && p.wr[j].dst_o == w.src_o) return false;
    for (int j = 0; j < k; ++j)
      if (p.wr[j].dst_store == w.dst_store && p.wr[j].dst_o == w.dst_o) return false;
    for (int f = 0; f < p.nface; ++f)
      for (int m = 0; m < 4; ++m)
        if (p.face[f].store == w.dst_store && kIncoming[p.face[f].dir][m] == w.dst_o) out.keep[f] &= ~(1 << m);
    out.dst_store[k] = w.dst_store;
    out.dst_o[k] = w.dst_o - 1;
    out.face[k] = w.face;
    out.src[k] = src;
  }
  return true;
}

uint8_t face_mask(int v) {
  // The wall label names the fluid sides: E (+x), W (-x), N (+y), S (-y), F (+z), B (-z).
  switch (v) {
    case L_E: return FACE_E; case L_W: return FACE_W; case L_N: return FACE_N;
    case L_S: return FACE_S; case L_F: return FACE_F; case L_B: return FACE_B;
    case L_EN: return FACE_E | FACE_N; case L_WN: return FACE_W | FACE_N;
    case L_ES: return FACE_E | FACE_S; case L_WS: return FACE_W | FACE_S;
    case L_NF: return FACE_N | FACE_F; case L_NB: return FACE_N | FACE_B;
    case L_SF: return FACE_S | FACE_F; case L_SB: return FACE_S | FACE_B;
    case L_EF: return FACE_E | FACE_F; case L_EB: return FACE_E | FACE_B;
    case L_WF: return FACE_W | FACE_F; case L_WB: return FACE_W | FACE_B;
    case L_ENF: return FACE_E | FACE_N | FACE_F; case L_WNF: return FACE_W | FACE_N | FACE_F;
    case L_WSF: return FACE_W | FACE_S | FACE_F; case L_ESF: return FACE_E | FACE_S | FACE_F;
    case L_ENB: return FACE_E | FACE_N | FACE_B; case L_WNB: return FACE_W | FACE_N | FACE_B;
    case L_WSB: return FACE_W | FACE_S | FACE_B; case L_ESB: return FACE_E | FACE_S | FACE_B;
    default: return 0;
  }
}
bool is_wall_label(int v) { return face_mask(v) != 0; }
bool is_corner3_label(int v) { return v >= 60 && v <= 73 && (v % 10) <= 3; }

// ---------------------------------------------------------------------------------------
// initParams adjustments (parameters.F90:120-134) and constants of setupPhysicalGrid/Flow.
piks_status make_setup(const piks_params &p, Setup &s, std::string &err) {
  if (p.Nx < 3 || p.Ny < 3 || p.Nz < 3) { err = "Nx, Ny, Nz must be >= 3"; return PIKS_ERR_ARG; }
  if (p.fluidlayer < 0 || p.block_repx < 1 || p.block_repy < 1 || p.block_repz < 1) {
    err = "fluidlayer must be >= 0 and block_rep* >= 1"; return PIKS_ERR_ARG;
  }
  if (!(p.Kn > 0) || p.chkConvergeStep < 1 || !(p.pressDrop != 0) || !(p.Ref_L > 0)) {
    err = "Kn > 0, pressDrop != 0, Ref_L > 0 and chkConvergeStep >= 1 are required"; return PIKS_ERR_ARG;
  }
  s.p = p;
  int Nx = p.Nx + 2 * p.fluidlayer;
  s.Nx_base = Nx; s.Ny_base = p.Ny; s.Nz_base = p.Nz;
  s.Nx = p.block_repx * Nx; s.Ny = p.block_repy * p.Ny; s.Nz = p.block_repz * p.Nz;
  s.ds = 1.0 / (s.Nx - 1 - 2 * p.fluidlayer);   // physicalGrid.F90:228
  s.mu = std::sqrt(kPi / 2.0) / p.Kn;          // flow.F90:90
  s.nranks = 1; s.rank = 0; s.xl = 1; s.xu = s.Nx;
  return PIKS_OK;
}

// mpiParams.F90:165-175: the xmax - xmin plane gaps are dealt out in equal parts, the first
// `partial` ranks one more, and the last rank also takes the plane xmax.
piks_status set_slab(Setup &s, int nranks, int rank, std::string &err) {
  if (nranks < 1 || rank < 0 || rank >= nranks) { err = "rank must be in [0, nranks)"; return PIKS_ERR_ARG; }
  const int xmin = 1, xmax = s.Nx;
  const int complete = (xmax - xmin) / nranks, partial = (xmax - xmin) - complete * nranks;
  auto bounds = [&](int c, int &xl, int &xu) {
    if (c + 1 <= partial) { xl = xmin + (complete + 1) * c; xu = xmin + (complete + 1) * (c + 1) - 1; }
    else { xl = xmin + complete * c + partial; xu = xmin + complete * (c + 1) + partial - 1; }
    if ((c + 1) % nranks == 0) xu = xu + 1;
  };
  for (int c = 0; c < nranks; ++c) {
    int l, u;
    bounds(c, l, u);
    if (u - l + 1 < 2) { err = "every rank needs at least two x planes (Nx too small for nranks)"; return PIKS_ERR_ARG; }
  }
  s.nranks = nranks;
  s.rank = rank;
  bounds(rank, s.xl, s.xu);
  return PIKS_OK;
}

// setupVelocityGrid (velocityGrid.F90:90-192)
piks_status make_velocity(const piks_params &p, Velocity &v, std::string &err) {
  const GHRow *row = nullptr;
  for (const GHRow &r : kGH)
    if (r.half == (p.halfRange ? 1 : 0) && r.n == p.Nc_fundamental) row = &r;
  if (!row) {
    err = "Nc_fundamental xi/wi for " + std::to_string(p.Nc_fundamental) + " has not been provided";
    return PIKS_ERR_NC;
  }
  const int n = p.Nc_fundamental;
  double xi[16], w1[16];
  for (int q = 0; q < n; ++q) { xi[q] = row->xi[q] * std::sqrt(2.0); w1[q] = row->w[q]; }
  v.Nc_fundamental = n;
  v.Nc = 8 * n * n * n;
  v.Nc8 = n * n * n;
  v.cx.resize(v.Nc8); v.cy.resize(v.Nc8); v.cz.resize(v.Nc8); v.w.resize(v.Nc8);
  for (int a = 0; a < n; ++a)          // z index (slowest)
    for (int b = 0; b < n; ++b)        // y index
      for (int c = 0; c < n; ++c) {    // x index (fastest)
        int k = c + b * n + a * n * n;
        v.cx[k] = xi[c]; v.cy[k] = xi[b]; v.cz[k] = xi[a];
        v.w[k] = w1[c] * w1[b] * w1[a];
      }
  double d = 0.0;
  for (int l = 0; l < v.Nc8; ++l) d = d + v.cz[l] * v.w[l];
  v.DiffFlux = d * 4;
  return PIKS_OK;
}

// ---------------------------------------------------------------------------------------
// Fortran ES15.6 (output.F90:156-158): one leading digit, 6 decimals, E+dd (no E when the
// exponent needs three digits), right-justified in 15 columns.
std::string fortran_es15_6(double val) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.6E", val);
  std::string s(buf);
  size_t e = s.find('E');
  if (e != std::string::npos) {
    int x = std::atoi(s.c_str() + e + 1);
    char eb[16];
    if (std::abs(x) >= 100) std::snprintf(eb, sizeof eb, "%+04d", x);
    else std::snprintf(eb, sizeof eb, "E%c%02d", x < 0 ? '-' : '+', std::abs(x));
    s = s.substr(0, e) + eb;
  }
  if (s.size() < 15) s.insert(0, 15 - s.size(), ' ');
  return s;
}

// ---------------------------------------------------------------------------------------
// Namelist reader for the five groups of parameters.F90:78-82.
namespace {
std::string lower(std::string s) { for (auto &c : s) c = (char)std::tolower((unsigned char)c); return s; }
bool parse_real(const std::string &t, double &out) {
  std::string u = t;
  for (auto &c : u) if (c == 'd' || c == 'D') c = 'e';
  char *end = nullptr;
  out = std::strtod(u.c_str(), &end);
  return end && *end == 0 && !u.empty();
}
bool parse_int(const std::string &t, int32_t &out) {
  char *end = nullptr;
  long v = std::strtol(t.c_str(), &end, 10);
  if (!end || *end != 0 || t.empty()) return false;
  out = (int32_t)v;
  return true;
}
bool parse_logical(const std::string &t, int32_t &out) {
  std::string u = lower(t);
  if (!u.empty() && u[0] == '.') u = u.substr(1);
  if (!u.empty() && (u[0] == 't')) { out = 1; return true; }
  if (!u.empty() && (u[0] == 'f')) { out = 0; return true; }
  return false;
}
}  // namespace

piks_status read_namelist(const char *path, piks_params &p, std::string &image_file, std::string &err) {
  std::ifstream in(path);
  if (!in) { err = std::string("ERROR: could not open namelist file ") + path; return PIKS_ERR_IO; }
  std::string text, line;
  while (std::getline(in, line)) {
    // strip '!' comments outside quotes
    bool q1 = false, q2 = false;
    for (size_t i = 0; i < line.size(); ++i) {
      char c = line[i];
      if (c == '\'' && !q2) q1 = !q1;
      else if (c == '"' && !q1) q2 = !q2;
      else if (c == '!' && !q1 && !q2) { line = line.substr(0, i); break; }
    }
    text += line + "\n";
  }
  std::map<std::string, std::map<std::string, std::string>> groups;
  size_t pos = 0;
  while ((pos = text.find('&', pos)) != std::string::npos) {
    size_t nend = pos + 1;
    while (nend < text.size() && (std::isalnum((unsigned char)text[nend]) || text[nend] == '_')) ++nend;
    std::string gname = lower(text.substr(pos + 1, nend - pos - 1));
    // body up to the terminating '/' outside quotes
    size_t i = nend;
    bool q1 = false, q2 = false;
    for (; i < text.size(); ++i) {
      char c = text[i];
      if (c == '\'' && !q2) q1 = !q1;
      else if (c == '"' && !q1) q2 = !q2;
      else if (c == '/' && !q1 && !q2) break;
    }
    if (i >= text.size()) { err = "ERROR: could not read example namelist"; return PIKS_ERR_IO; }
    std::string body = text.substr(nend, i - nend);
    // tokenize "name = value" items separated by commas / whitespace
    auto &kv = groups[gname];
    size_t k = 0;
    while (k < body.size()) {
      while (k < body.size() && (std::isspace((unsigned char)body[k]) || body[k] == ',')) ++k;
      if (k >= body.size()) break;
      size_t ks = k;
      while (k < body.size() && body[k] != '=' && !std::isspace((unsigned char)body[k])) ++k;
      std::string key = lower(body.substr(ks, k - ks));
      while (k < body.size() && std::isspace((unsigned char)body[k])) ++k;
      if (k >= body.size() || body[k] != '=') { err = "ERROR: could not read example namelist"; return PIKS_ERR_IO; }
      ++k;
      while (k < body.size() && std::isspace((unsigned char)body[k])) ++k;
      std::string val;
      if (k < body.size() && (body[k] == '\'' || body[k] == '"')) {
        char qc = body[k++];
        size_t vs = k;
        while (k < body.size() && body[k] != qc) ++k;
        val = body.substr(vs, k - vs);
        if (k < body.size()) ++k;
        kv[key] = "\x01" + val;  // mark as string
      } else {
        size_t vs = k;
        while (k < body.size() && body[k] != ',' && !std::isspace((unsigned char)body[k])) ++k;
        kv[key] = body.substr(vs, k - vs);
      }
    }
    pos = i + 1;
  }
  if (!groups.count("flownml")) { err = "ERROR: could not read example namelist"; return PIKS_ERR_IO; }
  piks_params_default(&p);
  auto geti = [&](const char *g, const char *k, int32_t &dst) -> bool {
    auto gi = groups.find(g);
    if (gi == groups.end()) return true;
    auto it = gi->second.find(k);
    if (it == gi->second.end()) return true;
    return parse_int(it->second, dst);
  };
  auto getr = [&](const char *g, const char *k, double &dst) -> bool {
    auto gi = groups.find(g);
    if (gi == groups.end()) return true;
    auto it = gi->second.find(k);
    if (it == gi->second.end()) return true;
    return parse_real(it->second, dst);
  };
  auto getl = [&](const char *g, const char *k, int32_t &dst) -> bool {
    auto gi = groups.find(g);
    if (gi == groups.end()) return true;
    auto it = gi->second.find(k);
    if (it == gi->second.end()) return true;
    return parse_logical(it->second, dst);
  };
  bool ok = true;
  ok &= geti("physicalnml", "nx", p.Nx); ok &= geti("physicalnml", "ny", p.Ny); ok &= geti("physicalnml", "nz", p.Nz);
  ok &= geti("physicalnml", "wallextorder", p.wallExtOrder); ok &= geti("physicalnml", "fluidlayer", p.fluidlayer);
  ok &= getr("physicalnml", "ref_l", p.Ref_L);
  ok &= geti("velocitynml", "nc_fundamental", p.Nc_fundamental); ok &= getl("velocitynml", "halfrange", p.halfRange);
  ok &= geti("mpinml", "mpi_xdim", p.mpi_xdim); ok &= geti("mpinml", "mpi_ydim", p.mpi_ydim); ok &= geti("mpinml", "mpi_zdim", p.mpi_zdim);
  ok &= geti("mpinml", "block_repx", p.block_repx); ok &= geti("mpinml", "block_repy", p.block_repy); ok &= geti("mpinml", "block_repz", p.block_repz);
  ok &= geti("solvernml", "maxstep", p.maxStep); ok &= geti("solvernml", "chkconvergestep", p.chkConvergeStep);
  ok &= geti("solvernml", "savestep", p.saveStep); ok &= getr("solvernml", "eps", p.eps);
  ok &= getl("solvernml", "savelast", p.saveLast); ok &= geti("solvernml", "saveformat", p.saveFormat);
  ok &= getr("flownml", "kn", p.Kn); ok &= getr("flownml", "pressdrop", p.pressDrop); ok &= getr("flownml", "accom", p.accom);
  if (!ok) { err = "ERROR: could not read example namelist"; return PIKS_ERR_IO; }
  image_file.clear();
  auto gi = groups.find("physicalnml");
  if (gi != groups.end()) {
    auto it = gi->second.find("imagefilename");
    if (it != gi->second.end()) image_file = it->second[0] == '\x01' ? it->second.substr(1) : it->second;
  }
  return PIKS_OK;
}

// ---------------------------------------------------------------------------------------
// Image preprocessing.
namespace {

// Working box with two ghost layers: b(i,j,k), i in [-1, N+2].
struct Box {
  int Nx, Ny, Nz, GX, GY;
  std::vector<uint8_t> v;
  Box(int nx, int ny, int nz) : Nx(nx), Ny(ny), Nz(nz), GX(nx + 4), GY(ny + 4), v((size_t)(nx + 4) * (ny + 4) * (nz + 4), L_FLUID) {}
  uint8_t &at(int i, int j, int k) { return v[(size_t)(i + 1) + (size_t)(j + 1) * GX + (size_t)(k + 1) * GX * GY]; }
  bool ghost(int i, int j, int k) const { return i < 1 || i > Nx || j < 1 || j > Ny || k < 1 || k > Nz; }
  void set_ghosts(uint8_t val) {
    for (int k = -1; k <= Nz + 2; ++k)
      for (int j = -1; j <= Ny + 2; ++j)
        for (int i = -1; i <= Nx + 2; ++i)
          if (ghost(i, j, k)) at(i, j, k) = val;
  }
};

// Opens 2x2x2 blocks around fluid voxels that are one voxel wide along some axis
// (physicalGrid.F90:352-377); in-place raster scan, x from 2 to Nx-1.
void drill_pass(Box &b) {
  for (int k = 1; k <= b.Nz; ++k)
    for (int j = 1; j <= b.Ny; ++j)
      for (int i = 2; i <= b.Nx - 1; ++i) {
        if (b.at(i, j, k) != L_FLUID) continue;
        bool narrow = (b.at(i + 1, j, k) != L_FLUID && b.at(i - 1, j, k) != L_FLUID) ||
                      (b.at(i, j + 1, k) != L_FLUID && b.at(i, j - 1, k) != L_FLUID) ||
                      (b.at(i, j, k + 1) != L_FLUID && b.at(i, j, k - 1) != L_FLUID);
        if (!narrow) continue;
        int j0 = (j == b.Ny) ? j - 1 : j;
        int k0 = (k == b.Nz) ? k - 1 : k;
        for (int kk = k0; kk <= k0 + 1; ++kk)
          for (int jj = j0; jj <= j0 + 1; ++jj)
            for (int ii = i; ii <= i + 1; ++ii) b.at(ii, jj, kk) = L_FLUID;
      }
}

// Turns solid voxels with fluid on both sides along some axis into fluid, ghosts counting
// as fluid (physicalGrid.F90:382-422); in-place raster scan.
void thin_pass(Box &b) {
  b.set_ghosts(L_FLUID);
  for (int k = 1; k <= b.Nz; ++k)
    for (int j = 1; j <= b.Ny; ++j)
      for (int i = 1; i <= b.Nx; ++i) {
        if (b.at(i, j, k) != L_SOLID) continue;
        if ((b.at(i + 1, j, k) == L_FLUID && b.at(i - 1, j, k) == L_FLUID) ||
            (b.at(i, j + 1, k) == L_FLUID && b.at(i, j - 1, k) == L_FLUID) ||
            (b.at(i, j, k + 1) == L_FLUID && b.at(i, j, k - 1) == L_FLUID))
          b.at(i, j, k) = L_FLUID;
      }
  b.set_ghosts(L_GHOST);
}

int label_from_sides(uint8_t sides) {
  // Solid voxel with fluid on `sides`; labels exist for at most one fluid side per axis
  // (physicalGrid.F90:562-667); any other combination stays plain solid.
  static const int table[64] = {
      L_SOLID, L_E, L_W, -1, L_N, L_EN, L_WN, -1, L_S, L_ES, L_WS, -1, -1, -1, -1, -1,
      L_F, L_EF, L_WF, -1, L_NF, L_ENF, L_WNF, -1, L_SF, L_ESF, L_WSF, -1, -1, -1, -1, -1,
      L_B, L_EB, L_WB, -1, L_NB, L_ENB, L_WNB, -1, L_SB, L_ESB, L_WSB, -1, -1, -1, -1, -1,
      -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
  int v = table[sides & 63];
  return v < 0 ? L_SOLID : v;
}

}  // namespace

piks_status preprocess_box(const Setup &s, const uint8_t *raw, int64_t nbytes, std::vector<uint8_t> &box,
                           std::string &err) {
  const int Nx = s.Nx, Ny = s.Ny, Nz = s.Nz, fl = s.p.fluidlayer;
  const int64_t need = (int64_t)s.Nz_base * s.Ny_base * (s.Nx_base - 2 * fl);
  if (!raw || nbytes < need) { err = "image stream shorter than Nx*Ny*Nz bytes"; return PIKS_ERR_IMAGE; }
  Box b(Nx, Ny, Nz);
  // stream read (physicalGrid.F90:257-280), fluid layers stay fluid
  int64_t pos = 0;
  for (int k = 1; k <= s.Nz_base; ++k)
    for (int j = 1; j <= s.Ny_base; ++j)
      for (int i = fl + 1; i <= s.Nx_base - fl; ++i) {
        uint8_t c = raw[pos++];
        if (c > 1) { err = "invalid image data file"; return PIKS_ERR_IMAGE; }
        b.at(i, j, k) = c ? L_SOLID : L_FLUID;
      }
  // block replication (physicalGrid.F90:285-298)
  for (int k = 0; k < s.p.block_repz; ++k)
    for (int j = 0; j < s.p.block_repy; ++j)
      for (int i = 0; i < s.p.block_repx; ++i)
        if (i || j || k)
          for (int kk = 1; kk <= s.Nz_base; ++kk)
            for (int jj = 1; jj <= s.Ny_base; ++jj)
              for (int ii = 1; ii <= s.Nx_base; ++ii)
                b.at(i * s.Nx_base + ii, j * s.Ny_base + jj, k * s.Nz_base + kk) = b.at(ii, jj, kk);
  b.set_ghosts(L_GHOST);
  for (int round = 0; round < 2; ++round) { drill_pass(b); thin_pass(b); }
  box.swap(b.v);
  return PIKS_OK;
}

void classify_host(const Setup &s, const std::vector<uint8_t> &box, Geometry &g) {
  const int Nx = s.Nx, Ny = s.Ny, Nz = s.Nz;
  const int BGX = Nx + 4, BGY = Ny + 4;
  auto B = [&](int i, int j, int k) -> uint8_t {
    return box[(size_t)(i + 1) + (size_t)(j + 1) * BGX + (size_t)(k + 1) * BGX * BGY];
  };
  g.Nx = Nx; g.Ny = Ny; g.Nz = Nz; g.GX = Nx + 4; g.GY = Ny + 4; g.GZ = Nz + 4;
  g.xl = s.xl; g.xu = s.xu; g.wglob = s.xl == 1; g.eglob = s.xu == Nx;
  const size_t NG = (size_t)g.GX * g.GY * g.GZ;
  g.label.assign(NG, L_GHOST);
  // labels (physicalGrid.F90:546-671); ghosts are not fluid here
  for (int k = 1; k <= Nz; ++k)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i) {
        uint8_t c = B(i, j, k);
        int lab = c;
        if (c == L_SOLID) {
          uint8_t sides = 0;
          if (B(i + 1, j, k) == L_FLUID) sides |= FACE_E;
          if (B(i - 1, j, k) == L_FLUID) sides |= FACE_W;
          if (B(i, j + 1, k) == L_FLUID) sides |= FACE_N;
          if (B(i, j - 1, k) == L_FLUID) sides |= FACE_S;
          if (B(i, j, k + 1) == L_FLUID) sides |= FACE_F;
          if (B(i, j, k - 1) == L_FLUID) sides |= FACE_B;
          lab = label_from_sides(sides);
        }
        g.label[g.ghost_index(i, j, k)] = (uint8_t)lab;
      }
  auto LAB = [&](int i, int j, int k) -> int { return g.label[g.ghost_index(i, j, k)]; };
  auto real = [&](int i, int j, int k) { return i >= 1 && i <= Nx && j >= 1 && j <= Ny && k >= 1 && k <= Nz; };

  // Nodes the solver reads: fluid voxels, and solid voxels within two cells of a fluid
  // voxel along an axis (upwind reads of the sweep, extrapolation reads of the walls).
  std::vector<uint8_t> keep(NG, 0);
  for (int k = 1; k <= Nz; ++k)
    for (int j = 1; j <= Ny; ++j)
      for (int i = 1; i <= Nx; ++i) {
        if (LAB(i, j, k) != L_FLUID) continue;
        for (int d = -2; d <= 2; ++d) {
          if (real(i + d, j, k)) keep[g.ghost_index(i + d, j, k)] = 1;
          if (real(i, j + d, k)) keep[g.ghost_index(i, j + d, k)] = 1;
          if (real(i, j, k + d)) keep[g.ghost_index(i, j, k + d)] = 1;
        }
      }
  // Nodes: the owned fluid voxels, then the other voxels of the slab's window that are read
  // (owned solids as above; on a side shared with a neighbour rank, the read voxels of its
  // two ghost planes, fluid or solid). For one rank the window is the box.
  g.nodemap.assign(NG, -2);
  g.node_g.clear();
  g.NF = 0;
  for (int pass = 0; pass < 2; ++pass) {
    for (int k = 1; k <= Nz; ++k)
      for (int j = 1; j <= Ny; ++j)
        for (int i = 1; i <= Nx; ++i) {
          int64_t gi = g.ghost_index(i, j, k);
          const bool fluid = LAB(i, j, k) == L_FLUID, own = i >= g.xl && i <= g.xu;
          if (pass == 0) {
            g.nodemap[gi] = -1;
            if (fluid && own) { g.nodemap[gi] = (int32_t)g.node_g.size(); g.node_g.push_back((int32_t)gi); }
          } else if (!(fluid && own) && g.in_window(i) && (fluid || keep[gi])) {
            g.nodemap[gi] = (int32_t)g.node_g.size();
            g.node_g.push_back((int32_t)gi);
          }
        }
    if (pass == 0) g.NF = (int32_t)g.node_g.size();
  }
  g.NB = (int32_t)g.node_g.size() - g.NF;

  // walls in raster (vecWall) order, 3-fold corners numbered in the same order
  g.wall_node.clear(); g.wall_label.clear(); g.wall_corner.clear(); g.wall_e.clear(); g.wall_nb.clear();
  g.bcorner.assign(g.NB, -1);
  g.nCorner = 0;
  for (int k = 1; k <= Nz; ++k)
    for (int j = 1; j <= Ny; ++j)
      for (int i = g.xl; i <= g.xu; ++i) {
        int lab = LAB(i, j, k);
        if (!is_wall_label(lab)) continue;
        int node = g.nodemap[g.ghost_index(i, j, k)];
        int corner = -1;
        if (is_corner3_label(lab)) corner = g.nCorner++;
        if (node >= g.NF) g.bcorner[node - g.NF] = corner;
        double e1, e2;
        wall_extrapolation(s, g, i, j, k, e1, e2);
        const WProg *P = wall_program(lab);
        int32_t nb[6];
        wall_neighbours(g, P, i, j, k, nb);
        g.wall_node.push_back(node);
        g.wall_label.push_back(lab);
        g.wall_corner.push_back(corner);
        g.wall_e.push_back(e1); g.wall_e.push_back(e2);
        for (int t = 0; t < 6; ++t) g.wall_nb.push_back(nb[t]);
      }
  g.nWall = (int32_t)g.wall_node.size();
}

// wallExtOrder's extrapolation coefficients of the wall at (i, j, k) (physicalGrid.F90:889-936).
void wall_extrapolation(const Setup &s, const Geometry &g, int i, int j, int k, double &e1, double &e2) {
  const int Nx = s.Nx, Ny = s.Ny, Nz = s.Nz;
  auto LAB = [&](int ii, int jj, int kk) -> int { return g.label[g.ghost_index(ii, jj, kk)]; };
  // reference local id (1-based) and its decode, used by wallExtOrder == 3 (physicalGrid.F90:895-936)
  const int64_t NXT = Nx + 4, NXYT = (int64_t)(Nx + 4) * (Ny + 4);
  e1 = 2.0; e2 = -1.0;
  if (s.p.wallExtOrder == 1) { e1 = 1.0; e2 = 0.0; }
  else if (s.p.wallExtOrder != 2) {
    int64_t localid = (int64_t)(i + 2) + (int64_t)(j + 1) * NXT + (int64_t)(k + 1) * NXYT;
    int kd = -1 + (int)(localid / NXYT);
    int jd = -1 + (int)((localid - (int64_t)(kd + 1) * NXYT) / NXT);
    int id = -1 + (int)(localid - (int64_t)(kd + 1) * NXYT - (int64_t)(jd + 1) * NXT);
    int v = LAB(id, jd, kd);
    uint8_t fm = face_mask(v);
    bool first = false;
    // the rank's own first / last plane (physicalGrid.F90:903-906 use xl, xu)
    if ((fm & FACE_W) && id == g.xl + 1 && LAB(g.xl, jd, kd) == L_FLUID) first = true;
    if ((fm & FACE_E) && id == g.xu - 1 && LAB(g.xu, jd, kd) == L_FLUID) first = true;
    if ((fm & FACE_S) && jd == 2 && LAB(id, 1, kd) == L_FLUID) first = true;
    if ((fm & FACE_N) && jd == Ny - 1 && LAB(id, Ny, kd) == L_FLUID) first = true;
    if ((fm & FACE_B) && kd == 2 && LAB(id, jd, 1) == L_FLUID) first = true;
    if ((fm & FACE_F) && kd == Nz - 1 && LAB(id, jd, Nz) == L_FLUID) first = true;
    if (first) { e1 = 1.0; e2 = 0.0; }
  }
}

// Node at +d and code at +2d along each face direction of wall program P at (i, j, k)
// (see Geometry::wall_nb).
void wall_neighbours(const Geometry &g, const WProg *P, int i, int j, int k, int32_t *nb) {
  const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
  auto real = [&](int ii, int jj, int kk) { return g.in_window(ii) && jj >= 1 && jj <= Ny && kk >= 1 && kk <= Nz; };
  for (int t = 0; t < 6; ++t) nb[t] = -1;
  for (int fi = 0; fi < P->nface; ++fi) {
    int dir = P->face[fi].dir;
    int dx = dir == DIR_PX ? 1 : dir == DIR_MX ? -1 : 0;
    int dy = dir == DIR_PY ? 1 : dir == DIR_MY ? -1 : 0;
    int dz = dir == DIR_PZ ? 1 : dir == DIR_MZ ? -1 : 0;
    nb[2 * fi] = g.nodemap[g.ghost_index(i + dx, j + dy, k + dz)];
    int i2 = i + 2 * dx, j2 = j + 2 * dy, k2 = k + 2 * dz;
    int32_t code;
    if (real(i2, j2, k2)) code = g.nodemap[g.ghost_index(i2, j2, k2)];  // node, or -1
    else if (i2 == 0 && j2 >= 1 && j2 <= Ny && k2 >= 1 && k2 <= Nz) code = -(2 + 2 * ((k2 - 1) * Ny + (j2 - 1)));
    else if (i2 == Nx + 1 && j2 >= 1 && j2 <= Ny && k2 >= 1 && k2 <= Nz) code = -(3 + 2 * ((k2 - 1) * Ny + (j2 - 1)));
    else code = -1;  // y/z ghost layers hold zeros on one rank
    nb[2 * fi + 1] = code;
  }
}

piks_status finish_geometry(const Setup &s, Geometry &g, std::string &err) {
  const int Nx = s.Nx, Ny = s.Ny, Nz = s.Nz;
  // node*8 + slot codes of the sweep must stay below 2^30
  if ((int64_t)g.node_g.size() * 8 >= (int64_t)1 << 30) { err = "image too large (more than 2^27 nodes read by the solver)"; return PIKS_ERR_ARG; }
  auto LAB = [&](int i, int j, int k) -> int { return g.label[g.ghost_index(i, j, k)]; };
  // voxels of the slab's window (the box for one rank) and the rank's own voxels
  auto real = [&](int i, int j, int k) { return g.in_window(i) && j >= 1 && j <= Ny && k >= 1 && k <= Nz; };
  auto owned = [&](int i, int j, int k) { return i >= g.xl && i <= g.xu && j >= 1 && j <= Ny && k >= 1 && k <= Nz; };
  // first / last swept x plane of an octant: the box's inflow plane is not swept
  // (physicalGrid.F90:976-985); a plane next to a neighbour rank's ghost planes is
  const int xs_lo = g.wglob ? 2 : g.xl, xs_hi = g.eglob ? Nx - 1 : g.xu;
  const int GX = g.GX, GXY = g.GX * g.GY;

  // Dependency levels: a wall whose extrapolation reads another wall's slots must see
  // that wall's new values if it comes earlier in vecWall order and its old values if it
  // comes later (the serial order of solver.F90:762). Longest-path levels over edges
  // earlier -> later give that order with all walls of one level independent.
  {
    std::vector<int32_t> widx_of_node(g.node_g.size(), -1);
    for (int q = 0; q < g.nWall; ++q) widx_of_node[g.wall_node[q]] = q;
    std::vector<std::vector<int32_t>> adj(g.nWall);
    for (int q = 0; q < g.nWall; ++q)
      for (int fi = 0; fi < 3; ++fi) {
        int32_t code = g.wall_nb[6 * q + 2 * fi + 1];
        if (g.wall_nb[6 * q + 2 * fi] < 0 && fi > 0) continue;
        if (code >= 0 && widx_of_node[code] >= 0) {
          int r = widx_of_node[code];
          adj[std::min(q, r)].push_back(std::max(q, r));
        }
      }
    std::vector<int32_t> level(g.nWall, 0);
    int maxl = 0;
    for (int q = 0; q < g.nWall; ++q)
      for (int r : adj[q]) { level[r] = std::max(level[r], level[q] + 1); maxl = std::max(maxl, level[r]); }
    g.level_start.assign(maxl + 2, 0);
    for (int q = 0; q < g.nWall; ++q) g.level_start[level[q] + 1]++;
    for (int L = 0; L <= maxl; ++L) g.level_start[L + 1] += g.level_start[L];
    g.wall_order.assign(g.nWall, 0);
    std::vector<int32_t> fill(g.level_start.begin(), g.level_start.end() - 1);
    for (int q = 0; q < g.nWall; ++q) g.wall_order[fill[level[q]]++] = q;
  }

  // Static resolution of the in-sweep switch: which slot a reader sees, by its position.
  {
    int8_t yrule[8][128], zrule[8][128];
    std::memset(yrule, -1, sizeof yrule);
    std::memset(zrule, -1, sizeof zrule);
    for (const SwitchRow &r : kSwitch) (r.axis == 0 ? yrule : zrule)[r.o][r.label] = (int8_t)r.src;
    auto swept = [&](int i, int j, int k, int o) {
      if (!owned(i, j, k) || LAB(i, j, k) != L_FLUID) return false;
      int sx = oct_sx(o), sy = oct_sy(o), sz = oct_sz(o);
      bool ix = sx > 0 ? (i >= xs_lo) : (i <= xs_hi);
      bool iy = sy > 0 ? (j >= 2) : (j <= Ny - 1);
      bool iz = sz > 0 ? (k >= 2) : (k <= Nz - 1);
      return ix && iy && iz;
    };
    g.roles.assign((size_t)g.NB * 8, 0);
    g.commit.clear();
    for (int32_t n = g.NF; n < (int32_t)g.node_g.size(); ++n) {
      int64_t gi = g.node_g[n];
      int i = (int)(gi % GX) - 1, j = (int)((gi / GX) % g.GY) - 1, k = (int)(gi / GXY) - 1;
      int lab = LAB(i, j, k);
      for (int o = 0; o < 8; ++o) {
        int sy = oct_sy(o), sz = oct_sz(o);
        int ys = yrule[o][lab], zs = zrule[o][lab];
        bool yswitched = ys >= 0 && swept(i, j + sy, k, o);
        bool zswitched = zs >= 0 && swept(i, j, k + sz, o);
        int after_y = yswitched ? ys : o;
        int r_y1 = ys >= 0 ? ys : o;
        int r_y2 = after_y;
        int r_z1 = zs >= 0 ? zs : after_y;
        int r_z2 = zswitched ? zs : after_y;
        int post = zswitched ? zs : after_y;
        g.roles[(size_t)(n - g.NF) * 8 + o] = (uint16_t)(r_y1 | (r_y2 << 4) | (r_z1 << 8) | (r_z2 << 12));
        if (post != o) { g.commit.push_back(n); g.commit.push_back(o); g.commit.push_back(post); }
      }
    }
  }

  // Sweep tasks ordered by hyperplane (see Geometry::tasks).
  {
    // u counts x planes from the plane before the first swept one (v, w likewise in y, z)
    const int ux_pos = g.wglob ? 1 : g.xl - 1, ux_neg = g.eglob ? Nx : g.xu + 1;
    const int umax = std::max(g.xu - ux_pos, ux_neg - g.xl);
    const int nhyper = umax + (Ny - 1) + (Nz - 1) - 2;  // u+v+w from 3 to umax+Ny+Nz-3
    std::vector<int64_t> count(nhyper + 1, 0);
    auto local = [&](int i, int n, int sgn) { return sgn > 0 ? i - 1 : n - i; };
    auto local_x = [&](int i, int sgn) { return sgn > 0 ? i - ux_pos : ux_neg - i; };
    auto upwind_code = [&](int i, int j, int k, int o, int role, bool first_order_zero) -> int32_t {
      // role: 0/1 x1/x2 (slot o as is), 2..5 y1, y2, z1, z2 (resolved switch roles)
      if (first_order_zero) return -2;
      if (!real(i, j, k)) return -2;
      const int32_t n = g.nodemap[g.ghost_index(i, j, k)];
      if (n < 0) return -2;  // never read with a non-zero coefficient
      if (n < g.NF) return n * 8 + o;
      if (role < 2) return n * 8 + o;
      const int src = (g.roles[(size_t)(n - g.NF) * 8 + o] >> (4 * (role - 2))) & 15;
      if (src < 8) return n * 8 + src;
      return (int32_t)(1 << 30) | (g.bcorner[n - g.NF] * 8 + o);
    };
    // one thread per octant: per-octant counts per hyperplane give every octant its own
    // positions (within a hyperplane, octant by octant, voxels in raster order)
    std::vector<std::vector<int64_t>> ocount(8, std::vector<int64_t>((size_t)nhyper, 0));
    auto sweep_octant = [&](int o, int pass, std::vector<int64_t> *fillpos) {
      const int sx = oct_sx(o), sy = oct_sy(o), sz = oct_sz(o);
      for (int k = 1; k <= Nz; ++k)
        for (int j = 1; j <= Ny; ++j)
          for (int i = g.xl; i <= g.xu; ++i) {
            if (LAB(i, j, k) != L_FLUID) continue;
            const int u = local_x(i, sx), v = local(j, Ny, sy), w = local(k, Nz, sz);
            if (u < 1 || v < 1 || w < 1) continue;  // inflow planes are not swept
            const int h = u + v + w - 3;
            if (pass == 0) { ocount[(size_t)o][(size_t)h]++; continue; }
            // first-order flags (physicalGrid.F90:1269-1298 and the seven sibling blocks)
            // the x rule in its label form: a ghost two planes upwind (the box's edge), not
            // the first swept plane of the slab, which reads its neighbour's planes
            const bool fx = LAB(i - 2 * sx, j, k) == L_GHOST || (face_mask(LAB(i - sx, j, k)) & (sx > 0 ? FACE_E : FACE_W));
            const bool fy = (v == 1) || (face_mask(LAB(i, j - sy, k)) & (sy > 0 ? FACE_N : FACE_S));
            const bool fz = (w == 1) || (face_mask(LAB(i, j, k - sz)) & (sz > 0 ? FACE_F : FACE_B));
            int32_t *t = &g.tasks[(size_t)(*fillpos)[(size_t)h]++ * 8];
            t[0] = g.nodemap[g.ghost_index(i, j, k)];
            t[1] = o | (fx ? 8 : 0) | (fy ? 16 : 0) | (fz ? 32 : 0);
            t[2] = upwind_code(i - sx, j, k, o, 0, false);
            t[3] = upwind_code(i - 2 * sx, j, k, o, 1, fx);
            t[4] = upwind_code(i, j - sy, k, o, 2, false);
            t[5] = upwind_code(i, j - 2 * sy, k, o, 3, fy);
            t[6] = upwind_code(i, j, k - sz, o, 4, false);
            t[7] = upwind_code(i, j, k - 2 * sz, o, 5, fz);
          }
    };
    std::vector<std::vector<int64_t>> fill(8);
    for (int pass = 0; pass < 2; ++pass) {
      if (pass == 1) {
        g.hyper_start.assign(nhyper + 1, 0);
        for (int h = 0; h < nhyper; ++h) {
          count[h] = 0;
          for (int o = 0; o < 8; ++o) count[h] += ocount[(size_t)o][(size_t)h];
          g.hyper_start[h + 1] = g.hyper_start[h] + count[h];
        }
        g.tasks.clear();
        g.tasks.resize((size_t)g.hyper_start[nhyper] * 8);  // every entry is written below
        for (int o = 0; o < 8; ++o) {
          fill[(size_t)o].resize((size_t)nhyper);
          for (int h = 0; h < nhyper; ++h) {
            int64_t before = 0;
            for (int o2 = 0; o2 < o; ++o2) before += ocount[(size_t)o2][(size_t)h];
            fill[(size_t)o][(size_t)h] = g.hyper_start[h] + before;
          }
        }
      }
      std::vector<std::thread> th;
      for (int o = 0; o < 8; ++o) th.emplace_back(sweep_octant, o, pass, &fill[(size_t)o]);
      for (auto &t : th) t.join();
    }
  }

  // x = 1 / x = Nx planes (inlet/outlet targets and halo sources), symmetry planes
  // (only the slabs at the box's sides hold them)
  g.plane_x1.assign((size_t)Ny * Nz, -1);
  g.plane_xN.assign((size_t)Ny * Nz, -1);
  for (int k = 1; k <= Nz; ++k)
    for (int j = 1; j <= Ny; ++j) {
      if (g.wglob) g.plane_x1[(size_t)(k - 1) * Ny + (j - 1)] = std::max(-1, g.nodemap[g.ghost_index(1, j, k)]);
      if (g.eglob) g.plane_xN[(size_t)(k - 1) * Ny + (j - 1)] = std::max(-1, g.nodemap[g.ghost_index(Nx, j, k)]);
    }
  g.sym_node.clear(); g.sym_flag.clear();
  for (int32_t n = 0; n < (int32_t)g.node_g.size(); ++n) {
    int64_t gi = g.node_g[n];
    int i = (int)(gi % GX) - 1, j = (int)((gi / GX) % g.GY) - 1, k = (int)(gi / GXY) - 1;
    if (i < g.xl || i > g.xu) continue;  // solver.F90:1870-1917 run over the rank's own planes
    uint8_t fl8 = (j == 1 ? 1 : 0) | (j == Ny ? 2 : 0) | (k == 1 ? 4 : 0) | (k == Nz ? 8 : 0);
    if (fl8) { g.sym_node.push_back(n); g.sym_flag.push_back(fl8); }
  }
  // x halos of a slab (solver.F90:535-560 move the two planes at each side)
  for (int side = 0; side < 2; ++side) {
    g.halo_send[side].clear();
    g.halo_recv[side].clear();
    if (side == 0 ? g.wglob : g.eglob) continue;
    const int s0 = side == 0 ? g.xl : g.xu - 1, r0 = side == 0 ? g.xl - 2 : g.xu + 1;
    for (int k = 1; k <= Nz; ++k)
      for (int j = 1; j <= Ny; ++j)
        for (int q = 0; q < 2; ++q) {
          const int32_t ns = g.nodemap[g.ghost_index(s0 + q, j, k)], nr = g.nodemap[g.ghost_index(r0 + q, j, k)];
          if (ns >= 0) g.halo_send[side].push_back(ns);
          if (nr >= 0) g.halo_recv[side].push_back(nr);
        }
  }
  // chkConverge's plane x = 2 in its summation order (output.F90:90-136); only the west-most
  // slab holds it (output.F90:89)
  g.flux_list.clear();
  for (int q = 0; q < 10; ++q) g.flux_groups[q] = 0;
  if (!g.wglob) return PIKS_OK;
  auto fnode = [&](int j, int k) -> int32_t {
    int32_t n = g.nodemap[g.ghost_index(2, j, k)];
    return (n >= 0 && n < g.NF) ? n : -1;
  };
  int gi = 0;
  g.flux_groups[gi++] = 0;
  for (int k = 2; k <= Nz - 1; ++k) for (int j = 2; j <= Ny - 1; ++j) g.flux_list.push_back(fnode(j, k));
  g.flux_groups[gi++] = (int32_t)g.flux_list.size();
  for (int k = 2; k <= Nz - 1; ++k) g.flux_list.push_back(fnode(1, k));          // south
  g.flux_groups[gi++] = (int32_t)g.flux_list.size();
  for (int k = 2; k <= Nz - 1; ++k) g.flux_list.push_back(fnode(Ny, k));         // north
  g.flux_groups[gi++] = (int32_t)g.flux_list.size();
  for (int j = 2; j <= Ny - 1; ++j) g.flux_list.push_back(fnode(j, Nz));         // front
  g.flux_groups[gi++] = (int32_t)g.flux_list.size();
  for (int j = 2; j <= Ny - 1; ++j) g.flux_list.push_back(fnode(j, 1));          // back
  g.flux_groups[gi++] = (int32_t)g.flux_list.size();
  g.flux_list.push_back(fnode(1, 1));   // SB
  g.flux_groups[gi++] = (int32_t)g.flux_list.size();
  g.flux_list.push_back(fnode(1, Nz));  // SF
  g.flux_groups[gi++] = (int32_t)g.flux_list.size();
  g.flux_list.push_back(fnode(Ny, 1));  // NB
  g.flux_groups[gi++] = (int32_t)g.flux_list.size();
  g.flux_list.push_back(fnode(Ny, Nz)); // NF
  g.flux_groups[gi++] = (int32_t)g.flux_list.size();
  return PIKS_OK;
}

piks_status preprocess(const Setup &s, const uint8_t *raw, int64_t nbytes, Geometry &g, std::string &err) {
  std::vector<uint8_t> box;
  piks_status st = preprocess_box(s, raw, nbytes, box, err);
  if (st) return st;
  classify_host(s, box, g);
  return finish_geometry(s, g, err);
}

}  // namespace piks
