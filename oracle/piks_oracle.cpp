// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT. See piks_oracle.h for scope and the
// list of reference routines restated here. Every function cites the Fortran it follows.
// Build: oracle/Makefile (g++ -O2 -fopenmp -ffp-contract=off; no -march, so no FMA).
#include "piks_oracle.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <chrono>

namespace {

// physicalGrid.F90:127-134
enum : int {
  FLUID = 0, SOLID = 1, GHOST = 4,
  wallE = 20, wallW = 21, wallN = 22, wallS = 23, wallF = 24, wallB = 25,
  wallEN = 30, wallWN = 31, wallES = 32, wallWS = 33,
  wallNF = 40, wallNB = 41, wallSF = 42, wallSB = 43,
  wallEF = 50, wallEB = 51, wallWF = 52, wallWB = 53,
  wallENF = 60, wallWNF = 61, wallWSF = 62, wallESF = 63,
  wallENB = 70, wallWNB = 71, wallWSB = 72, wallESB = 73
};

bool is_wall_label(int v) {  // allWallLabels (physicalGrid.F90:135-141)
  switch (v) {
    case wallE: case wallW: case wallN: case wallS: case wallF: case wallB:
    case wallEN: case wallWN: case wallES: case wallWS:
    case wallNF: case wallNB: case wallSF: case wallSB:
    case wallEF: case wallEB: case wallWF: case wallWB:
    case wallENF: case wallWNF: case wallWSF: case wallESF:
    case wallENB: case wallWNB: case wallWSB: case wallESB: return true;
    default: return false;
  }
}
bool is_3corner(int v) { return v >= 60 && v <= 73 && (v % 10) <= 3; }  // only3CornerLabels
// wallHasE/W/N/S/F/B (physicalGrid.F90:152-174)
bool has_E(int v) { return v == wallE || v == wallEN || v == wallES || v == wallEF || v == wallEB ||
                           v == wallENF || v == wallESF || v == wallENB || v == wallESB; }
bool has_W(int v) { return v == wallW || v == wallWN || v == wallWS || v == wallWF || v == wallWB ||
                           v == wallWNF || v == wallWSF || v == wallWNB || v == wallWSB; }
bool has_N(int v) { return v == wallN || v == wallEN || v == wallWN || v == wallNF || v == wallNB ||
                           v == wallWNF || v == wallENF || v == wallWNB || v == wallENB; }
bool has_S(int v) { return v == wallS || v == wallES || v == wallWS || v == wallSF || v == wallSB ||
                           v == wallWSF || v == wallESF || v == wallWSB || v == wallESB; }
bool has_F(int v) { return v == wallF || v == wallNF || v == wallSF || v == wallEF || v == wallWF ||
                           v == wallENF || v == wallWNF || v == wallWSF || v == wallESF; }
bool has_B(int v) { return v == wallB || v == wallNB || v == wallSB || v == wallEB || v == wallWB ||
                           v == wallENB || v == wallWNB || v == wallWSB || v == wallESB; }

// Gauss-Hermite data (gaussHermite.F90)
struct GHRow { int half, n; double xi[16]; double w[16]; };
const GHRow kGH[] = {
#include "gh_tables.inc"
};

// Wall re-emission program (solver.F90:772-1823)
enum { DIR_PX, DIR_MX, DIR_PY, DIR_MY, DIR_PZ, DIR_MZ };
enum { ST_F, ST_Z, ST_W };
struct WFace { int dir, store; };
struct WWrite { int dst_store, dst_o, face, src_store, src_o; };
struct WProg { int label, nface; WFace face[3]; int nwr; WWrite wr[12]; };
const WProg kWall[] = {
#include "wall_table.inc"
};
const int kIncoming[6][4] = {{2, 3, 6, 7}, {1, 4, 5, 8}, {3, 4, 7, 8},
                             {1, 2, 5, 6}, {5, 6, 7, 8}, {1, 2, 3, 4}};

// Sweep switch rules of solver.F90:184-204 (octant 1) ... :494-513 (octant 8):
// for octant o, a wall of label `lab` at the y-upwind (z-upwind) node gets slot o
// overwritten by slot `src` (src = 0: by fw(which_corner, l, o)) before the read.
struct SwitchRule { int lab, src; };
struct OctSwitch { int ny; SwitchRule y[3]; int nz; SwitchRule z[5]; };
const OctSwitch kSwitch[8] = {
  {3, {{wallEN, 3}, {wallENF, 0}, {wallENB, 0}}, 5, {{wallNF, 8}, {wallEF, 6}, {wallWNF, 0}, {wallESF, 0}, {wallENF, 7}}},
  {3, {{wallWN, 4}, {wallWNF, 0}, {wallWNB, 0}}, 5, {{wallNF, 7}, {wallWF, 5}, {wallENF, 0}, {wallWSF, 0}, {wallWNF, 8}}},
  {3, {{wallWS, 1}, {wallWSF, 0}, {wallWSB, 0}}, 5, {{wallSF, 6}, {wallWF, 8}, {wallWNF, 0}, {wallESF, 0}, {wallWSF, 5}}},
  {3, {{wallES, 2}, {wallESF, 0}, {wallESB, 0}}, 5, {{wallSF, 5}, {wallEF, 7}, {wallENF, 0}, {wallWSF, 0}, {wallESF, 6}}},
  {3, {{wallEN, 7}, {wallENF, 0}, {wallENB, 0}}, 5, {{wallNB, 4}, {wallEB, 2}, {wallESB, 0}, {wallWNB, 0}, {wallENB, 3}}},
  {3, {{wallWN, 8}, {wallWNF, 0}, {wallWNB, 0}}, 5, {{wallNB, 3}, {wallWB, 1}, {wallENB, 0}, {wallWSB, 0}, {wallWNB, 4}}},
  {3, {{wallWS, 8}, {wallWSF, 0}, {wallWSB, 0}}, 5, {{wallSB, 2}, {wallWB, 4}, {wallWNB, 0}, {wallESB, 0}, {wallWSB, 1}}},
  {3, {{wallES, 6}, {wallESF, 0}, {wallESB, 0}}, 5, {{wallSB, 1}, {wallEB, 3}, {wallENB, 0}, {wallWSB, 0}, {wallESB, 2}}},
};
// octant velocity signs (solver.F90 comments :174, :220, :265, :309, :353, :397, :441, :485)
const int kSx[8] = {+1, -1, -1, +1, +1, -1, -1, +1};
const int kSy[8] = {+1, +1, -1, -1, +1, +1, -1, -1};
const int kSz[8] = {+1, +1, +1, +1, -1, -1, -1, -1};

const double PI = std::atan(1.0) * 4.0;  // velocityGrid.F90:78

struct Oracle {
  // namelist / initParams (parameters.F90:87-136)
  int Nx, Ny, Nz, wallExtOrder, fluidlayer;
  double Ref_L;
  int Nc_fundamental, halfRange;
  int block_repx, block_repy, block_repz;
  int maxStep, chkConvergeStep, saveStep;
  double eps;
  int saveLast, saveFormat;
  double Kn, pressDrop, accom;
  int Nx_base, Ny_base, Nz_base;
  int xmin, xmax, ymin, ymax, zmin, zmax;
  // mpiParams: an x-only Cartesian grid of mpi_xdim ranks (mpi_ydim = mpi_zdim = 1)
  int mpi_xdim = 1, rank = 0;
  int xl, xu, yl, yu, zl, zu, xlg, xug, ylg, yug, zlg, zug;
  int Nxtotal, Nytotal, Nztotal, Nxytotal, Nxsub, Nysub, Nzsub;
  size_t Ntotal;
  double ds;
  // velocity grid
  int Nc, Nc8;
  std::vector<double> cx, cy, cz, w;
  double DiffFlux;
  // geometry
  std::vector<int> array3D, array3Dg, image, which_corner;
  int nWall = 0, nCorner = 0, Nfluid = 0;
  std::vector<int> vecWall, mapF;
  std::vector<double> extCoef;
  int Nstencil[8];
  std::vector<int> dir[8];
  std::vector<double> coef[8];
  bool wall_chain = false;  // some wall BC reads another wall's slots (serial order needed)
  // flow
  double mu, mass;
  std::vector<double> f, fw, Rho, Ux, Uy, Uz;
  std::vector<double> west_snd, east_snd, west_rcv, east_rcv;
  int iStep = 0;
  double error = 1.0, permeability = 0.0;
  int nthreads = 1;

  // --- index helpers (Fortran 1-based) ---
  size_t a3(int i, int j, int k) const { return (size_t)(i - 1) + (size_t)(j - 1) * Nx + (size_t)(k - 1) * Nx * Ny; }
  size_t a3g(int i, int j, int k) const {
    return (size_t)(i - xmin + 2) + (size_t)(j - ymin + 2) * (Nx + 4) + (size_t)(k - zmin + 2) * (size_t)(Nx + 4) * (Ny + 4);
  }
  size_t im(int i, int j, int k) const {
    return (size_t)(i - xlg) + (size_t)(j - ylg) * Nxtotal + (size_t)(k - zlg) * Nxytotal;
  }
  long lid(int i, int j, int k) const {  // localid, 1-based
    return (long)(i - xlg + 1) + (long)(j - ylg) * Nxtotal + (long)(k - zlg) * Nxytotal;
  }
  double &F(long k, int l, int o) { return f[(size_t)(k - 1) + (size_t)(l - 1) * Ntotal + (size_t)(o - 1) * Ntotal * Nc8]; }
  double &FW(int c, int l, int o) { return fw[(size_t)(c - 1) + (size_t)(l - 1) * nCorner + (size_t)(o - 1) * (size_t)nCorner * Nc8]; }
  int &IMG(int i, int j, int k) { return image[im(i, j, k)]; }
};

// ---------------------------------------------------------------------------------
// velocityGrid.F90:90-192
bool setup_velocity_grid(Oracle &s, std::string &err) {
  const GHRow *row = nullptr;
  for (const GHRow &r : kGH)
    if (r.half == (s.halfRange ? 1 : 0) && r.n == s.Nc_fundamental) row = &r;
  if (!row) { err = "Nc_fundamental xi/wi for " + std::to_string(s.Nc_fundamental) + " has not been provided"; return false; }
  int n = s.Nc_fundamental;
  std::vector<double> xi(row->xi, row->xi + n), w1(row->w, row->w + n);
  s.Nc = (2 * n) * (2 * n) * (2 * n);
  s.Nc8 = s.Nc / 8;
  s.cx.assign(s.Nc8, 0); s.cy.assign(s.Nc8, 0); s.cz.assign(s.Nc8, 0); s.w.assign(s.Nc8, 0);
  for (int l = 0; l < n; ++l) xi[l] = xi[l] * std::sqrt(2.0);
  for (int l = 1; l <= n; ++l)
    for (int m = 1; m <= n; ++m)
      for (int q = 1; q <= n; ++q) {
        int k = q + (m - 1) * n + (l - 1) * n * n;
        s.cx[k - 1] = xi[q - 1];
        s.cy[k - 1] = xi[m - 1];
        s.cz[k - 1] = xi[l - 1];
        s.w[k - 1] = w1[q - 1] * w1[m - 1] * w1[l - 1];
      }
  double d = 0.0;
  for (int l = 0; l < s.Nc8; ++l) d = d + s.cz[l] * s.w[l];
  s.DiffFlux = d * 4;
  return true;
}

// ---------------------------------------------------------------------------------
// mpiParams.F90:150-191 setupVirtualProcessGrid for dims = (mpi_xdim, 1, 1); the rank's
// Cartesian coordinate is its rank (x-only grid).
void setup_process_grid(Oracle &s) {
  const int dims = s.mpi_xdim, c = s.rank;
  int complete = (s.xmax - s.xmin) / dims;
  int partial = (s.xmax - s.xmin) - complete * dims;
  if (c + 1 <= partial) {
    s.xl = s.xmin + (complete + 1) * c;
    s.xu = s.xmin + (complete + 1) * (c + 1) - 1;
  } else {
    s.xl = s.xmin + complete * c + partial;
    s.xu = s.xmin + complete * (c + 1) + partial - 1;
  }
  if ((c + 1) % dims == 0) s.xu = s.xu + 1;
  complete = (s.ymax - s.ymin) / 1;
  s.yl = s.ymin; s.yu = s.ymin + complete - 1 + 1;
  complete = (s.zmax - s.zmin) / 1;
  s.zl = s.zmin; s.zu = s.zmin + complete - 1 + 1;
  s.xlg = s.xl - 2; s.xug = s.xu + 2;
  s.ylg = s.yl - 2; s.yug = s.yu + 2;
  s.zlg = s.zl - 2; s.zug = s.zu + 2;
}

// physicalGrid.F90:352-377 / :427-452 (drill small pores)
void drill(Oracle &s) {
  auto &g = s.array3Dg;
  auto set_block = [&](int i0, int i1, int j0, int j1, int k0, int k1) {
    for (int k = k0; k <= k1; ++k)
      for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) g[s.a3g(i, j, k)] = FLUID;
  };
  for (int k = 1; k <= s.Nz; ++k)
    for (int j = 1; j <= s.Ny; ++j)
      for (int i = 2; i <= s.Nx - 1; ++i) {
        if (g[s.a3g(i, j, k)] != FLUID) continue;
        bool thin = (g[s.a3g(i + 1, j, k)] != FLUID && g[s.a3g(i - 1, j, k)] != FLUID) ||
                    (g[s.a3g(i, j + 1, k)] != FLUID && g[s.a3g(i, j - 1, k)] != FLUID) ||
                    (g[s.a3g(i, j, k + 1)] != FLUID && g[s.a3g(i, j, k - 1)] != FLUID);
        if (!thin) continue;
        if (j == s.Ny) {
          if (k == s.Nz) set_block(i, i + 1, j - 1, j, k - 1, k);
          else set_block(i, i + 1, j - 1, j, k, k + 1);
        } else if (k == s.Nz) {
          set_block(i, i + 1, j, j + 1, k - 1, k);
        } else {
          set_block(i, i + 1, j, j + 1, k, k + 1);
        }
      }
}

// physicalGrid.F90:382-391 / :413-422 (ghost <-> fluid toggling)
void set_ghost_layers(Oracle &s, int value) {
  for (int k = s.zmin - 2; k <= s.zmax + 2; ++k)
    for (int j = s.ymin - 2; j <= s.ymax + 2; ++j)
      for (int i = s.xmin - 2; i <= s.xmax + 2; ++i)
        if (k < s.zmin || k > s.zmax || j < s.ymin || j > s.ymax || i < s.xmin || i > s.xmax)
          s.array3Dg[s.a3g(i, j, k)] = value;
}

// physicalGrid.F90:396-408 / :471-483 (remove 1-voxel walls, in place)
void thin(Oracle &s) {
  auto &g = s.array3Dg;
  for (int k = 1; k <= s.Nz; ++k)
    for (int j = 1; j <= s.Ny; ++j)
      for (int i = 1; i <= s.Nx; ++i) {
        if (g[s.a3g(i, j, k)] != SOLID) continue;
        if ((g[s.a3g(i + 1, j, k)] == FLUID && g[s.a3g(i - 1, j, k)] == FLUID) ||
            (g[s.a3g(i, j + 1, k)] == FLUID && g[s.a3g(i, j - 1, k)] == FLUID) ||
            (g[s.a3g(i, j, k + 1)] == FLUID && g[s.a3g(i, j, k - 1)] == FLUID))
          g[s.a3g(i, j, k)] = FLUID;
      }
}

int label_of_product(int p) {  // physicalGrid.F90:562-667
  switch (p) {
    case 2: return wallE; case 3: return wallW; case 5: return wallN; case 7: return wallS;
    case 9: return wallF; case 11: return wallB;
    case 10: return wallEN; case 15: return wallWN; case 14: return wallES; case 21: return wallWS;
    case 18: return wallEF; case 22: return wallEB; case 27: return wallWF; case 33: return wallWB;
    case 45: return wallNF; case 55: return wallNB; case 63: return wallSF; case 77: return wallSB;
    case 90: return wallENF; case 110: return wallENB; case 135: return wallWNF; case 165: return wallWNB;
    case 126: return wallESF; case 154: return wallESB; case 189: return wallWSF; case 231: return wallWSB;
    default: return -1;
  }
}

// physicalGrid.F90:217-1625
bool setup_physical_grid(Oracle &s, const uint8_t *raw, int64_t nbytes, std::string &err) {
  s.ds = 1.0 / (s.Nx - 1 - 2 * s.fluidlayer);
  s.Nxtotal = s.xug - s.xlg + 1;
  s.Nytotal = s.yug - s.ylg + 1;
  s.Nztotal = s.zug - s.zlg + 1;
  s.Nxytotal = s.Nxtotal * s.Nytotal;
  s.Nxsub = s.xu - s.xl + 1;
  s.Nysub = s.yu - s.yl + 1;
  s.Nzsub = s.zu - s.zl + 1;
  s.Ntotal = (size_t)s.Nxtotal * s.Nytotal * s.Nztotal;

  s.array3D.assign((size_t)s.Nx * s.Ny * s.Nz, FLUID);
  s.array3Dg.assign((size_t)(s.Nx + 4) * (s.Ny + 4) * (s.Nz + 4), FLUID);
  s.image.assign(s.Ntotal, FLUID);
  s.which_corner.assign(s.Ntotal, 0);

  // :257-280 stream read, i fastest
  int64_t need = (int64_t)s.Nz_base * s.Ny_base * (s.Nx_base - 2 * s.fluidlayer);
  if (nbytes < need) { err = "image stream shorter than Nx*Ny*Nz bytes"; return false; }
  int64_t pos = 0;
  for (int k = 1; k <= s.Nz_base; ++k)
    for (int j = 1; j <= s.Ny_base; ++j)
      for (int i = s.fluidlayer + 1; i <= s.Nx_base - s.fluidlayer; ++i) {
        uint8_t c = raw[pos++];
        if (c == 0) s.array3D[s.a3(i, j, k)] = FLUID;
        else if (c == 1) s.array3D[s.a3(i, j, k)] = SOLID;
        else { err = "invalid image data file"; return false; }
      }
  // :285-298 block replication
  for (int k = 0; k < s.block_repz; ++k)
    for (int j = 0; j < s.block_repy; ++j)
      for (int i = 0; i < s.block_repx; ++i)
        for (int kk = 1; kk <= s.Nz_base; ++kk)
          for (int jj = 1; jj <= s.Ny_base; ++jj)
            for (int ii = 1; ii <= s.Nx_base; ++ii)
              s.array3D[s.a3(i * s.Nx_base + ii, j * s.Ny_base + jj, k * s.Nz_base + kk)] = s.array3D[s.a3(ii, jj, kk)];
  // :303-314 ghost + inner
  for (int k = s.zmin - 2; k <= s.zmax + 2; ++k)
    for (int j = s.ymin - 2; j <= s.ymax + 2; ++j)
      for (int i = s.xmin - 2; i <= s.xmax + 2; ++i) {
        bool gh = k < s.zmin || k > s.zmax || j < s.ymin || j > s.ymax || i < s.xmin || i > s.xmax;
        s.array3Dg[s.a3g(i, j, k)] = gh ? GHOST : s.array3D[s.a3(i, j, k)];
      }
  // :352-497 two rounds of drill + thin
  for (int round = 0; round < 2; ++round) {
    drill(s);
    set_ghost_layers(s, FLUID);
    thin(s);
    set_ghost_layers(s, GHOST);
  }
  // :503-509
  for (int k = s.zmin; k <= s.zmax; ++k)
    for (int j = s.ymin; j <= s.ymax; ++j)
      for (int i = s.xmin; i <= s.xmax; ++i) s.array3D[s.a3(i, j, k)] = s.array3Dg[s.a3g(i, j, k)];
  // :512-543 local image (single rank: whole box) + ghost flags
  for (int k = s.zlg; k <= s.zug; ++k)
    for (int j = s.ylg; j <= s.yug; ++j)
      for (int i = s.xlg; i <= s.xug; ++i) {
        bool gh = i < s.xmin || i > s.xmax || j < s.ymin || j > s.ymax || k < s.zmin || k > s.zmax;
        s.IMG(i, j, k) = gh ? GHOST : s.array3Dg[s.a3g(i, j, k)];
      }
  // :546-671 wall labels from the product of fluid-neighbour primes, over :512-523's
  // bounds: the rank's own planes plus its ghost planes where a neighbour rank owns them
  s.nWall = 0;
  const int lxl = s.xl == s.xmin ? s.xl : s.xlg, lxu = s.xu == s.xmax ? s.xu : s.xug;
  for (int k = s.zl; k <= s.zu; ++k)
    for (int j = s.yl; j <= s.yu; ++j)
      for (int i = lxl; i <= lxu; ++i) {
        if (s.array3D[s.a3(i, j, k)] != SOLID) continue;
        int p = 1;
        const auto &g = s.array3Dg;
        if (g[s.a3g(i + 1, j, k)] == FLUID) p *= 2;
        if (g[s.a3g(i - 1, j, k)] == FLUID) p *= 3;
        if (g[s.a3g(i, j + 1, k)] == FLUID) p *= 5;
        if (g[s.a3g(i, j - 1, k)] == FLUID) p *= 7;
        if (g[s.a3g(i, j, k + 1)] == FLUID) p *= 9;
        if (g[s.a3g(i, j, k - 1)] == FLUID) p *= 11;
        int lab = label_of_product(p);
        if (lab >= 0) { s.IMG(i, j, k) = lab; s.nWall++; }
      }
  // :682-748 vecWall (raster order) and which_corner
  s.vecWall.clear();
  s.nCorner = 0;
  for (int k = s.zlg; k <= s.zug; ++k)
    for (int j = s.ylg; j <= s.yug; ++j)
      for (int i = s.xlg; i <= s.xug; ++i) {
        int v = s.IMG(i, j, k);
        if (!is_wall_label(v)) continue;
        if (j >= s.yl && j <= s.yu && i >= s.xl && i <= s.xu && k >= s.zl && k <= s.zu)
          s.vecWall.push_back((int)s.lid(i, j, k));
        if (is_3corner(v)) { s.nCorner++; s.which_corner[s.im(i, j, k)] = s.nCorner; }
      }
  s.nWall = (int)s.vecWall.size();
  s.fw.assign((size_t)s.nCorner * s.Nc8 * 8, 0.0);
  // :891-948 extrapolation coefficients. For wallExtOrder == 3 the per-wall override
  // decodes (i,j,k) from the 1-based local id as :897-899 does (i comes out one larger
  // than the wall's own x); restated as written.
  s.extCoef.assign((size_t)s.nWall * 2, 0.0);
  for (int l = 0; l < s.nWall; ++l) { s.extCoef[l] = 2.0; s.extCoef[s.nWall + l] = -1.0; }
  for (int l = 0; l < s.nWall; ++l) {
    long localid = s.vecWall[l];
    int k = s.zlg + (int)(localid / s.Nxytotal);
    int j = s.ylg + (int)((localid - (long)(k - s.zlg) * s.Nxytotal) / s.Nxtotal);
    int i = s.xlg + (int)(localid - (long)(k - s.zlg) * s.Nxytotal - (long)(j - s.ylg) * s.Nxtotal);
    int v = s.IMG(i, j, k);
    auto first = [&]() { s.extCoef[l] = 1.0; s.extCoef[s.nWall + l] = 0.0; };
    if (has_W(v) && i == s.xl + 1 && s.IMG(s.xl, j, k) == FLUID) first();
    if (has_E(v) && i == s.xu - 1 && s.IMG(s.xu, j, k) == FLUID) first();
    if (has_S(v) && j == s.yl + 1 && s.IMG(i, s.yl, k) == FLUID) first();
    if (has_N(v) && j == s.yu - 1 && s.IMG(i, s.yu, k) == FLUID) first();
    if (has_B(v) && k == s.zl + 1 && s.IMG(i, j, s.zl) == FLUID) first();
    if (has_F(v) && k == s.zu - 1 && s.IMG(i, j, s.zu) == FLUID) first();
  }
  if (s.wallExtOrder == 2) {
    for (int l = 0; l < s.nWall; ++l) { s.extCoef[l] = 2.0; s.extCoef[s.nWall + l] = -1.0; }
  } else if (s.wallExtOrder == 1) {
    for (int l = 0; l < s.nWall; ++l) { s.extCoef[l] = 1.0; s.extCoef[s.nWall + l] = 0.0; }
  } else if (s.wallExtOrder != 3) {
    std::fprintf(stderr, " Error: wallExtOrder wroond shoud be [1|2|3]\n");
  }
  // :951-974 mapF
  s.mapF.clear();
  for (int k = s.zl; k <= s.zu; ++k)
    for (int j = s.yl; j <= s.yu; ++j)
      for (int i = s.xl; i <= s.xu; ++i)
        if (s.IMG(i, j, k) == FLUID) s.mapF.push_back((int)s.lid(i, j, k));
  s.Nfluid = (int)s.mapF.size();
  // :976-1246 sweep lists; :1249-1622 upwind coefficients
  for (int o = 0; o < 8; ++o) {
    int sx = kSx[o], sy = kSy[o], sz = kSz[o];
    int bxl = s.xl, bxu = s.xu, byl = s.yl, byu = s.yu, bzl = s.zl, bzu = s.zu;
    // :976-985: the first plane along the sweep is an inflow plane only at the box's edge
    if (sx > 0) { if (s.xl == s.xmin) bxl = s.xl + 1; } else { if (s.xu == s.xmax) bxu = s.xu - 1; }
    if (sy > 0) byl = s.yl + 1; else byu = s.yu - 1;
    if (sz > 0) bzl = s.zl + 1; else bzu = s.zu - 1;
    auto &d = s.dir[o];
    d.clear();
    for (int kq = 0; kq <= bzu - bzl; ++kq) {
      int k = sz > 0 ? bzl + kq : bzu - kq;
      for (int jq = 0; jq <= byu - byl; ++jq) {
        int j = sy > 0 ? byl + jq : byu - jq;
        for (int iq = 0; iq <= bxu - bxl; ++iq) {
          int i = sx > 0 ? bxl + iq : bxu - iq;
          if (s.IMG(i, j, k) == FLUID) { d.push_back(i); d.push_back(j); d.push_back(k); }
        }
      }
    }
    int n = (int)d.size() / 3;
    s.Nstencil[o] = n;
    auto &c = s.coef[o];
    c.assign((size_t)n * 9, 0.0);
    for (int q = 0; q < n; ++q) {
      int ii = d[3 * q], jj = d[3 * q + 1], kk = d[3 * q + 2];
      double C[9];
      C[0] = sx > 0 ? 1.5 / s.ds : -1.5 / s.ds;
      C[1] = sx > 0 ? 2.0 / s.ds : -2.0 / s.ds;
      C[2] = sx > 0 ? -0.5 / s.ds : 0.5 / s.ds;
      C[3] = sy > 0 ? 1.5 / s.ds : -1.5 / s.ds;
      C[4] = sy > 0 ? 2.0 / s.ds : -2.0 / s.ds;
      C[5] = sy > 0 ? -0.5 / s.ds : 0.5 / s.ds;
      C[6] = sz > 0 ? 1.5 / s.ds : -1.5 / s.ds;
      C[7] = sz > 0 ? 2.0 / s.ds : -2.0 / s.ds;
      C[8] = sz > 0 ? -0.5 / s.ds : 0.5 / s.ds;
      bool fx = sx > 0 ? (s.IMG(ii - 2, jj, kk) == GHOST || has_E(s.IMG(ii - 1, jj, kk)))
                       : (s.IMG(ii + 2, jj, kk) == GHOST || has_W(s.IMG(ii + 1, jj, kk)));
      bool fy = sy > 0 ? (s.IMG(ii, jj - 2, kk) == GHOST || has_N(s.IMG(ii, jj - 1, kk)))
                       : (s.IMG(ii, jj + 2, kk) == GHOST || has_S(s.IMG(ii, jj + 1, kk)));
      bool fz = sz > 0 ? (s.IMG(ii, jj, kk - 2) == GHOST || has_F(s.IMG(ii, jj, kk - 1)))
                       : (s.IMG(ii, jj, kk + 2) == GHOST || has_B(s.IMG(ii, jj, kk + 1)));
      if (fx) { C[0] = sx > 0 ? 1.0 / s.ds : -1.0 / s.ds; C[1] = C[0]; C[2] = 0.0; }
      if (fy) { C[3] = sy > 0 ? 1.0 / s.ds : -1.0 / s.ds; C[4] = C[3]; C[5] = 0.0; }
      if (fz) { C[6] = sz > 0 ? 1.0 / s.ds : -1.0 / s.ds; C[7] = C[6]; C[8] = 0.0; }
      for (int t = 0; t < 9; ++t) c[(size_t)t * n + q] = C[t];
    }
  }
  // Does any wall's extrapolation read a node that is itself a wall? If so the wall
  // pass must run in the serial vecWall order (solver.F90:762 is an OMP DO whose result
  // then depends on the thread schedule; the single-thread order is the defined one).
  s.wall_chain = false;
  const long offs[6] = {+1, -1, +s.Nxtotal, -s.Nxtotal, +s.Nxytotal, -s.Nxytotal};
  for (int q = 0; q < s.nWall && !s.wall_chain; ++q) {
    long k = s.vecWall[q];
    int v = s.image[k - 1];
    for (const WProg &P : kWall)
      if (P.label == v)
        for (int fi = 0; fi < P.nface; ++fi)
          for (int m = 1; m <= 2; ++m)
            if (is_wall_label(s.image[k - 1 + m * offs[P.face[fi].dir]])) s.wall_chain = true;
  }
  return true;
}

// flow.F90:76-113 and :115-163 (face part of the x buffers; y/z receive buffers stay 0)
void setup_flow(Oracle &s) {
  s.f.assign(s.Ntotal * s.Nc8 * 8, 0.0);
  s.Rho.assign(s.Ntotal, 0.0);
  s.Ux.assign(s.Ntotal, 0.0);
  s.Uy.assign(s.Ntotal, 0.0);
  s.Uz.assign(s.Ntotal, 0.0);
  s.mu = std::sqrt(PI / 2.0) / s.Kn;
  s.mass = 1.0;
  size_t face = (size_t)s.Nytotal * s.Nztotal * 2 * s.Nc;
  s.west_snd.assign(face, 0.0); s.east_snd.assign(face, 0.0);
  s.west_rcv.assign(face, 0.0); s.east_rcv.assign(face, 0.0);
}

// ---------------------------------------------------------------------------------
// solver.F90:176-526, one octant for one velocity index l (0-based o, 1-based l)
void sweep_octant_l(Oracle &s, int o, int l) {
  const int sx = kSx[o], sy = kSy[o], sz = kSz[o];
  const int O = o + 1;
  const long NX = s.Nxtotal, NXY = s.Nxytotal;
  const double cxl = s.cx[l - 1], cyl = s.cy[l - 1], czl = s.cz[l - 1], wl = s.w[l - 1];
  const double mu = s.mu;
  const int n = s.Nstencil[o];
  const int *d = s.dir[o].data();
  const double *c = s.coef[o].data();
  const OctSwitch &sw = kSwitch[o];
  for (int q = 0; q < n; ++q) {
    int ii = d[3 * q], jj = d[3 * q + 1], kk = d[3 * q + 2];
    long k = s.lid(ii, jj, kk);
    // switch at the y-upwind wall node (:186-191 for octant 1)
    {
      int vy = s.IMG(ii, jj - sy, kk);
      long ky = k - sy * NX;
      for (int r = 0; r < sw.ny; ++r)
        if (vy == sw.y[r].lab) {
          s.F(ky, l, O) = sw.y[r].src ? s.F(ky, l, sw.y[r].src)
                                      : s.FW(s.which_corner[s.im(ii, jj - sy, kk)], l, O);
          break;
        }
      int vz = s.IMG(ii, jj, kk - sz);
      long kz = k - sz * NXY;
      for (int r = 0; r < sw.nz; ++r)
        if (vz == sw.z[r].lab) {
          s.F(kz, l, O) = sw.z[r].src ? s.F(kz, l, sw.z[r].src)
                                      : s.FW(s.which_corner[s.im(ii, jj, kk - sz)], l, O);
          break;
        }
    }
    // fEq (:206)
    double ex = cxl * s.Ux[k - 1]; if (sx < 0) ex = -ex;
    double ey = cyl * s.Uy[k - 1]; if (sy < 0) ey = -ey;
    double ez = czl * s.Uz[k - 1]; if (sz < 0) ez = -ez;
    double fEq = wl * (s.Rho[k - 1] + 1.0 * ((ex + ey) + ez));
    // update (:207-214), left-to-right; a negative-sign octant subtracts its term
    double num = mu * (fEq - 0.5 * s.F(k, l, O));
    double t;
    t = cxl * c[(size_t)1 * n + q] * s.F(k - sx, l, O);        num = sx > 0 ? num + t : num - t;
    t = cxl * c[(size_t)2 * n + q] * s.F(k - 2 * sx, l, O);    num = sx > 0 ? num + t : num - t;
    t = cyl * c[(size_t)4 * n + q] * s.F(k - sy * NX, l, O);   num = sy > 0 ? num + t : num - t;
    t = cyl * c[(size_t)5 * n + q] * s.F(k - 2 * sy * NX, l, O); num = sy > 0 ? num + t : num - t;
    t = czl * c[(size_t)7 * n + q] * s.F(k - sz * NXY, l, O);  num = sz > 0 ? num + t : num - t;
    t = czl * c[(size_t)8 * n + q] * s.F(k - 2 * sz * NXY, l, O); num = sz > 0 ? num + t : num - t;
    double den = 0.5 * mu;
    t = cxl * c[(size_t)0 * n + q]; den = sx > 0 ? den + t : den - t;
    t = cyl * c[(size_t)3 * n + q]; den = sy > 0 ? den + t : den - t;
    t = czl * c[(size_t)6 * n + q]; den = sz > 0 ? den + t : den - t;
    s.F(k, l, O) = num / den;
  }
}

// solver.F90:761-1826, one wall (vecWall index q, 0-based); fwZ is per-thread scratch
void wall_bc(Oracle &s, int q, std::vector<double> &fwZ) {
  const long k = s.vecWall[q];
  const int lab = s.image[k - 1];
  const WProg *P = nullptr;
  for (const WProg &p : kWall) if (p.label == lab) P = &p;
  if (!P) return;
  const int c = s.which_corner[k - 1];
  const double e1 = s.extCoef[q], e2 = s.extCoef[s.nWall + q];
  const long offs[6] = {+1, -1, +s.Nxtotal, -s.Nxtotal, +s.Nxytotal, -s.Nxytotal};
  const int Nc8 = s.Nc8;
  auto slot = [&](int store, int l, int oo) -> double & {
    if (store == ST_F) return s.F(k, l, oo);
    if (store == ST_W) return s.FW(c, l, oo);
    return fwZ[(size_t)(oo - 1) * Nc8 + (l - 1)];
  };
  double rho[3] = {0.0, 0.0, 0.0};
  for (int l = 1; l <= Nc8; ++l) {
    for (int fi = 0; fi < P->nface; ++fi) {
      const long dd = offs[P->face[fi].dir];
      for (int m = 0; m < 4; ++m) {
        int oo = kIncoming[P->face[fi].dir][m];
        slot(P->face[fi].store, l, oo) = e1 * s.F(k + dd, l, oo) + e2 * s.F(k + 2 * dd, l, oo);
      }
    }
    for (int fi = 0; fi < P->nface; ++fi) {
      int dir = P->face[fi].dir;
      double ca = dir < 2 ? s.cx[l - 1] : dir < 4 ? s.cy[l - 1] : s.cz[l - 1];
      const int *in = kIncoming[dir];
      int st = P->face[fi].store;
      rho[fi] = rho[fi] + ca * (slot(st, l, in[0]) + slot(st, l, in[1]) + slot(st, l, in[2]) + slot(st, l, in[3]));
    }
  }
  for (int fi = 0; fi < P->nface; ++fi) rho[fi] = rho[fi] / s.DiffFlux;
  for (int l = 1; l <= Nc8; ++l) {
    for (int r = 0; r < P->nwr; ++r) {
      const WWrite &W = P->wr[r];
      double v = s.accom * s.w[l - 1] * rho[W.face] + (1.0 - s.accom) * slot(W.src_store, l, W.src_o);
      slot(W.dst_store, l, W.dst_o) = v;
    }
  }
}

// solver.F90:111-1940
void iterate(Oracle &s) {
  // :146-170: the west/east messages are the buffers packed during the previous
  // iteration; y/z neighbours are MPI_PROC_NULL. On one rank the x neighbours are the rank
  // itself; with several ranks the caller moves the messages before the call
  // (oracle_halo_send / oracle_halo_recv). The 3-fold-corner part of the x message is not
  // carried: on one rank it has no receiving map (map3CorWrcv/Ercv are empty), and with
  // several ranks it fills fw slots of corners in the ghost planes, which no statement
  // reads (the sweep's switch reads fw of a corner in the swept voxel's own x plane, the
  // wall loop only its own walls' slots). (The reference's MPI receive count on one rank
  // excludes it: with 3-fold corners in the planes x = 1, 2, Nx-1, Nx its MPI_WAITALL would
  // report a truncated message.)
  if (s.mpi_xdim == 1) {
    s.east_rcv = s.west_snd;
    s.west_rcv = s.east_snd;
  }
  const int Nc8 = s.Nc8;
#pragma omp parallel num_threads(s.nthreads)
  {
    for (int o = 0; o < 8; ++o) {
#pragma omp for schedule(static) nowait
      for (int l = 1; l <= Nc8; ++l) sweep_octant_l(s, o, l);
    }
  }
  // :535-612 pack/unpack
  const long NX = s.Nxtotal, NXY = s.Nxytotal;
  const int Nc = s.Nc;
  for (int k = 1; k <= s.Nztotal; ++k)
    for (int j = 1; j <= s.Nytotal; ++j)
      for (int i = 1; i <= 2; ++i) {
        long Msnd = (long)(k - 1) * NXY + (long)(j - 1) * NX + i + 2;
        long Mrcv = (long)(k - 1) * NXY + (long)(j - 1) * NX + i;
        long Psnd = (long)(k - 1) * NXY + (long)(j - 1) * NX + i + s.Nxsub;
        long Prcv = (long)(k - 1) * NXY + (long)(j - 1) * NX + i + 2 + s.Nxsub;
        size_t packid = (size_t)(k - 1) * s.Nytotal * 2 * Nc + (size_t)(j - 1) * 2 * Nc + (size_t)(i - 1) * Nc;
        for (int o = 1; o <= 8; ++o)
          for (int l = 1; l <= Nc8; ++l) {
            size_t b = packid + (size_t)(o - 1) * Nc8 + (l - 1);
            s.west_snd[b] = s.F(Msnd, l, o);
            s.F(Mrcv, l, o) = s.west_rcv[b];
            s.east_snd[b] = s.F(Psnd, l, o);
            s.F(Prcv, l, o) = s.east_rcv[b];
          }
      }
  for (int k = 1; k <= s.Nztotal; ++k)
    for (int j = 1; j <= 2; ++j)
      for (int i = 1; i <= s.Nxtotal; ++i) {
        long Mrcv = (long)(k - 1) * NXY + (long)(j - 1) * NX + i;
        long Prcv = (long)(k - 1) * NXY + (long)(j + s.Nysub + 2 - 1) * NX + i;
        for (int o = 1; o <= 8; ++o)
          for (int l = 1; l <= Nc8; ++l) { s.F(Mrcv, l, o) = 0.0; s.F(Prcv, l, o) = 0.0; }
      }
  for (int k = 1; k <= 2; ++k)
    for (int j = 1; j <= s.Nytotal; ++j)
      for (int i = 1; i <= s.Nxtotal; ++i) {
        long Mrcv = (long)(k - 1) * NXY + (long)(j - 1) * NX + i;
        long Prcv = (long)(k + s.Nzsub + 2 - 1) * NXY + (long)(j - 1) * NX + i;
        for (int o = 1; o <= 8; ++o)
          for (int l = 1; l <= Nc8; ++l) { s.F(Mrcv, l, o) = 0.0; s.F(Prcv, l, o) = 0.0; }
      }
  // :761-1826 wall boundary condition
  if (s.wall_chain) {
    std::vector<double> fwZ((size_t)Nc8 * 8, 0.0);
    for (int q = 0; q < s.nWall; ++q) wall_bc(s, q, fwZ);
  } else {
#pragma omp parallel num_threads(s.nthreads)
    {
      std::vector<double> fwZ((size_t)Nc8 * 8, 0.0);
#pragma omp for schedule(static)
      for (int q = 0; q < s.nWall; ++q) wall_bc(s, q, fwZ);
    }
  }
  // :1832-1862 inlet on the west-most rank, outlet on the east-most (whole ghosted y-z extent)
  if (s.xl == s.xmin)
    for (int k = s.zlg; k <= s.zug; ++k)
      for (int j = s.ylg; j <= s.yug; ++j) {
        long l = s.lid(s.xl, j, k);
        for (int o : {1, 4, 5, 8})
          for (int v = 1; v <= Nc8; ++v) s.F(l, v, o) = s.F(l - 1, v, o) + s.w[v - 1] * s.pressDrop;
      }
  if (s.xu == s.xmax)
    for (int k = s.zlg; k <= s.zug; ++k)
      for (int j = s.ylg; j <= s.yug; ++j) {
        long l = s.lid(s.xu, j, k);
        for (int o : {2, 3, 6, 7})
          for (int v = 1; v <= Nc8; ++v) s.F(l, v, o) = s.F(l + 1, v, o) - s.w[v - 1] * s.pressDrop;
      }
  // :1867-1918 symmetry planes
  auto copy = [&](long l, int dst, int src) {
    for (int v = 1; v <= Nc8; ++v) s.F(l, v, dst) = s.F(l, v, src);
  };
  for (int k = s.zl; k <= s.zu; ++k)
    for (int i = s.xl; i <= s.xu; ++i) {
      long l = s.lid(i, s.yl, k);
      copy(l, 2, 3); copy(l, 1, 4); copy(l, 6, 7); copy(l, 5, 8);
    }
  for (int k = s.zl; k <= s.zu; ++k)
    for (int i = s.xl; i <= s.xu; ++i) {
      long l = s.lid(i, s.yu, k);
      copy(l, 3, 2); copy(l, 4, 1); copy(l, 7, 6); copy(l, 8, 5);
    }
  for (int j = s.yl; j <= s.yu; ++j)
    for (int i = s.xl; i <= s.xu; ++i) {
      long l = s.lid(i, j, s.zl);
      copy(l, 1, 5); copy(l, 2, 6); copy(l, 3, 7); copy(l, 4, 8);
    }
  for (int j = s.yl; j <= s.yu; ++j)
    for (int i = s.xl; i <= s.xu; ++i) {
      long l = s.lid(i, j, s.zu);
      copy(l, 5, 1); copy(l, 6, 2); copy(l, 7, 3); copy(l, 8, 4);
    }
  // :1923-1938 moments
#pragma omp parallel for schedule(static) num_threads(s.nthreads)
  for (int q = 0; q < s.Nfluid; ++q) {
    long k = s.mapF[q];
    double r = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
    for (int l = 1; l <= Nc8; ++l) {
      double f1 = s.F(k, l, 1), f2 = s.F(k, l, 2), f3 = s.F(k, l, 3), f4 = s.F(k, l, 4);
      double f5 = s.F(k, l, 5), f6 = s.F(k, l, 6), f7 = s.F(k, l, 7), f8 = s.F(k, l, 8);
      r = r + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8;
      ux = ux + s.cx[l - 1] * (f1 - f2 - f3 + f4 + f5 - f6 - f7 + f8);
      uy = uy + s.cy[l - 1] * (f1 + f2 - f3 - f4 + f5 + f6 - f7 - f8);
      uz = uz + s.cz[l - 1] * (f1 + f2 + f3 + f4 - f5 - f6 - f7 - f8);
    }
    s.Rho[k - 1] = r; s.Ux[k - 1] = ux; s.Uy[k - 1] = uy; s.Uz[k - 1] = uz;
  }
}

// Fortran ESw.d edit descriptor (w = 15, d = 6): one leading digit, exponent E+dd;
// exponents beyond two digits drop the E, as Fortran does.
std::string es15_6(double v) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.6E", v);
  std::string s(buf);
  size_t e = s.find('E');
  if (e != std::string::npos) {
    std::string mant = s.substr(0, e), ex = s.substr(e + 1);
    int x = std::atoi(ex.c_str());
    char eb[16];
    if (std::abs(x) >= 100) std::snprintf(eb, sizeof eb, "%+04d", x);
    else std::snprintf(eb, sizeof eb, "E%c%02d", x < 0 ? '-' : '+', std::abs(x));
    s = mant + eb;
  }
  if (s.size() < 15) s = std::string(15 - s.size(), ' ') + s;
  return s;
}

// output.F90:60-164
void chk_converge(Oracle &s, const char *results_path, int verbose) {
  // :89: only the west-most rank holds the plane x = 2 (its caller broadcasts the result,
  // :162); with x-only ranks the inlet communicator has that one rank, so the reduction of
  // :144-145 is the rank's own value
  if (s.xl != s.xmin) return;
  int byl = s.yl + 1, byu = s.yu - 1, bzl = s.zl + 1, bzu = s.zu - 1;
  const long NX = s.Nxtotal, NXY = s.Nxytotal;
  const int col = 2 + 2;  // column + ghostLayers
  double ds = s.ds;
  double mInner = 0, mNoth = 0, mSuth = 0, mFrnt = 0, mBack = 0, mNF = 0, mNB = 0, mSF = 0, mSB = 0;
  for (int k = bzl; k <= bzu; ++k)
    for (int j = byl; j <= byu; ++j) {
      long l = (long)(k - s.zlg) * NXY + (long)(j - s.ylg) * NX + col;
      mInner = mInner + s.Ux[l - 1] * ds * ds;
    }
  for (int k = bzl; k <= bzu; ++k) {
    long l = (long)(k - s.zlg) * NXY + 2 * NX + col;
    mSuth = mSuth + s.Ux[l - 1] * ds * ds * 0.5;
  }
  for (int k = bzl; k <= bzu; ++k) {
    long l = (long)(k - s.zlg) * NXY + (long)(s.Nysub + 1) * NX + col;
    mNoth = mNoth + s.Ux[l - 1] * ds * ds * 0.5;
  }
  for (int j = byl; j <= byu; ++j) {
    long l = 2 * NXY + (long)(j - s.ylg) * NX + col;
    mBack = mBack + s.Ux[l - 1] * ds * ds * 0.5;
  }
  for (int j = byl; j <= byu; ++j) {
    long l = (long)(s.Nzsub + 1) * NXY + (long)(j - s.ylg) * NX + col;
    mFrnt = mFrnt + s.Ux[l - 1] * ds * ds * 0.5;
  }
  mSB = s.Ux[2 * NXY + 2 * NX + col - 1] * ds * ds * 0.25;
  mSF = s.Ux[(long)(s.Nzsub + 1) * NXY + 2 * NX + col - 1] * ds * ds * 0.25;
  mNB = s.Ux[2 * NXY + (long)(s.Nysub + 1) * NX + col - 1] * ds * ds * 0.25;
  mNF = s.Ux[(long)(s.Nzsub + 1) * NXY + (long)(s.Nysub + 1) * NX + col - 1] * ds * ds * 0.25;
  double inv = 1.0 / s.Ref_L;
  double massLocal = (mInner + mSuth + mNoth + mFrnt + mBack + mSB + mSF + mNB + mNF) *
                     std::sqrt(1.0 / 2.0) / s.pressDrop / (inv * inv);
  double mass2 = massLocal;  // MPI_ALLREDUCE over one rank
  s.error = std::fabs(1.0 - mass2 / s.mass) / (double)s.chkConvergeStep;
  s.mass = mass2;
  s.permeability = s.mass * s.Kn * std::sqrt(4.0 / PI);
  if (verbose) std::printf("%10d%s%s%s\n", s.iStep, es15_6(s.mass).c_str(), es15_6(s.permeability).c_str(), es15_6(s.error).c_str());
  if (results_path && results_path[0]) {
    FILE *fh = std::fopen(results_path, "a");
    if (fh) {
      std::fprintf(fh, "%s%s%s%s%15d\n", es15_6(s.Kn).c_str(), es15_6(s.mass).c_str(),
                   es15_6(s.permeability).c_str(), es15_6(s.error).c_str(), s.iStep);
      std::fclose(fh);
    }
  }
}

int save_fields(Oracle &s, const char *dir, int format) {
  std::string d = dir ? dir : ".";
  auto val = [&](int i, int j, int k, double *r, double *u, double *v, double *ww) {
    long l = s.lid(i, j, k);
    if (s.IMG(i, j, k) == FLUID) { *r = s.Rho[l - 1] + 1.0; *u = s.Ux[l - 1]; *v = s.Uy[l - 1]; *ww = s.Uz[l - 1]; return true; }
    *r = 0; *u = 0; *v = 0; *ww = 0; return false;
  };
  if (format == 1) {  // output.F90:250-360
    FILE *fh = std::fopen((d + "/Field_000.vti").c_str(), "w");
    if (!fh) return -1;
    std::fprintf(fh, "<?xml version=\"1.0\"?>\n<VTKFile type=\"ImageData\">\n");
    std::fprintf(fh, "<ImageData WholeExtent=\"%4d%4d%4d%4d%4d%4d \" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n",
                 s.xmin - 1, s.xmax, s.ymin - 1, s.ymax, s.zmin - 1, s.zmax);
    std::fprintf(fh, "<Piece Extent=\"%4d%4d%4d%4d%4d%4d\">\n", s.xl - 1, s.xu, s.yl - 1, s.yu, s.zl - 1, s.zu);
    std::fprintf(fh, "<CellData Scalars=\"flag Rho\" Vectors =\"U\">\n");
    std::fprintf(fh, "<DataArray type=\"Int32\" Name=\"flag\" format=\"ascii\">\n");
    for (int k = s.zl; k <= s.zu; ++k)
      for (int j = s.yl; j <= s.yu; ++j)
        for (int i = s.xl; i <= s.xu; ++i) std::fprintf(fh, "%2d\n", s.IMG(i, j, k));
    std::fprintf(fh, "</DataArray>\n<DataArray type=\"Float32\" Name=\"Rho\" format=\"ascii\">\n");
    for (int k = s.zl; k <= s.zu; ++k)
      for (int j = s.yl; j <= s.yu; ++j)
        for (int i = s.xl; i <= s.xu; ++i) { double r, u, v, ww; val(i, j, k, &r, &u, &v, &ww); std::fprintf(fh, "%s\n", es15_6(r).c_str()); }
    std::fprintf(fh, "</DataArray>\n<DataArray type=\"Float32\" Name=\"U\" format=\"ascii\" NumberOfComponents=\"3\">\n");
    for (int k = s.zl; k <= s.zu; ++k)
      for (int j = s.yl; j <= s.yu; ++j)
        for (int i = s.xl; i <= s.xu; ++i) {
          double r, u, v, ww; val(i, j, k, &r, &u, &v, &ww);
          std::fprintf(fh, "%s%s%s\n", es15_6(u).c_str(), es15_6(v).c_str(), es15_6(ww).c_str());
        }
    std::fprintf(fh, "</DataArray>\n</CellData>\n</Piece>\n</ImageData>\n</VTKFile>\n");
    std::fclose(fh);
    fh = std::fopen((d + "/Field.pvti").c_str(), "w");
    if (!fh) return -1;
    std::fprintf(fh, "<?xml version=\"1.0\"?>\n<VTKFile type=\"PImageData\">\n");
    std::fprintf(fh, "<PImageData WholeExtent=\"%4d%4d%4d%4d%4d%4d \" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n",
                 s.xmin - 1, s.xmax, s.ymin - 1, s.ymax, s.zmin - 1, s.zmax);
    std::fprintf(fh, "<PCellData Scalars=\"flag Rho\" Vectors =\"U\">\n");
    std::fprintf(fh, "<DataArray type=\"Int32\" Name=\"flag\" format=\"ascii\"/>\n");
    std::fprintf(fh, "<DataArray type=\"Float32\" Name=\"Rho\" format=\"ascii\"/>\n");
    std::fprintf(fh, "<DataArray type=\"Float32\" Name=\"U\" format=\"ascii\" NumberOfComponents=\"3\"/>\n");
    std::fprintf(fh, "</PCellData>\n");
    std::fprintf(fh, "<Piece Extent=\"%4d%4d%4d%4d%4d%4d\" Source=\"Field_000.vti\"/>\n", s.xl - 1, s.xu, s.yl - 1, s.yu, s.zl - 1, s.zu);
    std::fprintf(fh, "</PImageData>\n</VTKFile>\n");
    std::fclose(fh);
    return 0;
  }
  if (format == 2) {  // output.F90:166-189
    FILE *fh = std::fopen((d + "/Field_000.dat").c_str(), "w");
    if (!fh) return -1;
    std::fprintf(fh, "  TITLE=\" Field\"\n  VARIABLES=x,y,z,flag,Rho,Ux,Uy,Uz\n");
    std::fprintf(fh, " ZONE T=\"proc000\", I=%8d, J=%8d, K=%8d F=POINT\n", s.Nxsub, s.Nysub, s.Nzsub);
    for (int k = s.zl; k <= s.zu; ++k)
      for (int j = s.yl; j <= s.yu; ++j)
        for (int i = s.xl; i <= s.xu; ++i) {
          double r, u, v, ww;
          bool fl = val(i, j, k, &r, &u, &v, &ww);
          std::fprintf(fh, "%10d%10d%10d%10d%s%s%s%s\n", i, j, k, fl ? 0 : 1, es15_6(r).c_str(),
                       es15_6(u).c_str(), es15_6(v).c_str(), es15_6(ww).c_str());
        }
    std::fclose(fh);
    return 0;
  }
  if (format == 3) {  // output.F90:192-248
    FILE *fh = std::fopen((d + "/Field_000.vtk").c_str(), "w");
    if (!fh) return -1;
    std::fprintf(fh, "# vtk DataFile Version 2.0\nDVM MPI\nASCII\n\nDATASET STRUCTURED_POINTS\n");
    std::fprintf(fh, " DIMENSIONS%12d%12d%12d\n", s.Nxsub, s.Nysub, s.Nzsub);
    std::fprintf(fh, " ORIGIN%12d%12d%12d\n", s.xl, s.yl, s.zl);
    std::fprintf(fh, " SPACING%12d%12d%12d\n\n", 1, 1, 1);
    std::fprintf(fh, " POINT_DATA%12d\n\n", s.Nxsub * s.Nysub * s.Nzsub);
    std::fprintf(fh, "SCALARS Rho double\nLOOKUP_TABLE default\n");
    for (int k = s.zl; k <= s.zu; ++k)
      for (int j = s.yl; j <= s.yu; ++j)
        for (int i = s.xl; i <= s.xu; ++i) { double r, u, v, ww; val(i, j, k, &r, &u, &v, &ww); std::fprintf(fh, "%s\n", es15_6(r).c_str()); }
    std::fprintf(fh, "\nVECTORS Velocity double\n");
    for (int k = s.zl; k <= s.zu; ++k)
      for (int j = s.yl; j <= s.yu; ++j)
        for (int i = s.xl; i <= s.xu; ++i) {
          double r, u, v, ww; val(i, j, k, &r, &u, &v, &ww);
          std::fprintf(fh, "%s%s%s\n", es15_6(u).c_str(), es15_6(v).c_str(), es15_6(ww).c_str());
        }
    std::fclose(fh);
    return 0;
  }
  return -2;
}

}  // namespace

extern "C" {

void *oracle_create(const oracle_params *p, const uint8_t *raw, int64_t nbytes, int nthreads,
                    char *err, int errlen) {
  return oracle_create_rank(p, raw, nbytes, nthreads, 1, 0, err, errlen);
}

void *oracle_create_rank(const oracle_params *p, const uint8_t *raw, int64_t nbytes, int nthreads,
                         int32_t mpi_xdim, int32_t rank, char *err, int errlen) {
  auto *s = new Oracle();
  std::string e;
  if (mpi_xdim < 1 || rank < 0 || rank >= mpi_xdim) {
    if (err && errlen > 0) { std::strncpy(err, "bad rank / mpi_xdim", errlen - 1); err[errlen - 1] = 0; }
    delete s;
    return nullptr;
  }
  s->mpi_xdim = mpi_xdim;
  s->rank = rank;
  // parameters.F90:87-136
  s->Nx = p->Nx; s->Ny = p->Ny; s->Nz = p->Nz;
  s->wallExtOrder = p->wallExtOrder; s->fluidlayer = p->fluidlayer; s->Ref_L = p->Ref_L;
  s->Nc_fundamental = p->Nc_fundamental; s->halfRange = p->halfRange;
  s->block_repx = p->block_repx; s->block_repy = p->block_repy; s->block_repz = p->block_repz;
  s->maxStep = p->maxStep; s->chkConvergeStep = p->chkConvergeStep; s->saveStep = p->saveStep;
  s->eps = p->eps; s->saveLast = p->saveLast; s->saveFormat = p->saveFormat;
  s->Kn = p->Kn; s->pressDrop = p->pressDrop; s->accom = p->accom;
  s->nthreads = nthreads > 0 ? nthreads : omp_get_max_threads();
  s->Nx = s->Nx + 2 * s->fluidlayer;
  s->Nx_base = s->Nx; s->Ny_base = s->Ny; s->Nz_base = s->Nz;
  s->Nx = s->block_repx * s->Nx; s->Ny = s->block_repy * s->Ny; s->Nz = s->block_repz * s->Nz;
  s->xmin = 1; s->xmax = s->Nx; s->ymin = 1; s->ymax = s->Ny; s->zmin = 1; s->zmax = s->Nz;
  bool ok = setup_velocity_grid(*s, e);
  if (ok) {
    setup_process_grid(*s);
    // two ghost planes come from each neighbour rank: every rank owns at least two planes
    if (s->xu - s->xl + 1 < 2) { e = "fewer than two x planes per rank"; ok = false; }
  }
  if (ok) ok = setup_physical_grid(*s, raw, nbytes, e);
  if (ok) setup_flow(*s);
  if (!ok) {
    if (err && errlen > 0) { std::strncpy(err, e.c_str(), errlen - 1); err[errlen - 1] = 0; }
    delete s;
    return nullptr;
  }
  return s;
}

void oracle_destroy(void *h) { delete static_cast<Oracle *>(h); }

int oracle_iterate(void *h, int32_t nsteps) {
  auto *s = static_cast<Oracle *>(h);
  for (int n = 0; n < nsteps; ++n) { s->iStep++; iterate(*s); }
  return 0;
}

int oracle_chk_converge(void *h, const char *results_path, int verbose, double *mass, double *perm, double *err) {
  auto *s = static_cast<Oracle *>(h);
  chk_converge(*s, results_path, verbose);
  if (mass) *mass = s->mass;
  if (perm) *perm = s->permeability;
  if (err) *err = s->error;
  return 0;
}

// main.F90:95-128
int oracle_run(void *h, const char *results_path, int verbose, int32_t *steps_out, double *perm_out, double *seconds_out) {
  auto *s = static_cast<Oracle *>(h);
  s->error = 1.0;
  auto t0 = std::chrono::steady_clock::now();
  int step;
  for (step = 1; step <= s->maxStep; ++step) {
    s->iStep = step;
    iterate(*s);
    if (step % s->chkConvergeStep == 0) chk_converge(*s, results_path, verbose);
    if (s->error <= s->eps) {
      if (step < s->chkConvergeStep) chk_converge(*s, results_path, verbose);
      break;
    }
  }
  double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (verbose) {
    char wt[32];
    std::snprintf(wt, sizeof wt, "%11.3E", secs);
    std::printf("Walltime= %s, Steps= %6d, K= %s\n", wt, step, es15_6(s->permeability).c_str());
  }
  if (steps_out) *steps_out = step;
  if (perm_out) *perm_out = s->permeability;
  if (seconds_out) *seconds_out = secs;
  return 0;
}

void oracle_dims(void *h, int64_t *out) {
  auto *s = static_cast<Oracle *>(h);
  out[0] = s->Nx; out[1] = s->Ny; out[2] = s->Nz;
  out[3] = s->Nxtotal; out[4] = s->Nytotal; out[5] = s->Nztotal; out[6] = (int64_t)s->Ntotal;
  out[7] = s->Nc8; out[8] = s->nWall; out[9] = s->nCorner; out[10] = s->Nfluid; out[11] = s->iStep;
  for (int o = 0; o < 8; ++o) out[12 + o] = s->Nstencil[o];
}
void oracle_scalars(void *h, double *out) {
  auto *s = static_cast<Oracle *>(h);
  out[0] = s->ds; out[1] = s->mu; out[2] = s->DiffFlux; out[3] = s->mass; out[4] = s->error; out[5] = s->permeability;
}
void oracle_velocity(void *h, double *cx, double *cy, double *cz, double *w) {
  auto *s = static_cast<Oracle *>(h);
  std::copy(s->cx.begin(), s->cx.end(), cx); std::copy(s->cy.begin(), s->cy.end(), cy);
  std::copy(s->cz.begin(), s->cz.end(), cz); std::copy(s->w.begin(), s->w.end(), w);
}
void oracle_get_image(void *h, int32_t *out) { auto *s = static_cast<Oracle *>(h); std::copy(s->image.begin(), s->image.end(), out); }
void oracle_get_which_corner(void *h, int32_t *out) { auto *s = static_cast<Oracle *>(h); std::copy(s->which_corner.begin(), s->which_corner.end(), out); }
void oracle_get_vecwall(void *h, int32_t *out) { auto *s = static_cast<Oracle *>(h); std::copy(s->vecWall.begin(), s->vecWall.end(), out); }
void oracle_get_mapf(void *h, int32_t *out) { auto *s = static_cast<Oracle *>(h); std::copy(s->mapF.begin(), s->mapF.end(), out); }
void oracle_get_extcoef(void *h, double *out) { auto *s = static_cast<Oracle *>(h); std::copy(s->extCoef.begin(), s->extCoef.end(), out); }
void oracle_get_f(void *h, double *out) { auto *s = static_cast<Oracle *>(h); std::copy(s->f.begin(), s->f.end(), out); }
void oracle_set_f(void *h, const double *in) { auto *s = static_cast<Oracle *>(h); std::copy(in, in + s->f.size(), s->f.begin()); }
// f of n voxels (ghosted linear indices gidx) as out[n][8][Nc8]: rows of the reference layout
// f(Ntotal, Nc8, 8) for sampled comparisons of large cases.
void oracle_get_f_at(void *h, const int64_t *gidx, int32_t n, double *out) {
  auto *s = static_cast<Oracle *>(h);
  const size_t Ntot = s->f.size() / ((size_t)s->Nc8 * 8);
  for (int32_t q = 0; q < n; ++q)
    for (int o = 0; o < 8; ++o)
      for (int l = 0; l < s->Nc8; ++l)
        out[((size_t)q * 8 + o) * s->Nc8 + l] = s->f[(size_t)gidx[q] + (size_t)l * Ntot + (size_t)o * Ntot * s->Nc8];
}
void oracle_get_fw(void *h, double *out) { auto *s = static_cast<Oracle *>(h); std::copy(s->fw.begin(), s->fw.end(), out); }
void oracle_get_macro(void *h, double *rho, double *ux, double *uy, double *uz) {
  auto *s = static_cast<Oracle *>(h);
  std::copy(s->Rho.begin(), s->Rho.end(), rho); std::copy(s->Ux.begin(), s->Ux.end(), ux);
  std::copy(s->Uy.begin(), s->Uy.end(), uy); std::copy(s->Uz.begin(), s->Uz.end(), uz);
}
void oracle_get_dir(void *h, int octant, int32_t *out) {
  auto *s = static_cast<Oracle *>(h);
  std::copy(s->dir[octant - 1].begin(), s->dir[octant - 1].end(), out);
}
void oracle_get_coef(void *h, int octant, double *out) {
  auto *s = static_cast<Oracle *>(h);
  std::copy(s->coef[octant - 1].begin(), s->coef[octant - 1].end(), out);
}
int oracle_save(void *h, const char *dir, int format) { return save_fields(*static_cast<Oracle *>(h), dir, format); }

void oracle_slab(void *h, int32_t *out) {
  auto *s = static_cast<Oracle *>(h);
  out[0] = s->xl; out[1] = s->xu; out[2] = s->xlg; out[3] = s->mpi_xdim; out[4] = s->rank;
}
int64_t oracle_halo_size(void *h) { return (int64_t)static_cast<Oracle *>(h)->west_snd.size(); }
void oracle_halo_send(void *h, double *west, double *east) {
  auto *s = static_cast<Oracle *>(h);
  std::copy(s->west_snd.begin(), s->west_snd.end(), west);
  std::copy(s->east_snd.begin(), s->east_snd.end(), east);
}
void oracle_set_fw(void *h, const double *in) { auto *s = static_cast<Oracle *>(h); std::copy(in, in + s->fw.size(), s->fw.begin()); }
void oracle_set_macro(void *h, const double *rho, const double *ux, const double *uy, const double *uz) {
  auto *s = static_cast<Oracle *>(h);
  std::copy(rho, rho + s->Rho.size(), s->Rho.begin()); std::copy(ux, ux + s->Ux.size(), s->Ux.begin());
  std::copy(uy, uy + s->Uy.size(), s->Uy.begin()); std::copy(uz, uz + s->Uz.size(), s->Uz.begin());
}
void oracle_set_halo_send(void *h, const double *west, const double *east) {
  auto *s = static_cast<Oracle *>(h);
  std::copy(west, west + s->west_snd.size(), s->west_snd.begin());
  std::copy(east, east + s->east_snd.size(), s->east_snd.begin());
}
void oracle_halo_recv(void *h, const double *west, const double *east) {
  auto *s = static_cast<Oracle *>(h);
  std::copy(west, west + s->west_rcv.size(), s->west_rcv.begin());
  std::copy(east, east + s->east_rcv.size(), s->east_rcv.begin());
}

}  // extern "C"
