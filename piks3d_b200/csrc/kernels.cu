// Iteration kernels of the B200 solver for PIKS3D's source iteration (solver.F90:111-1940).
//
// FP64 arithmetic goes through __dmul_rn / __dadd_rn / __dsub_rn / __ddiv_rn in the
// reference's operation order (Fortran left-to-right evaluation), so no multiply-add is
// contracted and each value is rounded exactly as the CPU restatement rounds it.
#include <cuda_runtime.h>

#include "kernels.h"
#include "piks_internal.h"

namespace piks {

namespace {

__constant__ uint8_t c_face[128];        // fluid-side bits per label
__constant__ int8_t c_prog_of[128];      // label -> wall program index or -1
__constant__ WProg c_prog[26];
__constant__ int c_incoming[6][4];

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ size_t hidx(int node, int o, int Nc8, int l) {
  return ((size_t)node * 8 + o) * (size_t)Nc8 + l;
}
__device__ __forceinline__ int dsx(int o) { return (o == 0 || o == 3 || o == 4 || o == 7) ? 1 : -1; }
__device__ __forceinline__ int dsy(int o) { return (o == 0 || o == 1 || o == 4 || o == 5) ? 1 : -1; }
__device__ __forceinline__ int dsz(int o) { return o < 4 ? 1 : -1; }
// octant -> slot within a ghost plane (cx>0 octants 0,3,4,7 ; cx<0 octants 1,2,5,6)
__device__ __forceinline__ int plane_slot(int o) { return o >> 1; }

// Upwind value for a y/z neighbour of a fluid node in octant o's sweep.
//  fluid, inside this CTA's tile  -> the value computed this sweep (shared-memory ring)
//  fluid, outside the tile        -> global h (earlier tile of this sweep, or an inflow
//                                    boundary node whose value the BCs set)
//  solid node read by the solver  -> the slot its reader position sees (static switch
//                                    resolution of solver.F90:184-204 etc.)
//  anything else                  -> 0 (ghost layers; only ever multiplied by 0)
__device__ __forceinline__ double upwind_value(const DevState &a, int m, int o, int role, int l,
                                               bool in_tile, const double *ring_entry) {
  if (m >= 0 && m < a.NF) return in_tile ? *ring_entry : a.h[hidx(m, o, a.Nc8, l)];
  if (m >= a.NF) {
    const int b = m - a.NF;
    const int src = (a.roles[(size_t)b * 8 + o] >> (4 * role)) & 15;
    if (src < 8) return a.h[hidx(m, src, a.Nc8, l)];
    return a.fw[hidx(a.bcorner[b], o, a.Nc8, l)];
  }
  return 0.0;
}

// ---------------------------------------------------------------------------------------
// Octant sweeps (solver.F90:176-526). One CTA = one tile of TV x TW pencils of one octant
// and one 32-velocity chunk; warp (pv, pw) owns pencil (v, w) of the octant's local frame
// (u, v, w increase along the sweep) and walks u = 1 .. Nx-1 keeping the two x-upwind
// values in registers. Pencils advance on a diagonal schedule, pencil (pv, pw) handling u
// at step t = u - 1 + pv + pw, so the y/z-upwind values of a node were produced one or two
// steps earlier and are read from a 3-deep shared-memory ring. Tiles of one launch lie on
// one anti-diagonal of the tile grid; their y/z-upwind tiles finished in earlier launches.
template <int TV, int TW>
__global__ void __launch_bounds__(TV * TW * 32)
k_sweep(const DevState a, int diag, int ntw) {
  __shared__ double ring[3][TV * TW][32];
  const int per_tile = 8 * a.nchunk;
  const int tile = blockIdx.x / per_tile;
  const int rem = blockIdx.x - tile * per_tile;
  const int o = rem / a.nchunk;
  const int chunk = rem - o * a.nchunk;
  const int b = max(0, diag - (ntw - 1)) + tile;
  const int c = diag - b;
  const int sx = dsx(o), sy = dsy(o), sz = dsz(o);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pv = wid % TV, pw = wid / TV;
  const int v = 1 + b * TV + pv, w = 1 + c * TW + pw;
  const bool active = v <= a.Ny - 1 && w <= a.Nz - 1;
  const int Nc8 = a.Nc8;
  const int l = chunk * 32 + lane;
  const bool lv = l < Nc8;
  double cxl = 0.0, cyl = 0.0, czl = 0.0, wl = 0.0;
  if (lv) { cxl = a.cx[l]; cyl = a.cy[l]; czl = a.cz[l]; wl = a.w[l]; }
  // signed upwind coefficients (physicalGrid.F90:1254-1622): second / first order
  const double X0 = sx > 0 ? a.c15 : -a.c15, X1 = sx > 0 ? a.c20 : -a.c20, X2 = sx > 0 ? a.c05 : -a.c05;
  const double Y0 = sy > 0 ? a.c15 : -a.c15, Y1 = sy > 0 ? a.c20 : -a.c20, Y2 = sy > 0 ? a.c05 : -a.c05;
  const double Z0 = sz > 0 ? a.c15 : -a.c15, Z1 = sz > 0 ? a.c20 : -a.c20, Z2 = sz > 0 ? a.c05 : -a.c05;
  const double XF = sx > 0 ? a.c10 : -a.c10, YF = sy > 0 ? a.c10 : -a.c10, ZF = sz > 0 ? a.c10 : -a.c10;
  const uint8_t xbit = sx > 0 ? FACE_E : FACE_W;
  const uint8_t ybit = sy > 0 ? FACE_N : FACE_S;
  const uint8_t zbit = sz > 0 ? FACE_F : FACE_B;
  const int j = sy > 0 ? v + 1 : a.Ny - v;
  const int k = sz > 0 ? w + 1 : a.Nz - w;
  const int i0 = sx > 0 ? 1 : a.Nx;
  const long gbase = (long)(i0 + 1) + (long)(j + 1) * a.GX + (long)(k + 1) * a.GXY;
  const long SY = (long)sy * a.GX, SZ = (long)sz * a.GXY;
  const double half_mu = dmul(0.5, a.mu);

  double xm1 = 0.0, xm2 = 0.0;  // x-upwind values at u-1, u-2 (u-2 = ghost at u = 1)
  int labprev = L_GHOST;
  if (active) {
    const int m0 = a.nodemap[gbase];
    labprev = a.label[gbase];
    if (m0 >= 0 && lv) xm1 = a.h[hidx(m0, o, Nc8, l)];
  }
  const int nsteps = (a.Nx - 1) + (TV - 1) + (TW - 1);
  for (int t = 0; t < nsteps; ++t) {
    const int u = t - pv - pw + 1;
    if (active && u >= 1 && u <= a.Nx - 1) {
      const long g = gbase + (long)sx * u;
      const int m = a.nodemap[g];
      const int lab = a.label[g];
      double out = 0.0;
      if (m >= 0 && m < a.NF) {
        const bool fx = (u == 1) || (c_face[labprev] & xbit);
        const long gy1 = g - SY, gz1 = g - SZ;
        const int my1 = a.nodemap[gy1], my2 = a.nodemap[gy1 - SY];
        const int mz1 = a.nodemap[gz1], mz2 = a.nodemap[gz1 - SZ];
        const bool fy = (v == 1) || (c_face[a.label[gy1]] & ybit);
        const bool fz = (w == 1) || (c_face[a.label[gz1]] & zbit);
        if (lv) {
          const int p = wid;
          const double y1 = upwind_value(a, my1, o, 0, l, pv >= 1, &ring[(t + 2) % 3][p - (pv >= 1 ? 1 : 0)][lane]);
          const double y2 = upwind_value(a, my2, o, 1, l, pv >= 2, &ring[(t + 1) % 3][p - (pv >= 2 ? 2 : 0)][lane]);
          const double z1 = upwind_value(a, mz1, o, 2, l, pw >= 1, &ring[(t + 2) % 3][p - (pw >= 1 ? TV : 0)][lane]);
          const double z2 = upwind_value(a, mz2, o, 3, l, pw >= 2, &ring[(t + 1) % 3][p - (pw >= 2 ? 2 * TV : 0)][lane]);
          const double fold = a.h[hidx(m, o, Nc8, l)];
          // fEq = w*(Rho + (+-cx*Ux +- cy*Uy +- cz*Uz))   (solver.F90:206)
          double ex = dmul(cxl, a.ux[m]); if (sx < 0) ex = -ex;
          double ey = dmul(cyl, a.uy[m]); if (sy < 0) ey = -ey;
          double ez = dmul(czl, a.uz[m]); if (sz < 0) ez = -ez;
          const double feq = dmul(wl, dadd(a.rho[m], dadd(dadd(ex, ey), ez)));
          // (solver.F90:207-214) a term of a negative-velocity axis is subtracted with its
          // negative coefficient, exactly as the reference writes it
          double num = dmul(a.mu, dsub(feq, dmul(0.5, fold)));
          double tt;
          tt = dmul(dmul(cxl, fx ? XF : X1), xm1);   num = sx > 0 ? dadd(num, tt) : dsub(num, tt);
          tt = dmul(dmul(cxl, fx ? 0.0 : X2), xm2);  num = sx > 0 ? dadd(num, tt) : dsub(num, tt);
          tt = dmul(dmul(cyl, fy ? YF : Y1), y1);    num = sy > 0 ? dadd(num, tt) : dsub(num, tt);
          tt = dmul(dmul(cyl, fy ? 0.0 : Y2), y2);   num = sy > 0 ? dadd(num, tt) : dsub(num, tt);
          tt = dmul(dmul(czl, fz ? ZF : Z1), z1);    num = sz > 0 ? dadd(num, tt) : dsub(num, tt);
          tt = dmul(dmul(czl, fz ? 0.0 : Z2), z2);   num = sz > 0 ? dadd(num, tt) : dsub(num, tt);
          double den = half_mu;
          tt = dmul(cxl, fx ? XF : X0); den = sx > 0 ? dadd(den, tt) : dsub(den, tt);
          tt = dmul(cyl, fy ? YF : Y0); den = sy > 0 ? dadd(den, tt) : dsub(den, tt);
          tt = dmul(czl, fz ? ZF : Z0); den = sz > 0 ? dadd(den, tt) : dsub(den, tt);
          out = __ddiv_rn(num, den);
          a.h[hidx(m, o, Nc8, l)] = out;
          ring[t % 3][p][lane] = out;
        }
      } else if (m >= 0) {
        // solid node read by the solver: x readers always see its slot o unswitched
        if (lv) out = a.h[hidx(m, o, Nc8, l)];
      }
      xm2 = xm1;
      xm1 = out;
      labprev = lab;
    }
    __syncthreads();
  }
}

// Post-sweep content of switched wall slots: slot o of a wall ends the reference's sweep
// holding the last value switched into it (z-upwind reader, else y-upwind reader).
__global__ void k_commit(const DevState a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t total = (size_t)a.ncommit * a.Nc8;
  if (idx >= total) return;
  const int e = (int)(idx / a.Nc8), l = (int)(idx % a.Nc8);
  const int node = a.commit[3 * e], o = a.commit[3 * e + 1], src = a.commit[3 * e + 2];
  const double v = src < 8 ? a.h[hidx(node, src, a.Nc8, l)]
                           : a.fw[hidx(a.bcorner[node - a.NF], o, a.Nc8, l)];
  a.h[hidx(node, o, a.Nc8, l)] = v;
}

// Periodic x halo (solver.F90:535-560, one rank): the planes x = Nx (octants with cx > 0)
// and x = 1 (cx < 0) as they stand after the sweep become the ghost planes x = 0 and
// x = Nx+1 that the boundary conditions of the NEXT iteration read.
__global__ void k_capture(const DevState a, int buf) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t rows = (size_t)a.Ny * a.Nz;
  const size_t total = rows * 4 * a.Nc8;
  if (idx >= total) return;
  const int l = (int)(idx % a.Nc8);
  const int q = (int)((idx / a.Nc8) % 4);
  const size_t r = idx / ((size_t)a.Nc8 * 4);
  const int oW = (q == 0) ? 0 : (q == 1) ? 3 : (q == 2) ? 4 : 7;   // cx > 0
  const int oE = (q == 0) ? 1 : (q == 1) ? 2 : (q == 2) ? 5 : 6;   // cx < 0
  const int nW = a.plane_xN[r], nE = a.plane_x1[r];
  a.ghostW[buf][idx] = nW >= 0 ? a.h[hidx(nW, oW, a.Nc8, l)] : 0.0;
  a.ghostE[buf][idx] = nE >= 0 ? a.h[hidx(nE, oE, a.Nc8, l)] : 0.0;
}

// Value at a wall's +2d extrapolation point: a node, zero (y/z ghost layers), or a ghost
// plane x = 0 / x = Nx+1 (code -(2+2r) / -(3+2r) for plane row r).
__device__ __forceinline__ double ext_far(const DevState &a, int code, int o, int l, int gbuf) {
  if (code >= 0) return a.h[hidx(code, o, a.Nc8, l)];
  if (code == -1) return 0.0;
  const int c = -code - 2;
  const size_t r = (size_t)(c >> 1);
  const double *plane = (c & 1) ? a.ghostE[gbuf] : a.ghostW[gbuf];
  return plane[(r * 4 + plane_slot(o)) * a.Nc8 + l];
}

// Diffuse wall (solver.F90:761-1826): one warp per wall, lanes over velocities. The
// wall program (wall_table.inc) lists, per fluid-side face, the 4 extrapolated incoming
// octants and then the re-emission writes in the reference's statement order. The
// density sums run serially over l in lane order to keep the reference's rounding.
__global__ void k_walls(const DevState a, int begin, int end, int gbuf) {
  const int widx = begin + (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (widx >= end) return;  // whole warp
  const int lane = threadIdx.x & 31;
  const int q = a.wall_order[widx];
  const int node = a.wall_node[q];
  const int corner = a.wall_corner[q];
  const WProg &P = c_prog[c_prog_of[a.wall_label[q]]];
  const double e1 = a.wall_e[2 * q], e2 = a.wall_e[2 * q + 1];
  const int Nc8 = a.Nc8;
  const int *nb = a.wall_nb + 6 * q;
  double rho[3] = {0.0, 0.0, 0.0};
  for (int l0 = 0; l0 < Nc8; l0 += 32) {
    const int l = l0 + lane;
    const bool lv = l < Nc8;
    double tface[3] = {0.0, 0.0, 0.0};
    for (int fi = 0; fi < P.nface; ++fi) {
      const int dir = P.face[fi].dir, st = P.face[fi].store;
      double vals[4];
      for (int mm = 0; mm < 4; ++mm) {
        const int oo = c_incoming[dir][mm] - 1;
        double v = 0.0;
        if (lv) {
          v = dadd(dmul(e1, a.h[hidx(nb[2 * fi], oo, Nc8, l)]), dmul(e2, ext_far(a, nb[2 * fi + 1], oo, l, gbuf)));
          if (st == ST_F) a.h[hidx(node, oo, Nc8, l)] = v;
          else if (st == ST_W) a.fw[hidx(corner, oo, Nc8, l)] = v;
        }
        vals[mm] = v;
      }
      if (lv) {
        const double ca = dir < 2 ? a.cx[l] : dir < 4 ? a.cy[l] : a.cz[l];
        tface[fi] = dmul(ca, dadd(dadd(dadd(vals[0], vals[1]), vals[2]), vals[3]));
      }
    }
    const int nl = min(32, Nc8 - l0);
    for (int s = 0; s < nl; ++s)
      for (int fi = 0; fi < 3; ++fi) {
        const double tv = __shfl_sync(0xffffffffu, tface[fi], s);
        if (fi < P.nface) rho[fi] = dadd(rho[fi], tv);
      }
  }
  for (int fi = 0; fi < P.nface; ++fi) rho[fi] = __ddiv_rn(rho[fi], a.DiffFlux);
  const double one_m = dsub(1.0, a.accom);
  int zface = -1;
  for (int fi = 0; fi < P.nface; ++fi) if (P.face[fi].store == ST_Z) zface = fi;
  for (int l0 = 0; l0 < Nc8; l0 += 32) {
    const int l = l0 + lane;
    if (l >= Nc8) continue;
    const double aw = dmul(a.accom, a.w[l]);
    for (int r = 0; r < P.nwr; ++r) {
      const WWrite &W = P.wr[r];
      const int so = W.src_o - 1, dso = W.dst_o - 1;
      double src;
      if (W.src_store == ST_F) src = a.h[hidx(node, so, Nc8, l)];
      else if (W.src_store == ST_W) src = a.fw[hidx(corner, so, Nc8, l)];
      else src = dadd(dmul(e1, a.h[hidx(nb[2 * zface], so, Nc8, l)]), dmul(e2, ext_far(a, nb[2 * zface + 1], so, l, gbuf)));
      const double v = dadd(dmul(aw, rho[W.face]), dmul(one_m, src));
      if (W.dst_store == ST_F) a.h[hidx(node, dso, Nc8, l)] = v;
      else a.fw[hidx(corner, dso, Nc8, l)] = v;
    }
  }
}

// Inlet x = 1 and outlet x = Nx with the pressure jump (solver.F90:1832-1862), reading the
// ghost planes captured in the previous iteration.
__global__ void k_inlet_outlet(const DevState a, int gbuf) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t total = (size_t)a.Ny * a.Nz * 4 * a.Nc8;
  if (idx >= total) return;
  const int l = (int)(idx % a.Nc8);
  const int q = (int)((idx / a.Nc8) % 4);
  const size_t r = idx / ((size_t)a.Nc8 * 4);
  const double wdp = dmul(a.w[l], a.pressDrop);
  const int n1 = a.plane_x1[r], nN = a.plane_xN[r];
  if (n1 >= 0) {
    const int o = (q == 0) ? 0 : (q == 1) ? 3 : (q == 2) ? 4 : 7;
    a.h[hidx(n1, o, a.Nc8, l)] = dadd(a.ghostW[gbuf][idx], wdp);
  }
  if (nN >= 0) {
    const int o = (q == 0) ? 1 : (q == 1) ? 2 : (q == 2) ? 5 : 6;
    a.h[hidx(nN, o, a.Nc8, l)] = dsub(a.ghostE[gbuf][idx], wdp);
  }
}

// Specular symmetry planes y = 1, y = Ny, z = 1, z = Nz in the reference's order
// (solver.F90:1867-1918).
__global__ void k_symmetry(const DevState a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t total = (size_t)a.nsym * a.Nc8;
  if (idx >= total) return;
  const int s = (int)(idx / a.Nc8), l = (int)(idx % a.Nc8);
  const int n = a.sym_node[s];
  const uint8_t f = a.sym_flag[s];
  double *hp = a.h + (size_t)n * 8 * a.Nc8 + l;
  const size_t S = a.Nc8;
  if (f & 1) { hp[1 * S] = hp[2 * S]; hp[0 * S] = hp[3 * S]; hp[5 * S] = hp[6 * S]; hp[4 * S] = hp[7 * S]; }
  if (f & 2) { hp[2 * S] = hp[1 * S]; hp[3 * S] = hp[0 * S]; hp[6 * S] = hp[5 * S]; hp[7 * S] = hp[4 * S]; }
  if (f & 4) { hp[0 * S] = hp[4 * S]; hp[1 * S] = hp[5 * S]; hp[2 * S] = hp[6 * S]; hp[3 * S] = hp[7 * S]; }
  if (f & 8) { hp[4 * S] = hp[0 * S]; hp[5 * S] = hp[1 * S]; hp[6 * S] = hp[2 * S]; hp[7 * S] = hp[3 * S]; }
}

// Moments Rho, Ux, Uy, Uz (solver.F90:1923-1938): one warp per fluid node stages 32
// velocities x 8 octants in shared memory; lanes 0..3 run the four sums serially over
// (l, octant) in the reference's order.
constexpr int kMomWarps = 8;
__global__ void __launch_bounds__(kMomWarps * 32) k_moments(const DevState a) {
  __shared__ double sm[kMomWarps][8][33];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int node = blockIdx.x * kMomWarps + wid;
  if (node >= a.NF) return;  // whole warp
  const int Nc8 = a.Nc8;
  double acc = 0.0;
  for (int l0 = 0; l0 < Nc8; l0 += 32) {
    const int l = l0 + lane;
    for (int o = 0; o < 8; ++o) sm[wid][o][lane] = l < Nc8 ? a.h[hidx(node, o, Nc8, l)] : 0.0;
    __syncwarp();
    if (lane < 4) {
      const int nl = min(32, Nc8 - l0);
      for (int s = 0; s < nl; ++s) {
        const double f1 = sm[wid][0][s], f2 = sm[wid][1][s], f3 = sm[wid][2][s], f4 = sm[wid][3][s];
        const double f5 = sm[wid][4][s], f6 = sm[wid][5][s], f7 = sm[wid][6][s], f8 = sm[wid][7][s];
        if (lane == 0) {
          acc = dadd(dadd(dadd(dadd(dadd(dadd(dadd(dadd(acc, f1), f2), f3), f4), f5), f6), f7), f8);
        } else if (lane == 1) {
          const double d = dadd(dsub(dsub(dadd(dadd(dsub(dsub(f1, f2), f3), f4), f5), f6), f7), f8);
          acc = dadd(acc, dmul(a.cx[l0 + s], d));
        } else if (lane == 2) {
          const double d = dsub(dsub(dadd(dadd(dsub(dsub(dadd(f1, f2), f3), f4), f5), f6), f7), f8);
          acc = dadd(acc, dmul(a.cy[l0 + s], d));
        } else {
          const double d = dsub(dsub(dsub(dsub(dadd(dadd(dadd(f1, f2), f3), f4), f5), f6), f7), f8);
          acc = dadd(acc, dmul(a.cz[l0 + s], d));
        }
      }
    }
    __syncwarp();
  }
  if (lane == 0) a.rho[node] = acc;
  else if (lane == 1) a.ux[node] = acc;
  else if (lane == 2) a.uy[node] = acc;
  else if (lane == 3) a.uz[node] = acc;
}

// Mass flux through x = 2 (output.F90:90-142) in the reference's summation order; one
// thread, the plane has only Ny*Nz terms.
__global__ void k_flux(const DevState a, double ds, double sqrt_half, double inv_refl2) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double part[9];
  for (int gi = 0; gi < 9; ++gi) {
    double s = 0.0;
    for (int e = a.flux_groups[gi]; e < a.flux_groups[gi + 1]; ++e) {
      const int n = a.flux_list[e];
      const double u = n >= 0 ? a.ux[n] : 0.0;
      double term = dmul(dmul(u, ds), ds);
      if (gi >= 1 && gi <= 4) term = dmul(term, 0.5);
      else if (gi >= 5) term = dmul(term, 0.25);
      s = gi <= 4 ? dadd(s, term) : term;
    }
    part[gi] = s;
  }
  double m = part[0];
  for (int gi = 1; gi < 9; ++gi) m = dadd(m, part[gi]);
  m = __ddiv_rn(__ddiv_rn(dmul(m, sqrt_half), a.pressDrop), inv_refl2);
  a.flux_out[0] = m;
}

inline unsigned blocks_for(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

void upload_tables() {
  uint8_t face[128];
  int8_t prog_of[128];
  WProg progs[26];
  int n = 0;
  for (int lab = 0; lab < 128; ++lab) {
    face[lab] = face_mask(lab);
    prog_of[lab] = -1;
    const WProg *p = wall_program(lab);
    if (p) { progs[n] = *p; prog_of[lab] = (int8_t)n; ++n; }
  }
  cudaMemcpyToSymbol(c_face, face, sizeof face);
  cudaMemcpyToSymbol(c_prog_of, prog_of, sizeof prog_of);
  cudaMemcpyToSymbol(c_prog, progs, sizeof progs);
  cudaMemcpyToSymbol(c_incoming, kIncoming, sizeof(int) * 24);
}

int sweep_num_diagonals(const DevState &s) {
  const int ntv = (s.Ny - 1 + kTV - 1) / kTV, ntw = (s.Nz - 1 + kTW - 1) / kTW;
  return ntv + ntw - 1;
}

void launch_sweep_diagonal(const DevState &s, int diag, cudaStream_t st) {
  const int ntv = (s.Ny - 1 + kTV - 1) / kTV, ntw = (s.Nz - 1 + kTW - 1) / kTW;
  const int blo = diag - (ntw - 1) > 0 ? diag - (ntw - 1) : 0;
  const int bhi = diag < ntv - 1 ? diag : ntv - 1;
  const int ntiles = bhi - blo + 1;
  if (ntiles <= 0) return;
  k_sweep<kTV, kTW><<<ntiles * 8 * s.nchunk, kTV * kTW * 32, 0, st>>>(s, diag, ntw);
}

void launch_commit(const DevState &s, cudaStream_t st) {
  if (s.ncommit == 0) return;
  const size_t n = (size_t)s.ncommit * s.Nc8;
  k_commit<<<blocks_for(n, 256), 256, 0, st>>>(s);
}

void launch_capture(const DevState &s, int buf, cudaStream_t st) {
  const size_t n = (size_t)s.Ny * s.Nz * 4 * s.Nc8;
  k_capture<<<blocks_for(n, 256), 256, 0, st>>>(s, buf);
}

void launch_inlet_outlet(const DevState &s, int buf, cudaStream_t st) {
  const size_t n = (size_t)s.Ny * s.Nz * 4 * s.Nc8;
  k_inlet_outlet<<<blocks_for(n, 256), 256, 0, st>>>(s, buf);
}

void launch_symmetry(const DevState &s, cudaStream_t st) {
  if (s.nsym == 0) return;
  const size_t n = (size_t)s.nsym * s.Nc8;
  k_symmetry<<<blocks_for(n, 256), 256, 0, st>>>(s);
}

void launch_moments(const DevState &s, cudaStream_t st) {
  if (s.NF == 0) return;
  k_moments<<<blocks_for((size_t)s.NF, kMomWarps), kMomWarps * 32, 0, st>>>(s);
}

void launch_walls(const DevState &s, int begin, int end, int gbuf, cudaStream_t st) {
  if (end <= begin) return;
  const size_t threads = (size_t)(end - begin) * 32;
  k_walls<<<blocks_for(threads, 256), 256, 0, st>>>(s, begin, end, gbuf);
}

void launch_flux(const DevState &s, double ds, double sqrt_half, double inv_refl2, cudaStream_t st) {
  k_flux<<<1, 32, 0, st>>>(s, ds, sqrt_half, inv_refl2);
}

}  // namespace piks
