// Iteration kernels of the B200 solver for PIKS3D's source iteration (solver.F90:111-1940).
//
// FP64 arithmetic goes through __dmul_rn / __dadd_rn / __dsub_rn / __ddiv_rn in the
// reference's operation order (Fortran left-to-right evaluation), so no multiply-add is
// contracted and each value is rounded exactly as the CPU restatement rounds it.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <set>
#include <tuple>

#include "kernels.h"
#include "piks_internal.h"

namespace piks {

namespace {

__constant__ uint8_t c_face[128];        // fluid-side bits per label
__constant__ int8_t c_prog_of[128];      // label -> wall program index or -1
__constant__ WProg c_prog[26];
__constant__ WPlan c_plan[26];
bool g_plan_ok = false;                  // every program resolved (make_wall_plan)
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
// Asynchronous global->shared copies (cp.async, 8 bytes through L1) with commit groups.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
// 16 bytes through L2 only (the moments read each value once).
__device__ __forceinline__ void cp_async16_cg(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
// octant -> slot within a ghost plane (cx>0 octants 0,3,4,7 ; cx<0 octants 1,2,5,6)
__device__ __forceinline__ int plane_slot(int o) { return o >> 1; }

// ---------------------------------------------------------------------------------------
// Octant sweeps (solver.F90:176-526).
//
// In octant o's frame (u, v, w increase along the sweep) a node depends on the nodes one
// and two cells upwind along each axis, so all swept nodes with the same u+v+w are
// independent, for all eight octants at once. The host lists one task per (swept fluid
// node, octant) ordered by that hyperplane index; one launch runs one hyperplane. A task
// is a warp-sized group of lanes over the octant's velocities; every value it reads was
// written by an earlier launch (or is a boundary value the sweep never writes), so the
// loads of a task are independent and the warp issues them all before any arithmetic.
//
// Arithmetic (solver.F90:206-214) in the reference's order. In the octant's frame every
// upwind term is added with the coefficient of the positive-velocity octant: for a
// negative velocity axis the reference subtracts (c * -C) * f, which is bit-identical to
// adding (c * C) * f, and fEq's +-c*U equals the product with the signed component. The
// denominators depend only on the velocity and the first/second-order class, so they
// are tabulated with the same operations; the division num/den is evaluated from the
// correctly rounded reciprocal y = RN(1/den) by Markstein's correction
// q = RN(q0 + RN-exact(num - den*q0) * y), q0 = RN(num*y), which returns RN(num/den)
// (Markstein, IBM J. Res. Dev. 34 (1990); piks_selftest_division checks it).
__device__ __forceinline__ double markstein_div(double num, double den, double y) {
  const double q0 = __dmul_rn(num, y);
  const double r = __fma_rn(-q0, den, num);
  return __fma_rn(r, y, q0);
}

constexpr int kFwBit = 1 << 30;

template <int VPL>
__device__ __forceinline__ void load_row(const DevState &a, int code, size_t l0, double (&v)[VPL]) {
  const double *base = (code & kFwBit) ? a.fw : a.h;
  const double *p = base + (size_t)(code & ~kFwBit) * (size_t)a.Nc8 + l0;
  if (VPL == 2) {
    const double2 t = __ldcg(reinterpret_cast<const double2 *>(p));
    v[0] = t.x; v[VPL - 1] = t.y;
  } else {
    v[0] = __ldcg(p);
  }
}

// LPT lanes per task (32, or 8 when an octant has 8 velocities), VPL velocities per lane.
template <int LPT, int VPL>
__global__ void __launch_bounds__(256)
k_sweep(const DevState a, long t0, long ntask) {
  constexpr int TPW = 32 / LPT;  // tasks per warp
  const long gl = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long slot = gl / LPT;                 // (task, chunk) slot of this lane group
  const int sub = (int)(gl % LPT);
  const long ti = slot / a.nchunk;
  const int chunk = (int)(slot - ti * a.nchunk);
  if (ti >= ntask) return;
  const int Nc8 = a.Nc8;
  const int lfirst = chunk * LPT * VPL + sub * VPL;
  if (lfirst >= Nc8) return;
  const int4 *rec = reinterpret_cast<const int4 *>(a.tasks + (size_t)(t0 + ti) * 8);
  const int4 r0 = __ldg(rec), r1 = __ldg(rec + 1);
  const int m = r0.x, fl = r0.y;
  const int o = fl & 7;
  const bool fx = fl & 8, fy = fl & 16, fz = fl & 32;
  const size_t l0 = (size_t)lfirst;
  // loads first: own value, moments, upwind values
  double fold[VPL], x1[VPL], x2[VPL], y1[VPL], y2[VPL], z1[VPL], z2[VPL];
  load_row<VPL>(a, m * 8 + o, l0, fold);
  load_row<VPL>(a, r0.z, l0, x1);
  load_row<VPL>(a, r1.x, l0, y1);
  load_row<VPL>(a, r1.z, l0, z1);
  if (!fx) load_row<VPL>(a, r0.w, l0, x2);
  if (!fy) load_row<VPL>(a, r1.y, l0, y2);
  if (!fz) load_row<VPL>(a, r1.w, l0, z2);
  const double2 m01 = __ldg(reinterpret_cast<const double2 *>(a.mom) + 2 * (size_t)m);
  const double2 m23 = __ldg(reinterpret_cast<const double2 *>(a.mom) + 2 * (size_t)m + 1);
  const double rho = m01.x, ux = m01.y, uy = m23.x, uz = m23.y;
  const int cls = (fx ? 1 : 0) | (fy ? 2 : 0) | (fz ? 4 : 0);
  const bool nx_ = dsx(o) < 0, ny_ = dsy(o) < 0, nz_ = dsz(o) < 0;
  // per-velocity constants: one 16-byte load gives both velocities of a lane (VPL = 2)
  double K[kVtab][VPL];
  if (VPL == 2) {
    const double2 *vt = a.vtab2 + (size_t)(lfirst >> 1) * kVtab;
#pragma unroll
    for (int k = 0; k < 13; ++k) { const double2 t = __ldg(vt + k); K[k][0] = t.x; K[k][VPL - 1] = t.y; }
    const double2 dn = __ldg(vt + 13 + cls), rc = __ldg(vt + 21 + cls);
    K[13][0] = dn.x; K[13][VPL - 1] = dn.y; K[21][0] = rc.x; K[21][VPL - 1] = rc.y;
  } else {
    const double *vt = a.vtab + (size_t)lfirst * kVtab;
#pragma unroll
    for (int k = 0; k < 13; ++k) K[k][0] = __ldg(vt + k);
    K[13][0] = __ldg(vt + 13 + cls); K[21][0] = __ldg(vt + 21 + cls);
  }
  double out[VPL];
#pragma unroll
  for (int q = 0; q < VPL; ++q) {
    const double cx = K[0][q], cy = K[1][q], cz = K[2][q], wl = K[3][q];
    const double ex = dmul(nx_ ? -cx : cx, ux), ey = dmul(ny_ ? -cy : cy, uy), ez = dmul(nz_ ? -cz : cz, uz);
    const double feq = dmul(wl, dadd(rho, dadd(dadd(ex, ey), ez)));
    double num = dmul(a.mu, dsub(feq, dmul(0.5, fold[q])));
    num = dadd(num, dmul(fx ? K[5][q] : K[4][q], x1[q]));
    if (!fx) num = dadd(num, dmul(K[6][q], x2[q]));
    num = dadd(num, dmul(fy ? K[8][q] : K[7][q], y1[q]));
    if (!fy) num = dadd(num, dmul(K[9][q], y2[q]));
    num = dadd(num, dmul(fz ? K[11][q] : K[10][q], z1[q]));
    if (!fz) num = dadd(num, dmul(K[12][q], z2[q]));
    out[q] = markstein_div(num, K[13][q], K[21][q]);
  }
  double *hp = a.h + ((size_t)m * 8 + o) * (size_t)Nc8 + l0;
  if (VPL == 2) *reinterpret_cast<double2 *>(hp) = make_double2(out[0], out[VPL - 1]);
  else hp[0] = out[0];
  (void)TPW;
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

// The same commits as 16-byte copies, for rows (node, octant) whose byte size is a multiple
// of 16; `h` / `fw` are the FP64 or the FP32 arrays, `pieces` the 16-byte pieces per row.
__global__ void k_commit16(const int32_t *commit, const int32_t *bcorner, int NF, int4 *h, const int4 *fw,
                           int ncommit, int pieces) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)ncommit * pieces) return;
  const int e = (int)(idx / pieces), pc = (int)(idx % pieces);
  const int node = commit[3 * e], o = commit[3 * e + 1], src = commit[3 * e + 2];
  const int4 v = src < 8 ? h[((size_t)node * 8 + src) * pieces + pc]
                         : fw[((size_t)bcorner[node - NF] * 8 + o) * pieces + pc];
  h[((size_t)node * 8 + o) * pieces + pc] = v;
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

// Diffuse wall (solver.F90:761-1826): one warp per wall, lanes over velocities (VPL per
// lane). The wall program (wall_table.inc) lists, per fluid-side face, the 4 extrapolated
// incoming octants and then the re-emission writes in the reference's statement order.
// All neighbour values are loaded before any arithmetic; the density sums run serially
// over l in the reference's order by passing the per-velocity terms through the warp.
template <int VPL>
__device__ __forceinline__ void ld_vpl(const double *p, double (&v)[VPL]) {
  if (VPL == 2) { const double2 t = __ldcg(reinterpret_cast<const double2 *>(p)); v[0] = t.x; v[VPL - 1] = t.y; }
  else v[0] = __ldcg(p);
}
template <int VPL>
__device__ __forceinline__ void ld_vpl_sm(const double *p, double (&v)[VPL]) {
  if (VPL == 2) { const double2 t = *reinterpret_cast<const double2 *>(p); v[0] = t.x; v[VPL - 1] = t.y; }
  else v[0] = p[0];
}
template <int VPL>
__device__ __forceinline__ void st_vpl(double *p, const double (&v)[VPL]) {
  if (VPL == 2) *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[VPL - 1]);
  else p[0] = v[0];
}

// At most 51 registers (five 256-thread blocks per SM): a wall's time is mostly memory
// round trips, so more resident walls pay (measured 1.38 -> 1.04 ms on a 128^3 pack).
template <int VPL>
__global__ void __launch_bounds__(256, 5) k_walls(const DevState a, int begin, int end, int gbuf) {
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
  const int nface = P.nface;
  const int chunkw = 32 * VPL;
  double rho0 = 0.0, rho1 = 0.0, rho2 = 0.0;
  for (int fi = 0; fi < nface; ++fi) {
    const int dir = P.face[fi].dir, st = P.face[fi].store;
    const int n1 = nb[2 * fi], code = nb[2 * fi + 1];
    const double *plane = nullptr;
    size_t prow = 0;
    if (code < -1) {
      const int cc = -code - 2;
      plane = (cc & 1) ? a.ghostE[gbuf] : a.ghostW[gbuf];
      prow = (size_t)(cc >> 1) * 4;
    }
    double racc = 0.0;
    for (int l0 = 0; l0 < Nc8; l0 += chunkw) {
      const int lf = l0 + lane * VPL;
      const bool lv = lf < Nc8;
      double near_[4][VPL], far_[4][VPL];
#pragma unroll
      for (int mm = 0; mm < 4; ++mm) {
        const int oo = c_incoming[dir][mm] - 1;
#pragma unroll
        for (int v = 0; v < VPL; ++v) { near_[mm][v] = 0.0; far_[mm][v] = 0.0; }
        if (!lv) continue;
        ld_vpl<VPL>(a.h + hidx(n1, oo, Nc8, lf), near_[mm]);
        if (code >= 0) ld_vpl<VPL>(a.h + hidx(code, oo, Nc8, lf), far_[mm]);
        else if (plane) ld_vpl<VPL>(plane + (prow + plane_slot(oo)) * Nc8 + lf, far_[mm]);
      }
      double ext[4][VPL];
#pragma unroll
      for (int mm = 0; mm < 4; ++mm) {
        const int oo = c_incoming[dir][mm] - 1;
#pragma unroll
        for (int v = 0; v < VPL; ++v) ext[mm][v] = dadd(dmul(e1, near_[mm][v]), dmul(e2, far_[mm][v]));
        if (lv) {
          if (st == ST_F) st_vpl<VPL>(a.h + hidx(node, oo, Nc8, lf), ext[mm]);
          else if (st == ST_W) st_vpl<VPL>(a.fw + hidx(corner, oo, Nc8, lf), ext[mm]);
        }
      }
      double tface[VPL];
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int l = lf + v;
        const double ca = !lv ? 0.0 : dir < 2 ? __ldg(a.cx + l) : dir < 4 ? __ldg(a.cy + l) : __ldg(a.cz + l);
        tface[v] = dmul(ca, dadd(dadd(dadd(ext[0][v], ext[1][v]), ext[2][v]), ext[3][v]));
      }
      const int nl = min(chunkw, Nc8 - l0);
      for (int sidx = 0; sidx < nl; ++sidx) {
        const int srcl = sidx / VPL, v = sidx % VPL;
        racc = dadd(racc, __shfl_sync(0xffffffffu, (VPL == 2 && v == 1) ? tface[VPL - 1] : tface[0], srcl));
      }
    }
    if (fi == 0) rho0 = racc; else if (fi == 1) rho1 = racc; else rho2 = racc;
  }
  rho0 = __ddiv_rn(rho0, a.DiffFlux);
  if (nface > 1) rho1 = __ddiv_rn(rho1, a.DiffFlux);
  if (nface > 2) rho2 = __ddiv_rn(rho2, a.DiffFlux);
  const double one_m = dsub(1.0, a.accom);
  int zface = -1;
  for (int fi = 0; fi < nface; ++fi) if (P.face[fi].store == ST_Z) zface = fi;
  for (int l0 = 0; l0 < Nc8; l0 += chunkw) {
    const int lf = l0 + lane * VPL;
    if (lf >= Nc8) continue;
    double aw[VPL];
#pragma unroll
    for (int v = 0; v < VPL; ++v) aw[v] = dmul(a.accom, __ldg(a.w + lf + v));
    // re-emission in groups of four writes: the sources of a group are loaded before its
    // stores (no write of a wall program reads a slot that an earlier write stores)
    for (int r0 = 0; r0 < P.nwr; r0 += 4) {
      double src[4][VPL];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (r0 + k >= P.nwr) break;
        const WWrite &W = P.wr[r0 + k];
        const int so = W.src_o - 1;
        if (W.src_store == ST_F) ld_vpl<VPL>(a.h + hidx(node, so, Nc8, lf), src[k]);
        else if (W.src_store == ST_W) ld_vpl<VPL>(a.fw + hidx(corner, so, Nc8, lf), src[k]);
        else {
          double n1v[VPL], farv[VPL];
          ld_vpl<VPL>(a.h + hidx(nb[2 * zface], so, Nc8, lf), n1v);
          const int code = nb[2 * zface + 1];
#pragma unroll
          for (int v = 0; v < VPL; ++v) farv[v] = 0.0;
          if (code >= 0) ld_vpl<VPL>(a.h + hidx(code, so, Nc8, lf), farv);
          else if (code != -1) {
            const int cc = -code - 2;
            const double *plane = (cc & 1) ? a.ghostE[gbuf] : a.ghostW[gbuf];
            ld_vpl<VPL>(plane + ((size_t)(cc >> 1) * 4 + plane_slot(so)) * Nc8 + lf, farv);
          }
#pragma unroll
          for (int v = 0; v < VPL; ++v) src[k][v] = dadd(dmul(e1, n1v[v]), dmul(e2, farv[v]));
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (r0 + k >= P.nwr) break;
        const WWrite &W = P.wr[r0 + k];
        const int dso = W.dst_o - 1;
        double val[VPL];
        const double rf = W.face == 0 ? rho0 : W.face == 1 ? rho1 : rho2;
#pragma unroll
        for (int v = 0; v < VPL; ++v) val[v] = dadd(dmul(aw[v], rf), dmul(one_m, src[k][v]));
        if (W.dst_store == ST_F) st_vpl<VPL>(a.h + hidx(node, dso, Nc8, lf), val);
        else st_vpl<VPL>(a.fw + hidx(corner, dso, Nc8, lf), val);
      }
    }
  }
}

// The diffuse wall for octants of at most 32 * VPL velocities (one pass of the warp), with
// the extrapolated face values kept in shared memory: the re-emission reads them there
// (WPlan) instead of re-loading the slots, and a face value is stored only where it is
// the slot's final content. Same operations on the same operands as k_walls, in the same
// order; per warp, 12 * Nc8 face values and Nc8 density terms. One wall (warp) per block,
// 24 blocks per SM (74 registers, no spills): a block's shared memory is free as soon as its
// wall is done (per iteration on a 128^3 pack: 8 walls per block 0.758 ms, 4 0.698, 2 0.648,
// 1 0.615).
constexpr int kWallWarps = 1;
template <int VPL>
__global__ void __launch_bounds__(kWallWarps * 32, 24 / kWallWarps) k_walls_onchip(const DevState a, int begin, int end, int gbuf) {
  extern __shared__ __align__(16) double wall_sm[];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int widx = begin + (int)blockIdx.x * kWallWarps + wib;
  if (widx >= end) return;  // whole warp (only warp-level synchronisation below)
  const int Nc8 = a.Nc8;
  double *E = wall_sm + (size_t)wib * 13 * Nc8;
  double *Tm = E + 12 * Nc8;
  // the wall's fields from its level-order record (one round trip; see DevState::wall_rec)
  const int4 *rp = a.wall_rec + (size_t)widx * 4;
  const int4 r0 = __ldg(rp);
  const double2 ee = __ldg(reinterpret_cast<const double2 *>(rp + 1));
  const int node = r0.x;
  const int corner = r0.y;
  const WPlan &P = c_plan[c_prog_of[r0.z]];
  const double e1 = ee.x, e2 = ee.y;
  const int nface = P.nface;
  const int lf = lane * VPL;
  const bool lv = lf < Nc8;
  double rho0 = 0.0, rho1 = 0.0, rho2 = 0.0;
  for (int fi = 0; fi < nface; ++fi) {
    const int dir = P.dir[fi], st = P.store[fi], keep = P.keep[fi];
    // the face's (neighbour, far point) pair: the record's second half, an L1 hit
    const int2 nbp = __ldg(reinterpret_cast<const int2 *>(rp + 2) + fi);
    const int n1 = nbp.x, code = nbp.y;
    if (lv) {
      const double *plane = nullptr;
      size_t prow = 0;
      if (code < -1) {
        const int cc = -code - 2;
        plane = (cc & 1) ? a.ghostE[gbuf] : a.ghostW[gbuf];
        prow = (size_t)(cc >> 1) * 4;
      }
      double near_[4][VPL], far_[4][VPL];
#pragma unroll
      for (int mm = 0; mm < 4; ++mm) {
        const int oo = c_incoming[dir][mm] - 1;
#pragma unroll
        for (int v = 0; v < VPL; ++v) far_[mm][v] = 0.0;
        ld_vpl<VPL>(a.h + hidx(n1, oo, Nc8, lf), near_[mm]);
        if (code >= 0) ld_vpl<VPL>(a.h + hidx(code, oo, Nc8, lf), far_[mm]);
        else if (plane) ld_vpl<VPL>(plane + (prow + plane_slot(oo)) * Nc8 + lf, far_[mm]);
      }
      double ext[4][VPL];
#pragma unroll
      for (int mm = 0; mm < 4; ++mm) {
        const int oo = c_incoming[dir][mm] - 1;
#pragma unroll
        for (int v = 0; v < VPL; ++v) ext[mm][v] = dadd(dmul(e1, near_[mm][v]), dmul(e2, far_[mm][v]));
        st_vpl<VPL>(E + (size_t)(fi * 4 + mm) * Nc8 + lf, ext[mm]);
        if (keep >> mm & 1) {
          if (st == ST_F) st_vpl<VPL>(a.h + hidx(node, oo, Nc8, lf), ext[mm]);
          else st_vpl<VPL>(a.fw + hidx(corner, oo, Nc8, lf), ext[mm]);
        }
      }
      double tface[VPL];
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int l = lf + v;
        const double ca = dir < 2 ? __ldg(a.cx + l) : dir < 4 ? __ldg(a.cy + l) : __ldg(a.cz + l);
        tface[v] = dmul(ca, dadd(dadd(dadd(ext[0][v], ext[1][v]), ext[2][v]), ext[3][v]));
      }
      st_vpl<VPL>(Tm + lf, tface);
    }
    __syncwarp();
    // rho_face = sum over l in ascending order (every lane, broadcast reads)
    double racc = 0.0;
    int l = 0;
    for (; l + 8 <= Nc8; l += 8) {
      double t[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) t[j] = Tm[l + j];
#pragma unroll
      for (int j = 0; j < 8; ++j) racc = dadd(racc, t[j]);
    }
    for (; l < Nc8; ++l) racc = dadd(racc, Tm[l]);
    __syncwarp();  // Tm is rewritten by the next face
    if (fi == 0) rho0 = racc; else if (fi == 1) rho1 = racc; else rho2 = racc;
  }
  if (!lv) return;
  rho0 = __ddiv_rn(rho0, a.DiffFlux);
  if (nface > 1) rho1 = __ddiv_rn(rho1, a.DiffFlux);
  if (nface > 2) rho2 = __ddiv_rn(rho2, a.DiffFlux);
  const double one_m = dsub(1.0, a.accom);
  double aw[VPL];
#pragma unroll
  for (int v = 0; v < VPL; ++v) aw[v] = dmul(a.accom, __ldg(a.w + lf + v));
  for (int k = 0; k < P.nwr; ++k) {
    double src[VPL], val[VPL];
    ld_vpl_sm<VPL>(E + (size_t)P.src[k] * Nc8 + lf, src);
    const double rf = P.face[k] == 0 ? rho0 : P.face[k] == 1 ? rho1 : rho2;
#pragma unroll
    for (int v = 0; v < VPL; ++v) val[v] = dadd(dmul(aw[v], rf), dmul(one_m, src[v]));
    if (P.dst_store[k] == ST_F) st_vpl<VPL>(a.h + hidx(node, P.dst_o[k], Nc8, lf), val);
    else st_vpl<VPL>(a.fw + hidx(corner, P.dst_o[k], Nc8, lf), val);
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

// Moments Rho, Ux, Uy, Uz (solver.F90:1923-1938). A warp owns 32 fluid nodes; lane n
// runs node n's four sums serially over (l, octant) in the reference's order. The values
// move through shared memory kMomL velocities at a time, double-buffered with cp.async:
// each copy is an 8-byte piece of a 32-byte (node, octant) segment, so a warp request
// covers 8 whole segments.
constexpr int kMomWarps = 4;
constexpr int kMomL = 4;
constexpr int kMomStride = 8 * kMomL + 1;  // odd stride: lane-per-node reads hit distinct banks
struct MomSmem { double buf[kMomWarps][2][32 * kMomStride]; };

__global__ void __launch_bounds__(kMomWarps * 32) k_moments(const DevState a) {
  extern __shared__ __align__(16) unsigned char mom_raw[];
  MomSmem &S = *reinterpret_cast<MomSmem *>(mom_raw);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int node0 = (blockIdx.x * kMomWarps + wid) * 32;
  if (node0 >= a.NF) return;  // whole warp
  const int Nc8 = a.Nc8;
  const int nvalid = min(32, a.NF - node0);
  // copy assignment: piece p = lane + 32*r (r < 32) of the 1024 pieces of a stage:
  // segment (nn, o) = p / kMomL, velocity lc = p % kMomL
  auto issue = [&](int l0, int b) {
    double *dst = S.buf[wid][b];
    for (int r = 0; r < 32; ++r) {
      const int piece = lane + 32 * r;
      const int seg = piece / kMomL, lc = piece % kMomL;
      const int nn = seg >> 3, o = seg & 7;
      if (nn < nvalid && l0 + lc < Nc8)
        cp_async8(dst + nn * kMomStride + o * kMomL + lc, a.h + hidx(node0 + nn, o, Nc8, l0 + lc));
    }
    cp_async_commit();
  };
  double r = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
  issue(0, 0);
  int b = 0;
  for (int l0 = 0; l0 < Nc8; l0 += kMomL) {
    if (l0 + kMomL < Nc8) { issue(l0 + kMomL, b ^ 1); cp_async_wait<1>(); }
    else cp_async_wait<0>();
    __syncwarp();
    const double *mine = S.buf[wid][b] + lane * kMomStride;
    const int nl = min(kMomL, Nc8 - l0);
    if (lane < nvalid) {
      for (int s2 = 0; s2 < nl; ++s2) {
        const double f1 = mine[0 * kMomL + s2], f2 = mine[1 * kMomL + s2], f3 = mine[2 * kMomL + s2], f4 = mine[3 * kMomL + s2];
        const double f5 = mine[4 * kMomL + s2], f6 = mine[5 * kMomL + s2], f7 = mine[6 * kMomL + s2], f8 = mine[7 * kMomL + s2];
        r = dadd(dadd(dadd(dadd(dadd(dadd(dadd(dadd(r, f1), f2), f3), f4), f5), f6), f7), f8);
        const double dx = dadd(dsub(dsub(dadd(dadd(dsub(dsub(f1, f2), f3), f4), f5), f6), f7), f8);
        const double dy = dsub(dsub(dadd(dadd(dsub(dsub(dadd(f1, f2), f3), f4), f5), f6), f7), f8);
        const double dz = dsub(dsub(dsub(dsub(dadd(dadd(dadd(f1, f2), f3), f4), f5), f6), f7), f8);
        ux = dadd(ux, dmul(__ldg(a.cx + l0 + s2), dx));
        uy = dadd(uy, dmul(__ldg(a.cy + l0 + s2), dy));
        uz = dadd(uz, dmul(__ldg(a.cz + l0 + s2), dz));
      }
    }
    __syncwarp();
    b ^= 1;
  }
  if (lane < nvalid) {
    const int n = node0 + lane;
    double2 *mp = reinterpret_cast<double2 *>(a.mom) + 2 * (size_t)n;
    mp[0] = make_double2(r, ux);
    mp[1] = make_double2(uy, uz);
  }
}

// The same sums for octants whose velocity count is a multiple of 8: each stage moves 8
// velocities of every (node, octant) of the warp's 32 nodes, a 64-byte segment per
// (node, octant) in four 16-byte copies (four lanes per segment, eight segments per warp
// request). A node's staged row holds 66 doubles (8 octants x 8 velocities + 2 pad), so a
// quarter-warp's 16-byte reads cover all 32 banks.
constexpr int kMomWWarps = 2;
constexpr int kMomWL = 8;
constexpr int kMomWStride = 8 * kMomWL + 2;
struct MomWSmem { double buf[kMomWWarps][2][32 * kMomWStride]; };

__global__ void __launch_bounds__(kMomWWarps * 32) k_moments_wide(const DevState a) {
  extern __shared__ __align__(16) unsigned char mom_raw[];
  MomWSmem &S = *reinterpret_cast<MomWSmem *>(mom_raw);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int node0 = (blockIdx.x * kMomWWarps + wid) * 32;
  if (node0 >= a.NF) return;  // whole warp
  const int Nc8 = a.Nc8;
  const int nvalid = min(32, a.NF - node0);
  // piece p = lane + 32*r (r < 32) of a stage's 1024: segment (nn, o) = p / 4, quarter p % 4
  const int pc = lane & 3;
  auto issue = [&](int l0, int b) {
    double *dst = S.buf[wid][b];
#pragma unroll 8
    for (int r = 0; r < 32; ++r) {
      const int seg = (lane >> 2) + 8 * r;
      const int nn = seg >> 3, o = seg & 7;
      if (nn < nvalid)
        cp_async16_cg(dst + nn * kMomWStride + o * kMomWL + 2 * pc, a.h + hidx(node0 + nn, o, Nc8, l0 + 2 * pc));
    }
    cp_async_commit();
  };
  double r = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
  issue(0, 0);
  int b = 0;
  for (int l0 = 0; l0 < Nc8; l0 += kMomWL) {
    if (l0 + kMomWL < Nc8) { issue(l0 + kMomWL, b ^ 1); cp_async_wait<1>(); }
    else cp_async_wait<0>();
    __syncwarp();
    double cxs[kMomWL], cys[kMomWL], czs[kMomWL];
#pragma unroll
    for (int s2 = 0; s2 < kMomWL; ++s2) {
      cxs[s2] = __ldg(a.cx + l0 + s2); cys[s2] = __ldg(a.cy + l0 + s2); czs[s2] = __ldg(a.cz + l0 + s2);
    }
    const double *mine = S.buf[wid][b] + lane * kMomWStride;
    if (lane < nvalid) {
#pragma unroll
      for (int j = 0; j < kMomWL / 2; ++j) {
        double2 g[8];
#pragma unroll
        for (int o = 0; o < 8; ++o) g[o] = *reinterpret_cast<const double2 *>(mine + o * kMomWL + 2 * j);
#pragma unroll
        for (int h2 = 0; h2 < 2; ++h2) {
          const double f1 = h2 ? g[0].y : g[0].x, f2 = h2 ? g[1].y : g[1].x, f3 = h2 ? g[2].y : g[2].x,
                       f4 = h2 ? g[3].y : g[3].x, f5 = h2 ? g[4].y : g[4].x, f6 = h2 ? g[5].y : g[5].x,
                       f7 = h2 ? g[6].y : g[6].x, f8 = h2 ? g[7].y : g[7].x;
          r = dadd(dadd(dadd(dadd(dadd(dadd(dadd(dadd(r, f1), f2), f3), f4), f5), f6), f7), f8);
          const double dx = dadd(dsub(dsub(dadd(dadd(dsub(dsub(f1, f2), f3), f4), f5), f6), f7), f8);
          const double dy = dsub(dsub(dadd(dadd(dsub(dsub(dadd(f1, f2), f3), f4), f5), f6), f7), f8);
          const double dz = dsub(dsub(dsub(dsub(dadd(dadd(dadd(f1, f2), f3), f4), f5), f6), f7), f8);
          ux = dadd(ux, dmul(cxs[2 * j + h2], dx));
          uy = dadd(uy, dmul(cys[2 * j + h2], dy));
          uz = dadd(uz, dmul(czs[2 * j + h2], dz));
        }
      }
    }
    __syncwarp();
    b ^= 1;
  }
  if (lane < nvalid) {
    const int n = node0 + lane;
    double2 *mp = reinterpret_cast<double2 *>(a.mom) + 2 * (size_t)n;
    mp[0] = make_double2(r, ux);
    mp[1] = make_double2(uy, uz);
  }
}

// Mass flux through x = 2 (output.F90:90-142) in the reference's summation order: the
// block gathers the plane's Ux values into shared memory in parallel, one thread then
// accumulates them serially. Runs over the plane in tiles of kFluxTile entries.
constexpr int kFluxTile = 4096;
__global__ void __launch_bounds__(256) k_flux(const DevState a, double ds, double sqrt_half, double inv_refl2) {
  __shared__ double tm[kFluxTile];
  __shared__ double part[9];
  __shared__ int fg[10];
  __shared__ int gi_s;
  __shared__ double acc_s;
  if (threadIdx.x < 10) fg[threadIdx.x] = a.flux_groups[threadIdx.x];
  if (threadIdx.x == 0) { gi_s = 0; acc_s = 0.0; }
  __syncthreads();
  const int total = fg[9];
  for (int base = 0; base < total; base += kFluxTile) {
    const int cnt = min(kFluxTile, total - base);
    // every entry's term (dx*dx*Ux, halved on the edges, quartered at the corners)
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
      const int idx = base + e;
      const int n = a.flux_list[idx];
      int g = 0;
      while (g < 8 && idx >= fg[g + 1]) ++g;
      double term = dmul(dmul(n >= 0 ? a.mom[4 * (size_t)n + 1] : 0.0, ds), ds);
      if (g >= 1 && g <= 4) term = dmul(term, 0.5);
      else if (g >= 5) term = dmul(term, 0.25);
      tm[e] = term;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      // the serial sums in the reference's order, one group segment at a time
      int gi = gi_s;
      double s = acc_s;
      int idx = base;
      const int end = base + cnt;
      while (idx < end) {
        while (idx >= fg[gi + 1]) { part[gi] = s; ++gi; s = 0.0; }
        const int seg_end = min(end, fg[gi + 1]);
        if (gi <= 4) {
#pragma unroll 8
          for (; idx < seg_end; ++idx) s = dadd(s, tm[idx - base]);
        } else {
          for (; idx < seg_end; ++idx) s = tm[idx - base];
        }
      }
      gi_s = gi;
      acc_s = s;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int gi = gi_s;
    double s = acc_s;
    while (gi < 9) { part[gi] = s; ++gi; s = 0.0; }
    double m = part[0];
    for (int g = 1; g < 9; ++g) m = dadd(m, part[g]);
    a.flux_out[0] = __ddiv_rn(__ddiv_rn(dmul(m, sqrt_half), a.pressDrop), inv_refl2);
  }
}

inline unsigned blocks_for(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// Self-test of markstein_div against __ddiv_rn: numerators and denominators spread over
// 2^-40 .. 2^40 with random mantissas (splitmix64), plus denominators in the range the
// sweep uses.
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ double random_double(uint64_t r, int emin, int erange) {
  const uint64_t mant = r & ((1ull << 52) - 1);
  const int e = emin + (int)((r >> 52) % (uint64_t)erange);
  const uint64_t bits = ((uint64_t)(e + 1023) << 52) | mant;
  double d = __longlong_as_double((long long)bits);
  return (r >> 63) ? -d : d;
}
__global__ void k_division_selftest(int64_t samples, uint64_t seed, unsigned long long *mismatches) {
  unsigned long long bad = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < samples; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t r1 = splitmix64(seed ^ (uint64_t)(2 * i)), r2 = splitmix64(seed ^ (uint64_t)(2 * i + 1));
    const double num = random_double(r1, -40, 80);
    double den = random_double(r2, -40, 80);
    if (i & 1) den = fabs(random_double(r2, -2, 9));  // 0.25 .. 128: the sweep's range
    const double y = __ddiv_rn(1.0, den);
    const double q = markstein_div(num, den, y);
    const double ref = __ddiv_rn(num, den);
    if (__double_as_longlong(q) != __double_as_longlong(ref)) ++bad;
  }
  if (bad) atomicAdd(mismatches, bad);
}

}  // namespace

// ---------------------------------------------------------------------------------------
// Allocation-free variant of the division self-test (piks_selftest_division_noalloc).
// Its scratch is this file-scope device array: one count per block of the test grid, then
// the total and the number of samples tested. Every GPU that loads the library holds it
// (8 KB + 16 bytes) until the process exits; all calls share it and it keeps the last
// call's contents.
constexpr int kNoAllocBlocks = 1024;
constexpr int kNoAllocThreads = 256;
constexpr int64_t kNoAllocPerBlock = (int64_t)kNoAllocThreads * 64;   // samples per block
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocBlocks + 2];

__device__ __forceinline__ bool division_sample_differs(int64_t i, uint64_t seed) {
  const uint64_t r1 = splitmix64(seed ^ (uint64_t)(2 * i)), r2 = splitmix64(seed ^ (uint64_t)(2 * i + 1));
  const double num = random_double(r1, -40, 80);
  double den = random_double(r2, -40, 80);
  if (i & 1) den = fabs(random_double(r2, -2, 9));
  const double y = __ddiv_rn(1.0, den);
  return __double_as_longlong(markstein_div(num, den, y)) != __double_as_longlong(__ddiv_rn(num, den));
}

// Each block counts the mismatches of its own sample range and writes its slot: the low 32
// bits hold the mismatches, the high 32 bits the number of samples the block tested (at
// most kNoAllocPerBlock each). The sum of the high halves is the call's completion count.
__global__ void __launch_bounds__(kNoAllocThreads)
k_division_selftest_blocks(int64_t samples, uint64_t seed, unsigned long long *partial) {
  __shared__ unsigned int warp_bad[kNoAllocThreads / 32];
  __shared__ unsigned int warp_done[kNoAllocThreads / 32];
  const int64_t lo = (int64_t)blockIdx.x * kNoAllocPerBlock;
  const int64_t hi = min(samples, lo + kNoAllocPerBlock);
  unsigned int bad = 0, done = 0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kNoAllocThreads) {
    bad += division_sample_differs(i, seed) ? 1u : 0u;
    ++done;
  }
  for (int off = 16; off > 0; off >>= 1) {
    bad += __shfl_down_sync(0xffffffffu, bad, off);
    done += __shfl_down_sync(0xffffffffu, done, off);
  }
  if ((threadIdx.x & 31) == 0) { warp_bad[threadIdx.x >> 5] = bad; warp_done[threadIdx.x >> 5] = done; }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long b = 0, d = 0;
    for (int w = 0; w < kNoAllocThreads / 32; ++w) { b += warp_bad[w]; d += warp_done[w]; }
    partial[blockIdx.x] = b | (d << 32);
  }
}

// total = (sum of mismatches, sum of tested samples); both fit 32 bits at the sample limit.
__global__ void k_sum_partials(const unsigned long long *partial, int n, unsigned long long *total) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long b = 0, d = 0;
    for (int k = 0; k < n; ++k) { b += partial[k] & 0xffffffffull; d += partial[k] >> 32; }
    total[0] = b;
    total[1] = d;
  }
}

namespace {
// Makes `device` current for the guard's lifetime and restores the caller's device after.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&prev) != cudaSuccess) { cudaGetLastError(); prev = -1; }
    ok = cudaSetDevice(device) == cudaSuccess;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};
}  // namespace

int division_selftest_noalloc(int device, int64_t samples, uint64_t seed, int64_t *mismatches, const char **err) {
  if (device < 0) { *err = "device index out of range"; return 1; }
  if (samples <= 0) { *err = "samples must be positive"; return 1; }
  const int64_t max_samples = (int64_t)kNoAllocBlocks * kNoAllocPerBlock;
  if (samples > max_samples) {
    *err = "samples exceeds 16777216, the most this allocation-free self-test runs with its static scratch";
    return 1;
  }
  DeviceGuard guard(device);
  if (!guard.ok) { cudaGetLastError(); *err = "cudaSetDevice failed"; return 4; }
  // The host-side name of the array is not a device address: look the address up on the
  // current device on every call (a lookup, which allocates nothing). The first lookup on a
  // device can load the library's device code, so make the first call before any capture.
  void *ptr = nullptr;
  if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) {
    cudaGetLastError();
    *err = "cudaGetSymbolAddress of the self-test scratch failed";
    return 4;
  }
  unsigned long long *scratch = static_cast<unsigned long long *>(ptr);
  // the total and the completion count start at zero, so a stale total never comes back
  if (cudaMemsetAsync(scratch + kNoAllocBlocks, 0, 2 * sizeof(unsigned long long), 0) != cudaSuccess) {
    cudaGetLastError();
    *err = "clearing the self-test total failed";
    return 4;
  }
  const int blocks = (int)((samples + kNoAllocPerBlock - 1) / kNoAllocPerBlock);
  k_division_selftest_blocks<<<blocks, kNoAllocThreads>>>(samples, seed, scratch);
  if (cudaGetLastError() != cudaSuccess) { *err = "self-test kernel launch failed"; return 4; }
  k_sum_partials<<<1, 32>>>(scratch, blocks, scratch + kNoAllocBlocks);
  if (cudaGetLastError() != cudaSuccess) { *err = "self-test sum launch failed"; return 4; }
  unsigned long long total[2] = {0, 0};
  if (cudaMemcpy(total, scratch + kNoAllocBlocks, sizeof total, cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    *err = "self-test copy failed";
    return 4;
  }
  if (total[1] != (unsigned long long)samples) {
    *err = "self-test kernels did not test every sample";
    return 4;
  }
  *mismatches = (int64_t)total[0];
  return 0;
}

namespace {
std::mutex g_config_mu;
std::set<std::pair<const void *, int>> g_configured;
std::map<std::tuple<const void *, int, int, size_t>, long> g_resident;
}  // namespace

void once_per_device(const void *key, void (*configure)(int device)) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_config_mu);
  if (g_configured.insert({key, dev}).second) configure(dev);
}

long resident_blocks(const void *fn, int threads, size_t smem) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_config_mu);
  const auto key = std::make_tuple(fn, dev, threads, smem);
  auto it = g_resident.find(key);
  if (it != g_resident.end()) return it->second;
  int nb = 0, nsm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess) { cudaGetLastError(); nb = 1; }
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) { cudaGetLastError(); nsm = 148; }
  const long r = (long)(nb < 1 ? 1 : nb) * (nsm < 1 ? 1 : nsm);
  g_resident[key] = r;
  return r;
}

void launch_division_selftest(int64_t samples, uint64_t seed, unsigned long long *mismatches) {
  k_division_selftest<<<148 * 8, 256>>>(samples, seed, mismatches);
}

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
  WPlan plans[26];
  int ok = n == 26;
  for (int i = 0; i < n; ++i) ok &= make_wall_plan(progs[i], plans[i]) ? 1 : 0;
  g_plan_ok = ok != 0;
  cudaMemcpyToSymbol(c_plan, plans, sizeof plans);
}

void launch_sweep_hyperplane(const DevState &s, long t0, long ntask, cudaStream_t st) {
  if (ntask <= 0) return;
  if (s.lpt == 32) {
    const size_t threads = (size_t)ntask * s.nchunk * 32;
    k_sweep<32, 2><<<blocks_for(threads, 256), 256, 0, st>>>(s, t0, ntask);
  } else {
    const size_t threads = (size_t)ntask * s.nchunk * 8;
    k_sweep<8, 1><<<blocks_for(threads, 256), 256, 0, st>>>(s, t0, ntask);
  }
}

void launch_commit_rows(const DevState &s, bool fp32, cudaStream_t st) {
  const int pieces = s.Nc8 * (fp32 ? 4 : 8) / 16;
  int4 *h = reinterpret_cast<int4 *>(fp32 ? (void *)s.h32 : (void *)s.h);
  const int4 *fw = reinterpret_cast<const int4 *>(fp32 ? (const void *)s.fw32 : (const void *)s.fw);
  k_commit16<<<blocks_for((size_t)s.ncommit * pieces, 256), 256, 0, st>>>(s.commit, s.bcorner, s.NF, h, fw,
                                                                          s.ncommit, pieces);
}

void launch_commit(const DevState &s, cudaStream_t st) {
  if (s.ncommit == 0) return;
  if (s.Nc8 % 2 == 0) return launch_commit_rows(s, false, st);
  const size_t n = (size_t)s.ncommit * s.Nc8;
  k_commit<<<blocks_for(n, 256), 256, 0, st>>>(s);
}

void launch_capture(const DevState &s, int buf, cudaStream_t st) {
  const size_t n = (size_t)s.Ny * s.Nz * 4 * s.Nc8;
  k_capture<<<blocks_for(n, 256), 256, 0, st>>>(s, buf);
}

// Halo rows (solver.F90:535-560 for the planes of a slab boundary): element idx of a
// [count][4][Nc8] buffer is row (nodes[q], octant set[k]) at velocity l; `pack` copies rows
// into the buffer, otherwise the buffer into the rows. cx > 0 octants are 0, 3, 4, 7.
template <typename T>
__global__ void k_halo_rows(T *h, T *buf, const int32_t *nodes, int count, int cx_pos, int Nc8, bool pack) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)count * 4 * Nc8) return;
  const int l = (int)(idx % Nc8);
  const int k = (int)((idx / Nc8) % 4);
  const int q = (int)(idx / ((size_t)Nc8 * 4));
  const int o = cx_pos ? ((k == 0) ? 0 : (k == 1) ? 3 : (k == 2) ? 4 : 7) : ((k == 0) ? 1 : (k == 1) ? 2 : (k == 2) ? 5 : 6);
  T *row = h + hidx(nodes[q], o, Nc8, l);
  if (pack) buf[idx] = *row;
  else *row = buf[idx];
}

template <typename T>
void halo_rows(T *h, T *buf, const int32_t *nodes, int count, int cx_pos, int Nc8, bool pack, cudaStream_t st) {
  if (count <= 0) return;
  const size_t n = (size_t)count * 4 * Nc8;
  k_halo_rows<T><<<blocks_for(n, 256), 256, 0, st>>>(h, buf, nodes, count, cx_pos, Nc8, pack);
}

void launch_halo(const DevState &s, bool fp32, int cap, cudaStream_t st) {
  for (int side = 0; side < 2; ++side) {
    // the west neighbour reads this slab's cx < 0 rows, the east one its cx > 0 rows; the
    // west ghost planes receive cx > 0 rows, the east ones cx < 0 rows
    const int send_pos = side == 1, recv_pos = side == 0;
    if (fp32) {
      halo_rows(s.h32, s.hsend32[side][cap], s.halo_send[side], s.nhalo_send[side], send_pos, s.Nc8, true, st);
      halo_rows(s.h32, s.hrecv32[side], s.halo_recv[side], s.nhalo_recv[side], recv_pos, s.Nc8, false, st);
    } else {
      halo_rows(s.h, s.hsend[side][cap], s.halo_send[side], s.nhalo_send[side], send_pos, s.Nc8, true, st);
      halo_rows(s.h, s.hrecv[side], s.halo_recv[side], s.nhalo_recv[side], recv_pos, s.Nc8, false, st);
    }
  }
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
  once_per_device(reinterpret_cast<const void *>(k_moments), [](int) {
    cudaFuncSetAttribute(k_moments, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MomSmem));
    cudaFuncSetAttribute(k_moments_wide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MomWSmem));
  });
  if (s.Nc8 % kMomWL == 0) {
    k_moments_wide<<<blocks_for((size_t)s.NF, kMomWWarps * 32), kMomWWarps * 32, sizeof(MomWSmem), st>>>(s);
    return;
  }
  k_moments<<<blocks_for((size_t)s.NF, kMomWarps * 32), kMomWarps * 32, sizeof(MomSmem), st>>>(s);
}

void launch_walls(const DevState &s, int begin, int end, int gbuf, cudaStream_t st) {
  if (end <= begin) return;
  if (g_plan_ok && s.Nc8 <= 64 && (s.Nc8 <= 32 || s.Nc8 % 2 == 0)) {
    once_per_device(reinterpret_cast<const void *>(k_walls_onchip<1>), [](int) {
      const int most = kWallWarps * 13 * 64 * (int)sizeof(double);
      cudaFuncSetAttribute(k_walls_onchip<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
      cudaFuncSetAttribute(k_walls_onchip<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
    });
    const size_t smem = (size_t)kWallWarps * 13 * s.Nc8 * sizeof(double);
    const unsigned grid = blocks_for((size_t)(end - begin), kWallWarps);
    if (s.Nc8 > 32) k_walls_onchip<2><<<grid, kWallWarps * 32, smem, st>>>(s, begin, end, gbuf);
    else k_walls_onchip<1><<<grid, kWallWarps * 32, smem, st>>>(s, begin, end, gbuf);
    return;
  }
  const size_t threads = (size_t)(end - begin) * 32;
  if (s.Nc8 % 64 == 0) k_walls<2><<<blocks_for(threads, 256), 256, 0, st>>>(s, begin, end, gbuf);
  else k_walls<1><<<blocks_for(threads, 256), 256, 0, st>>>(s, begin, end, gbuf);
}

void launch_flux(const DevState &s, double ds, double sqrt_half, double inv_refl2, cudaStream_t st) {
  k_flux<<<1, 256, 0, st>>>(s, ds, sqrt_half, inv_refl2);
}

}  // namespace piks
