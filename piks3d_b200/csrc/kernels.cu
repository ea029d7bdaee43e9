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
  const double rho = __ldg(a.rho + m), ux = __ldg(a.ux + m), uy = __ldg(a.uy + m), uz = __ldg(a.uz + m);
  const int cls = (fx ? 1 : 0) | (fy ? 2 : 0) | (fz ? 4 : 0);
  const bool nx_ = dsx(o) < 0, ny_ = dsy(o) < 0, nz_ = dsz(o) < 0;
  double out[VPL];
#pragma unroll
  for (int q = 0; q < VPL; ++q) {
    const int l = lfirst + q;
    const double *vt = a.vtab + (size_t)l * kVtab;  // cx cy cz w, products, dens, recips
    const double cx = __ldg(vt + 0), cy = __ldg(vt + 1), cz = __ldg(vt + 2), wl = __ldg(vt + 3);
    const double ex = dmul(nx_ ? -cx : cx, ux), ey = dmul(ny_ ? -cy : cy, uy), ez = dmul(nz_ ? -cz : cz, uz);
    const double feq = dmul(wl, dadd(rho, dadd(dadd(ex, ey), ez)));
    double num = dmul(a.mu, dsub(feq, dmul(0.5, fold[q])));
    num = dadd(num, dmul(__ldg(vt + (fx ? 5 : 4)), x1[q]));
    if (!fx) num = dadd(num, dmul(__ldg(vt + 6), x2[q]));
    num = dadd(num, dmul(__ldg(vt + (fy ? 8 : 7)), y1[q]));
    if (!fy) num = dadd(num, dmul(__ldg(vt + 9), y2[q]));
    num = dadd(num, dmul(__ldg(vt + (fz ? 11 : 10)), z1[q]));
    if (!fz) num = dadd(num, dmul(__ldg(vt + 12), z2[q]));
    out[q] = markstein_div(num, __ldg(vt + 13 + cls), __ldg(vt + 21 + cls));
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

// Moments Rho, Ux, Uy, Uz (solver.F90:1923-1938). One lane per fluid node runs the four
// sums serially over (l, octant) in the reference's order; a warp stages its 32 nodes'
// values 8 velocities at a time in shared memory with coalesced 64-byte row loads.
constexpr int kMomWarps = 2;
constexpr int kMomL = 8;
constexpr int kMomStride = 8 * kMomL + 1;  // odd stride in doubles: conflict-free lane reads
__global__ void __launch_bounds__(kMomWarps * 32) k_moments(const DevState a) {
  __shared__ double sm[kMomWarps][32 * kMomStride];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int node0 = (blockIdx.x * kMomWarps + wid) * 32;
  if (node0 >= a.NF) return;  // whole warp
  const int Nc8 = a.Nc8;
  const int my = node0 + lane;
  const bool valid = my < a.NF;
  double r = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
  double *buf = sm[wid];
  for (int l0 = 0; l0 < Nc8; l0 += kMomL) {
    // 32 nodes x 8 octants rows of kMomL values; lane group g (4 groups of 8 lanes) loads a row
    const int sub = lane & 7, grp = lane >> 3;
    for (int row = grp; row < 32 * 8; row += 4) {
      const int nn = row >> 3, o = row & 7;
      const int node = node0 + nn;
      double val = 0.0;
      if (node < a.NF && l0 + sub < Nc8) val = __ldcs(a.h + hidx(node, o, Nc8, l0 + sub));
      buf[nn * kMomStride + o * kMomL + sub] = val;
    }
    __syncwarp();
    const int nl = min(kMomL, Nc8 - l0);
    const double *mine = buf + lane * kMomStride;
    for (int s = 0; s < nl; ++s) {
      const double f1 = mine[0 * kMomL + s], f2 = mine[1 * kMomL + s], f3 = mine[2 * kMomL + s], f4 = mine[3 * kMomL + s];
      const double f5 = mine[4 * kMomL + s], f6 = mine[5 * kMomL + s], f7 = mine[6 * kMomL + s], f8 = mine[7 * kMomL + s];
      r = dadd(dadd(dadd(dadd(dadd(dadd(dadd(dadd(r, f1), f2), f3), f4), f5), f6), f7), f8);
      const double dx = dadd(dsub(dsub(dadd(dadd(dsub(dsub(f1, f2), f3), f4), f5), f6), f7), f8);
      const double dy = dsub(dsub(dadd(dadd(dsub(dsub(dadd(f1, f2), f3), f4), f5), f6), f7), f8);
      const double dz = dsub(dsub(dsub(dsub(dadd(dadd(dadd(f1, f2), f3), f4), f5), f6), f7), f8);
      ux = dadd(ux, dmul(__ldg(a.cx + l0 + s), dx));
      uy = dadd(uy, dmul(__ldg(a.cy + l0 + s), dy));
      uz = dadd(uz, dmul(__ldg(a.cz + l0 + s), dz));
    }
    __syncwarp();
  }
  if (valid) { a.rho[my] = r; a.ux[my] = ux; a.uy[my] = uy; a.uz[my] = uz; }
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
  k_moments<<<blocks_for((size_t)s.NF, kMomWarps * 32), kMomWarps * 32, 0, st>>>(s);
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
