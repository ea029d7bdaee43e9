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
// One CTA = one tile of TV x TW pencils of one octant and one chunk of 32*VPL velocities
// (VPL per lane). Warp (pv, pw) owns pencil (v, w) of the octant's local frame (u, v, w
// increase along the sweep) and walks u = 1 .. Nx-1 keeping the two x-upwind values in
// registers. Pencils advance on a diagonal schedule, pencil (pv, pw) handling u at step
// t = u - 1 + pv + pw, so a node's y/z-upwind values inside the tile were produced one or
// two steps earlier and sit in a 3-deep shared-memory ring. Tiles of one launch lie on one
// anti-diagonal of the tile grid; their y/z-upwind tiles finished in earlier launches.
//
// Everything a step reads from global memory (node map rows, the old value, the moments,
// upwind values that are not produced inside the tile) is fetched one step ahead, node-map
// rows 32 positions at a time, so a step waits only for the ring and its own arithmetic.
//
// Arithmetic (solver.F90:206-214) in the reference's order. Written in the octant's local
// frame every term is added with a non-negative-octant coefficient: for a negative
// velocity axis the reference subtracts (c * -C) * f, which is bit-identical to adding
// (c * C) * f. The coefficient products c*C and the denominators depend only on the
// velocity and on the first/second-order flags of the three axes, so they are tabulated
// (same operations, same rounding); the division num/den is evaluated from the correctly
// rounded reciprocal y = RN(1/den) by Markstein's correction q = RN(q0 + RN-exact(num -
// den*q0) * y) with q0 = RN(num*y), which returns RN(num/den) (Markstein, IBM J. Res. Dev.
// 34 (1990); see piks_selftest_division for the check against __ddiv_rn).
__device__ __forceinline__ double markstein_div(double num, double den, double y) {
  const double q0 = __dmul_rn(num, y);
  const double r = __fma_rn(-q0, den, num);
  return __fma_rn(r, y, q0);
}

// Asynchronous global->shared copies (cp.async): 16-byte L2-only and 8-byte variants.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Where a fluid node's y1/y2/z1/z2 upwind value comes from, resolved when the node-map
// block is loaded: kSrcRing (fluid node of this tile: shared ring), kSrcZero (ghost layer,
// only ever multiplied by 0), or a static slot: node*8 + slot of h, or with kSrcFw set,
// corner*8 + octant of fw (a wall slot as switched in the reference, solver.F90:184-204).
constexpr int kSrcRing = -1, kSrcZero = -2, kSrcFw = 1 << 30;

template <int TV, int TW, int VPL, int D>
struct SweepSmem {
  static constexpr int NP = TV * TW, NV = 32 * VPL;
  double ring[3][NP][NV];
  double Dn[8][NV];           // denominators by first-order class (fx | fy<<1 | fz<<2)
  double Rc[8][NV];           // their correctly rounded reciprocals
  struct Stage {
    double fold[NV];          // old value of the node (or slot o of a solid node)
    double st[4][NV];         // static upwind values (y1, y2, z1, z2)
    double mom[4];            // Rho, Ux, Uy, Uz
  } pipe[NP][D];
  int meta[NP][D][2];         // node, flags
};

// flags of a pencil position: bit 0 fy, bit 1 fz (first order in y / z), bits 2..5 which
// of y1, y2, z1, z2 come from the ring, bits 8..15 the voxel label.
template <int TV, int TW, int VPL, int D>
__global__ void __launch_bounds__(TV * TW * 32, 1)
k_sweep(const DevState a, int diag, int ntw) {
  using SM = SweepSmem<TV, TW, VPL, D>;
  constexpr int NV = SM::NV;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SM &S = *reinterpret_cast<SM *>(smem_raw);
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
  const int lbase = chunk * NV;
  for (int e = threadIdx.x; e < NV; e += blockDim.x) {
    const int l = lbase + e;
    const bool ok = l < Nc8;
    for (int cls = 0; cls < 8; ++cls) {
      S.Dn[cls][e] = ok ? a.dtab[(size_t)cls * Nc8 + l] : 1.0;
      S.Rc[cls][e] = ok ? a.rtab[(size_t)cls * Nc8 + l] : 1.0;
    }
  }
  // this lane's velocities: e = lane*VPL + q (contiguous pairs for 16-byte copies).
  // fEq needs +-c*U: multiplying by the signed velocity component rounds identically.
  double scx[VPL], scy[VPL], scz[VPL], wv[VPL];
  double px2[VPL], px1[VPL], pxh[VPL], py2[VPL], py1[VPL], pyh[VPL], pz2[VPL], pz1[VPL], pzh[VPL];
  bool lv[VPL];
#pragma unroll
  for (int q = 0; q < VPL; ++q) {
    const int l = lbase + lane * VPL + q;
    lv[q] = l < Nc8;
    const double cx = lv[q] ? a.cx[l] : 0.0, cy = lv[q] ? a.cy[l] : 0.0, cz = lv[q] ? a.cz[l] : 0.0;
    scx[q] = sx > 0 ? cx : -cx; scy[q] = sy > 0 ? cy : -cy; scz[q] = sz > 0 ? cz : -cz;
    wv[q] = lv[q] ? a.w[l] : 0.0;
    // coefficient products c*C of the upwind terms: second-order C1 = 2/ds, first-order
    // C1 = 1/ds, second-order C2 = -0.5/ds (physicalGrid.F90:1259-1297)
    px2[q] = dmul(cx, a.c20); px1[q] = dmul(cx, a.c10); pxh[q] = dmul(cx, a.c05);
    py2[q] = dmul(cy, a.c20); py1[q] = dmul(cy, a.c10); pyh[q] = dmul(cy, a.c05);
    pz2[q] = dmul(cz, a.c20); pz1[q] = dmul(cz, a.c10); pzh[q] = dmul(cz, a.c05);
  }
  const bool lane_ok = lv[0];  // VPL = 2 is used only when Nc8 is a multiple of 64
  const uint8_t xbit = sx > 0 ? FACE_E : FACE_W;
  const uint8_t ybit = sy > 0 ? FACE_N : FACE_S;
  const uint8_t zbit = sz > 0 ? FACE_F : FACE_B;
  const int j = sy > 0 ? v + 1 : a.Ny - v;
  const int k = sz > 0 ? w + 1 : a.Nz - w;
  const int i0 = sx > 0 ? 1 : a.Nx;
  const long gbase = (long)(i0 + 1) + (long)(j + 1) * a.GX + (long)(k + 1) * a.GXY;
  const long SY = (long)sy * a.GX, SZ = (long)sz * a.GXY;
  const double mu = a.mu;
  const int Nx = a.Nx;
  const bool intile[4] = {pv >= 1, pv >= 2, pw >= 1, pw >= 2};

  // Node-map block: lane i describes position u = ub + i of this pencil.
  struct Block { int m, flags, src[4]; };
  auto load_block = [&](int ubase, Block &B) {
    const int u = ubase + lane;
    B.m = -2; B.flags = 0;
    B.src[0] = B.src[1] = B.src[2] = B.src[3] = kSrcZero;
    if (!active || u > Nx - 1) return;
    const long g = gbase + (long)sx * u;
    B.m = __ldg(a.nodemap + g);
    const int lab = __ldg(a.label + g);
    const bool fy = (v == 1) || (c_face[__ldg(a.label + g - SY)] & ybit);
    const bool fz = (w == 1) || (c_face[__ldg(a.label + g - SZ)] & zbit);
    int fl = (fy ? 1 : 0) | (fz ? 2 : 0) | (lab << 8);
    if (B.m >= 0 && B.m < a.NF && u >= 1) {
      const long gq[4] = {g - SY, g - 2 * SY, g - SZ, g - 2 * SZ};
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int mr = __ldg(a.nodemap + gq[r]);
        int code = kSrcZero;
        if (mr >= 0 && mr < a.NF) {
          if (intile[r]) { code = kSrcRing; fl |= 4 << r; }
          else code = mr * 8 + o;
        } else if (mr >= a.NF) {
          const int bb = mr - a.NF;
          const int src = (__ldg(a.roles + (size_t)bb * 8 + o) >> (4 * r)) & 15;
          code = src < 8 ? mr * 8 + src : (kSrcFw | (__ldg(a.bcorner + bb) * 8 + o));
        }
        B.src[r] = code;
      }
    }
    B.flags = fl;
  };
  Block cur, nxt;
  int ub = 0;
  load_block(0, cur);
  load_block(32, nxt);

  // Issue the copies of position ui into pipeline stage ui % D (one commit group).
  auto issue = [&](int ui) {
    if (ui <= Nx - 1) {
      if (ui - ub >= 32) {
        ub += 32;
        cur = nxt;
        load_block(ub + 32, nxt);
      }
      const int s = ui - ub;
      const int m = __shfl_sync(0xffffffffu, cur.m, s);
      const int fl = __shfl_sync(0xffffffffu, cur.flags, s);
      const int slot = ui % D;
      typename SM::Stage &st = S.pipe[wid][slot];
      if (lane == 0) { S.meta[wid][slot][0] = m; S.meta[wid][slot][1] = fl; }
      if (m >= 0 && lane_ok) {
        const double *gp = a.h + hidx(m, o, Nc8, lbase + lane * VPL);
        if (VPL == 2) cp_async16(&st.fold[lane * 2], gp); else cp_async8(&st.fold[lane], gp);
      }
      if (m >= 0 && m < a.NF && ui >= 1) {
        if (lane < 4) {
          const double *mp = lane == 0 ? a.rho : lane == 1 ? a.ux : lane == 2 ? a.uy : a.uz;
          cp_async8(&st.mom[lane], mp + m);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int sr = __shfl_sync(0xffffffffu, cur.src[r], s);
          if (sr < 0 || !lane_ok) continue;
          const double *gp = (sr & kSrcFw) ? a.fw + (size_t)(sr & ~kSrcFw) * Nc8 : a.h + (size_t)sr * Nc8;
          gp += lbase + lane * VPL;
          if (VPL == 2) cp_async16(&st.st[r][lane * 2], gp); else cp_async8(&st.st[r][lane], gp);
        }
      }
    }
    cp_async_commit();
  };
  // mu*(fEq - 0.5*f) of the node in a stage (solver.F90:206-207), computed one step ahead
  auto base_of = [&](const typename SM::Stage &st, int q) {
    const int e = lane * VPL + q;
    const double ex = dmul(scx[q], st.mom[1]), ey = dmul(scy[q], st.mom[2]), ez = dmul(scz[q], st.mom[3]);
    const double feq = dmul(wv[q], dadd(st.mom[0], dadd(dadd(ex, ey), ez)));
    return dmul(mu, dsub(feq, dmul(0.5, st.fold[e])));
  };

  double xm1[VPL], xm2[VPL], base[VPL];
#pragma unroll
  for (int q = 0; q < VPL; ++q) { xm1[q] = 0.0; xm2[q] = 0.0; base[q] = 0.0; }
  int labprev = L_GHOST;
  if (active) {
    issue(0);
    cp_async_wait<0>();
    __syncwarp();
    const int m0 = S.meta[wid][0][0];
#pragma unroll
    for (int q = 0; q < VPL; ++q) xm1[q] = (m0 >= 0) ? S.pipe[wid][0].fold[lane * VPL + q] : 0.0;
    labprev = S.meta[wid][0][1] >> 8 & 0xff;
    __syncwarp();
    for (int ui = 1; ui < D; ++ui) issue(ui);
    cp_async_wait<D - 2>();  // position 1 landed
    __syncwarp();
    if (S.meta[wid][1 % D][0] >= 0 && S.meta[wid][1 % D][0] < a.NF) {
#pragma unroll
      for (int q = 0; q < VPL; ++q) base[q] = base_of(S.pipe[wid][1 % D], q);
    }
  }
  __syncthreads();  // tables in shared memory

  const int nsteps = (Nx - 1) + (TV - 1) + (TW - 1);
  for (int t = 0; t < nsteps; ++t) {
    const int u = t - pv - pw + 1;
    if (active && u >= 1 && u <= Nx - 1) {
      issue(u + D - 1);
      cp_async_wait<D - 2>();  // positions <= u + 1 landed
      __syncwarp();
      const int slot = u % D;
      const typename SM::Stage &st = S.pipe[wid][slot];
      const int m = S.meta[wid][slot][0];
      const int fl = S.meta[wid][slot][1];
      double out[VPL];
      if (m >= 0 && m < a.NF) {
        const bool fx = (u == 1) || (c_face[labprev] & xbit);
        const bool fy = fl & 1, fz = fl & 2;
        const int cls = (fx ? 1 : 0) | (fy ? 2 : 0) | (fz ? 4 : 0);
#pragma unroll
        for (int q = 0; q < VPL; ++q) {
          const int e = lane * VPL + q;
          double num = dadd(base[q], dmul(fx ? px1[q] : px2[q], xm1[q]));
          if (!fx) num = dadd(num, dmul(pxh[q], xm2[q]));
          const double y1 = (fl & 4) ? S.ring[(t + 2) % 3][wid - 1][e] : st.st[0][e];
          num = dadd(num, dmul(fy ? py1[q] : py2[q], y1));
          if (!fy) {
            const double y2 = (fl & 8) ? S.ring[(t + 1) % 3][wid - 2][e] : st.st[1][e];
            num = dadd(num, dmul(pyh[q], y2));
          }
          const double z1 = (fl & 16) ? S.ring[(t + 2) % 3][wid - TV][e] : st.st[2][e];
          num = dadd(num, dmul(fz ? pz1[q] : pz2[q], z1));
          if (!fz) {
            const double z2 = (fl & 32) ? S.ring[(t + 1) % 3][wid - 2 * TV][e] : st.st[3][e];
            num = dadd(num, dmul(pzh[q], z2));
          }
          out[q] = markstein_div(num, S.Dn[cls][e], S.Rc[cls][e]);
          S.ring[t % 3][wid][e] = out[q];
        }
        if (lane_ok) {
          double *hp = a.h + hidx(m, o, Nc8, lbase + lane * VPL);
          if (VPL == 2) *reinterpret_cast<double2 *>(hp) = make_double2(out[0], out[VPL - 1]);
          else hp[0] = out[0];
        }
      } else {
        // solid node read by the solver: x readers see its slot o unswitched; others 0
#pragma unroll
        for (int q = 0; q < VPL; ++q) out[q] = (m >= 0) ? st.fold[lane * VPL + q] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < VPL; ++q) { xm2[q] = xm1[q]; xm1[q] = out[q]; }
      labprev = fl >> 8 & 0xff;
      // next position's base while this step's results drain
      if (u + 1 <= Nx - 1) {
        const int sn = (u + 1) % D;
        const int mn = S.meta[wid][sn][0];
        if (mn >= 0 && mn < a.NF) {
#pragma unroll
          for (int q = 0; q < VPL; ++q) base[q] = base_of(S.pipe[wid][sn], q);
        }
      }
      __syncwarp();
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

template <int TV, int TW, int VPL, int D>
size_t sweep_smem_bytes() { return sizeof(SweepSmem<TV, TW, VPL, D>); }

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

int sweep_num_diagonals(const DevState &s) {
  const int ntv = (s.Ny - 1 + kTV - 1) / kTV, ntw = (s.Nz - 1 + kTW - 1) / kTW;
  return ntv + ntw - 1;
}

constexpr int kStages = 4;

void launch_sweep_diagonal(const DevState &s, int diag, cudaStream_t st) {
  const int ntv = (s.Ny - 1 + kTV - 1) / kTV, ntw = (s.Nz - 1 + kTW - 1) / kTW;
  const int blo = diag - (ntw - 1) > 0 ? diag - (ntw - 1) : 0;
  const int bhi = diag < ntv - 1 ? diag : ntv - 1;
  const int ntiles = bhi - blo + 1;
  if (ntiles <= 0) return;
  static unsigned long long configured = 0;  // one bit per device
  const size_t sm2 = sweep_smem_bytes<kTV, kTW, 2, kStages>();
  const size_t sm1 = sweep_smem_bytes<kTV, kTW, 1, kStages>();
  int dev = 0;
  cudaGetDevice(&dev);
  if (!(configured >> (dev & 63) & 1ull)) {
    cudaFuncSetAttribute(k_sweep<kTV, kTW, 2, kStages>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
    cudaFuncSetAttribute(k_sweep<kTV, kTW, 1, kStages>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
    configured |= 1ull << (dev & 63);
  }
  if (s.vpl == 2)
    k_sweep<kTV, kTW, 2, kStages><<<ntiles * 8 * s.nchunk, kTV * kTW * 32, sm2, st>>>(s, diag, ntw);
  else
    k_sweep<kTV, kTW, 1, kStages><<<ntiles * 8 * s.nchunk, kTV * kTW * 32, sm1, st>>>(s, diag, ntw);
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
