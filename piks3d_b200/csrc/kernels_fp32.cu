// FP32 path of the source iteration: the distribution function, the wall slots, the
// 3-fold corner storage and the ghost planes are stored and swept in FP32; the moments
// (Rho, U), the diffuse-wall densities, the mass flux and the convergence test stay FP64
// (the moments and the flux reuse the FP64 arrays of DevState). The data flow is the one
// of kernels.cu (same tasks, roles, commits, wall programs and boundary order); only the
// arithmetic type differs, so the FP32 iterate approximates the FP64 one.
#include <cuda_runtime.h>

#include "kernels.h"
#include "piks_internal.h"

namespace piks {

namespace {

__constant__ WProg c32_prog[26];
__constant__ WPlan c32_plan[26];
bool g32_plan_ok = false;  // every program resolved (make_wall_plan)
__constant__ int8_t c32_prog_of[128];
__constant__ int c32_incoming[6][4];

__device__ __forceinline__ size_t hidx(int node, int o, int Nc8, int l) {
  return ((size_t)node * 8 + o) * (size_t)Nc8 + l;
}
__device__ __forceinline__ int plane_slot(int o) { return o >> 1; }
constexpr int kFwBit = 1 << 30;

template <int VPL>
__device__ __forceinline__ void ld32(const float *p, float (&v)[VPL]) {
  if constexpr (VPL == 4) {
    const float4 t = __ldcg(reinterpret_cast<const float4 *>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else if constexpr (VPL == 2) {
    const float2 t = __ldcg(reinterpret_cast<const float2 *>(p));
    v[0] = t.x; v[1] = t.y;
  } else {
    v[0] = __ldcg(p);
  }
}
template <int VPL>
__device__ __forceinline__ void st32(float *p, const float (&v)[VPL]) {
  if constexpr (VPL == 4) *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  else if constexpr (VPL == 2) *reinterpret_cast<float2 *>(p) = make_float2(v[0], v[1]);
  else p[0] = v[0];
}

// Hyperplane sweep task (same task records as the FP64 kernel); upwind rows from h32/fw32.
template <int LPT, int VPL>
__global__ void __launch_bounds__(256)
k_sweep32(const DevState a, long t0, long ntask) {
  const long gl = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long slot = gl / LPT;
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
  auto row = [&](int code, float (&v)[VPL]) {
    const float *base = (code & kFwBit) ? a.fw32 : a.h32;
    ld32<VPL>(base + (size_t)(code & ~kFwBit) * (size_t)Nc8 + lfirst, v);
  };
  float fold[VPL], x1[VPL], x2[VPL], y1[VPL], y2[VPL], z1[VPL], z2[VPL];
  row(m * 8 + o, fold);
  row(r0.z, x1);
  row(r1.x, y1);
  row(r1.z, z1);
  if (!fx) row(r0.w, x2);
  if (!fy) row(r1.y, y2);
  if (!fz) row(r1.w, z2);
  const double2 m01 = __ldg(reinterpret_cast<const double2 *>(a.mom) + 2 * (size_t)m);
  const double2 m23 = __ldg(reinterpret_cast<const double2 *>(a.mom) + 2 * (size_t)m + 1);
  const float rho = (float)m01.x, ux = (float)m01.y, uy = (float)m23.x, uz = (float)m23.y;
  const int cls = (fx ? 1 : 0) | (fy ? 2 : 0) | (fz ? 4 : 0);
  const float sxf = (o == 0 || o == 3 || o == 4 || o == 7) ? 1.f : -1.f;
  const float syf = (o == 0 || o == 1 || o == 4 || o == 5) ? 1.f : -1.f;
  const float szf = o < 4 ? 1.f : -1.f;
  const float mu = (float)a.mu;
  float out[VPL];
#pragma unroll
  for (int q = 0; q < VPL; ++q) {
    const float *vt = a.vtab32 + (size_t)(lfirst + q) * kVtab;
    const float cx = __ldg(vt + 0), cy = __ldg(vt + 1), cz = __ldg(vt + 2), wl = __ldg(vt + 3);
    const float feq = wl * (rho + (sxf * cx * ux + syf * cy * uy + szf * cz * uz));
    float num = mu * (feq - 0.5f * fold[q]);
    num += __ldg(vt + (fx ? 5 : 4)) * x1[q];
    if (!fx) num += __ldg(vt + 6) * x2[q];
    num += __ldg(vt + (fy ? 8 : 7)) * y1[q];
    if (!fy) num += __ldg(vt + 9) * y2[q];
    num += __ldg(vt + (fz ? 11 : 10)) * z1[q];
    if (!fz) num += __ldg(vt + 12) * z2[q];
    out[q] = num * __ldg(vt + 21 + cls);
  }
  st32<VPL>(a.h32 + ((size_t)m * 8 + o) * (size_t)Nc8 + lfirst, out);
}

__global__ void k_commit32(const DevState a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)a.ncommit * a.Nc8) return;
  const int e = (int)(idx / a.Nc8), l = (int)(idx % a.Nc8);
  const int node = a.commit[3 * e], o = a.commit[3 * e + 1], src = a.commit[3 * e + 2];
  a.h32[hidx(node, o, a.Nc8, l)] = src < 8 ? a.h32[hidx(node, src, a.Nc8, l)]
                                           : a.fw32[hidx(a.bcorner[node - a.NF], o, a.Nc8, l)];
}

__global__ void k_capture32(const DevState a, int buf) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)a.Ny * a.Nz * 4 * a.Nc8) return;
  const int l = (int)(idx % a.Nc8);
  const int q = (int)((idx / a.Nc8) % 4);
  const size_t r = idx / ((size_t)a.Nc8 * 4);
  const int oW = q == 0 ? 0 : q == 1 ? 3 : q == 2 ? 4 : 7;
  const int oE = q == 0 ? 1 : q == 1 ? 2 : q == 2 ? 5 : 6;
  const int nW = a.plane_xN[r], nE = a.plane_x1[r];
  a.ghostW32[buf][idx] = nW >= 0 ? a.h32[hidx(nW, oW, a.Nc8, l)] : 0.f;
  a.ghostE32[buf][idx] = nE >= 0 ? a.h32[hidx(nE, oE, a.Nc8, l)] : 0.f;
}

// Walls: extrapolation and re-emission in FP32, the wall densities summed in FP64 (a warp
// reduction) and the re-emitted value formed in FP64 before rounding.
template <int VPL, int LANES>
__global__ void __launch_bounds__(256) k_walls32(const DevState a, int begin, int end, int gbuf) {
  // LANES lanes per wall (32 / LANES walls per warp), VPL velocities per lane
  const int widx = begin + (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) / LANES);
  if (widx >= end) return;
  const int lane = threadIdx.x % LANES;
  const unsigned seg = LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << (threadIdx.x & 31 & ~(LANES - 1)));
  const int q = a.wall_order[widx];
  const int node = a.wall_node[q];
  const int corner = a.wall_corner[q];
  const WProg &P = c32_prog[c32_prog_of[a.wall_label[q]]];
  const float e1 = (float)a.wall_e[2 * q], e2 = (float)a.wall_e[2 * q + 1];
  const int Nc8 = a.Nc8;
  const int *nb = a.wall_nb + 6 * q;
  const int nface = P.nface;
  const int chunkw = LANES * VPL;
  auto far_ptr = [&](int code, int oo, int lf) -> const float * {
    if (e2 == 0.f) return nullptr;  // as in k_walls32_onchip
    if (code >= 0) return a.h32 + hidx(code, oo, Nc8, lf);
    if (code == -1) return nullptr;
    const int cc = -code - 2;
    const float *plane = (cc & 1) ? a.ghostE32[gbuf] : a.ghostW32[gbuf];
    return plane + ((size_t)(cc >> 1) * 4 + plane_slot(oo)) * Nc8 + lf;
  };
  double rho0 = 0.0, rho1 = 0.0, rho2 = 0.0;
  for (int fi = 0; fi < nface; ++fi) {
    const int dir = P.face[fi].dir, st = P.face[fi].store;
    const int n1 = nb[2 * fi], code = nb[2 * fi + 1];
    double racc = 0.0;
    for (int l0 = 0; l0 < Nc8; l0 += chunkw) {
      const int lf = l0 + lane * VPL;
      const bool lv = lf < Nc8;
      float ext[4][VPL];
#pragma unroll
      for (int mm = 0; mm < 4; ++mm) {
        const int oo = c32_incoming[dir][mm] - 1;
        float nv[VPL], fv[VPL];
#pragma unroll
        for (int v = 0; v < VPL; ++v) { nv[v] = 0.f; fv[v] = 0.f; }
        if (lv) {
          ld32<VPL>(a.h32 + hidx(n1, oo, Nc8, lf), nv);
          const float *fp = far_ptr(code, oo, lf);
          if (fp) ld32<VPL>(fp, fv);
        }
#pragma unroll
        for (int v = 0; v < VPL; ++v) ext[mm][v] = e1 * nv[v] + e2 * fv[v];
        if (lv) {
          if (st == ST_F) st32<VPL>(a.h32 + hidx(node, oo, Nc8, lf), ext[mm]);
          else if (st == ST_W) st32<VPL>(a.fw32 + hidx(corner, oo, Nc8, lf), ext[mm]);
        }
      }
      double tface[VPL];
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int l = lf + v;
        const double ca = !lv ? 0.0 : dir < 2 ? __ldg(a.cx + l) : dir < 4 ? __ldg(a.cy + l) : __ldg(a.cz + l);
        tface[v] = ca * (((double)ext[0][v] + (double)ext[1][v]) + (double)ext[2][v] + (double)ext[3][v]);
      }
#pragma unroll
      for (int v = 0; v < VPL; ++v) racc += tface[v];
    }
    // warp sum in FP64 (the FP32 path does not keep the reference's summation order)
    for (int off = LANES / 2; off > 0; off >>= 1) racc += __shfl_xor_sync(seg, racc, off, LANES);
    if (fi == 0) rho0 = racc; else if (fi == 1) rho1 = racc; else rho2 = racc;
  }
  rho0 /= a.DiffFlux; rho1 /= a.DiffFlux; rho2 /= a.DiffFlux;
  const double one_m = 1.0 - a.accom;
  int zface = -1;
  for (int fi = 0; fi < nface; ++fi) if (P.face[fi].store == ST_Z) zface = fi;
  for (int l0 = 0; l0 < Nc8; l0 += chunkw) {
    const int lf = l0 + lane * VPL;
    if (lf >= Nc8) continue;
    // re-emission in groups of four writes: the sources of a group are loaded before its
    // stores (no write of a wall program reads a slot that an earlier write stores)
    for (int r0 = 0; r0 < P.nwr; r0 += 4) {
      float src[4][VPL];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (r0 + k >= P.nwr) break;
        const WWrite &W = P.wr[r0 + k];
        const int so = W.src_o - 1;
        if (W.src_store == ST_F) ld32<VPL>(a.h32 + hidx(node, so, Nc8, lf), src[k]);
        else if (W.src_store == ST_W) ld32<VPL>(a.fw32 + hidx(corner, so, Nc8, lf), src[k]);
        else {
          float nv[VPL], fv[VPL];
          ld32<VPL>(a.h32 + hidx(nb[2 * zface], so, Nc8, lf), nv);
#pragma unroll
          for (int v = 0; v < VPL; ++v) fv[v] = 0.f;
          const float *fp = far_ptr(nb[2 * zface + 1], so, lf);
          if (fp) ld32<VPL>(fp, fv);
#pragma unroll
          for (int v = 0; v < VPL; ++v) src[k][v] = e1 * nv[v] + e2 * fv[v];
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (r0 + k >= P.nwr) break;
        const WWrite &W = P.wr[r0 + k];
        const int dso = W.dst_o - 1;
        const double rf = W.face == 0 ? rho0 : W.face == 1 ? rho1 : rho2;
        float val[VPL];
#pragma unroll
        for (int v = 0; v < VPL; ++v)
          val[v] = (float)(a.accom * __ldg(a.w + lf + v) * rf + one_m * (double)src[k][v]);
        if (W.dst_store == ST_F) st32<VPL>(a.h32 + hidx(node, dso, Nc8, lf), val);
        else st32<VPL>(a.fw32 + hidx(corner, dso, Nc8, lf), val);
      }
    }
  }
}

// The FP32 diffuse wall for octants of at most LANES * VPL velocities (one pass of the
// lane segment), with the extrapolated face values kept in shared memory (12 * Nc8 floats
// per wall): the re-emission reads them there (WPlan) instead of re-loading the slots,
// and a face value is stored only where it is the slot's final content.
template <int VPL, int LANES>
__global__ void __launch_bounds__(256, 3) k_walls32_onchip(const DevState a, int begin, int end, int gbuf) {
  extern __shared__ __align__(16) float wall32_sm[];
  const int wib = threadIdx.x / LANES;
  const int widx = begin + (int)blockIdx.x * (256 / LANES) + wib;
  if (widx >= end) return;  // whole segment
  const int lane = threadIdx.x % LANES;
  const unsigned seg = LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << (threadIdx.x & 31 & ~(LANES - 1)));
  const int Nc8 = a.Nc8;
  float *E = wall32_sm + (size_t)wib * 12 * Nc8;
  const int4 *rp = a.wall_rec + (size_t)widx * 4;
  const int4 r0 = __ldg(rp);
  const double2 ee = __ldg(reinterpret_cast<const double2 *>(rp + 1));
  const int node = r0.x;
  const int corner = r0.y;
  const WPlan &P = c32_plan[c32_prog_of[r0.z]];
  const float e1 = (float)ee.x, e2 = (float)ee.y;
  const int nface = P.nface;
  const int lf = lane * VPL;
  const bool lv = lf < Nc8;
  // the second extrapolation point only matters when its coefficient does (wallExtOrder 1
  // makes it 0: the FP32 path, exact to its tolerance and not to the bit, skips the load)
  auto far_ptr = [&](int code, int oo) -> const float * {
    if (e2 == 0.f) return nullptr;
    if (code >= 0) return a.h32 + hidx(code, oo, Nc8, lf);
    if (code == -1) return nullptr;
    const int cc = -code - 2;
    const float *plane = (cc & 1) ? a.ghostE32[gbuf] : a.ghostW32[gbuf];
    return plane + ((size_t)(cc >> 1) * 4 + plane_slot(oo)) * Nc8 + lf;
  };
  double rho0 = 0.0, rho1 = 0.0, rho2 = 0.0;
  for (int fi = 0; fi < nface; ++fi) {
    const int dir = P.dir[fi], st = P.store[fi], keep = P.keep[fi];
    // the face's (neighbour, far point) pair from the record's second half (the same
    // 128-byte line as its first, so an L1 hit after the loads above)
    const int2 nbp = __ldg(reinterpret_cast<const int2 *>(rp + 2) + fi);
    const int n1 = nbp.x, code = nbp.y;
    double racc = 0.0;
    if (lv) {
      float nv[4][VPL], fv[4][VPL];
#pragma unroll
      for (int mm = 0; mm < 4; ++mm) {
        const int oo = c32_incoming[dir][mm] - 1;
#pragma unroll
        for (int v = 0; v < VPL; ++v) fv[mm][v] = 0.f;
        ld32<VPL>(a.h32 + hidx(n1, oo, Nc8, lf), nv[mm]);
        const float *fp = far_ptr(code, oo);
        if (fp) ld32<VPL>(fp, fv[mm]);
      }
      float ext[4][VPL];
#pragma unroll
      for (int mm = 0; mm < 4; ++mm) {
        const int oo = c32_incoming[dir][mm] - 1;
#pragma unroll
        for (int v = 0; v < VPL; ++v) ext[mm][v] = e1 * nv[mm][v] + e2 * fv[mm][v];
        st32<VPL>(E + (size_t)(fi * 4 + mm) * Nc8 + lf, ext[mm]);
        if (keep >> mm & 1) {
          if (st == ST_F) st32<VPL>(a.h32 + hidx(node, oo, Nc8, lf), ext[mm]);
          else st32<VPL>(a.fw32 + hidx(corner, oo, Nc8, lf), ext[mm]);
        }
      }
      // the four octants of a velocity summed in FP32 (one conversion per velocity rather
      // than four; FP64 ops and conversions are the kernel's short-scoreboard stalls), the
      // velocities and lanes in FP64
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int l = lf + v;
        const double ca = dir < 2 ? __ldg(a.cx + l) : dir < 4 ? __ldg(a.cy + l) : __ldg(a.cz + l);
        racc += ca * (double)__fadd_rn(__fadd_rn(__fadd_rn(ext[0][v], ext[1][v]), ext[2][v]), ext[3][v]);
      }
    }
    // segment sum in FP64 (the FP32 path does not keep the reference's summation order)
    for (int off = LANES / 2; off > 0; off >>= 1) racc += __shfl_xor_sync(seg, racc, off, LANES);
    if (fi == 0) rho0 = racc; else if (fi == 1) rho1 = racc; else rho2 = racc;
  }
  if (!lv) return;
  // re-emission in FP32: accom * rho_face rounded once per face, then w * that + (1 - accom)
  // * the extrapolated value, with the weights rounded to FP32 (vtab32 column 3)
  const float af[3] = {(float)(a.accom * (rho0 / a.DiffFlux)), (float)(a.accom * (rho1 / a.DiffFlux)),
                       (float)(a.accom * (rho2 / a.DiffFlux))};
  const float one_m = (float)(1.0 - a.accom);
  float wl[VPL];
#pragma unroll
  for (int v = 0; v < VPL; ++v) wl[v] = __ldg(a.vtab32 + (size_t)(lf + v) * kVtab + 3);
  for (int k = 0; k < P.nwr; ++k) {
    const float *sp = E + (size_t)P.src[k] * Nc8 + lf;
    const float rf = P.face[k] == 0 ? af[0] : P.face[k] == 1 ? af[1] : af[2];
    float val[VPL];
#pragma unroll
    for (int v = 0; v < VPL; ++v) val[v] = __fmaf_rn(rf, wl[v], __fmul_rn(one_m, sp[v]));
    if (P.dst_store[k] == ST_F) st32<VPL>(a.h32 + hidx(node, P.dst_o[k], Nc8, lf), val);
    else st32<VPL>(a.fw32 + hidx(corner, P.dst_o[k], Nc8, lf), val);
  }
}

__global__ void k_inlet_outlet32(const DevState a, int gbuf) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)a.Ny * a.Nz * 4 * a.Nc8) return;
  const int l = (int)(idx % a.Nc8);
  const int q = (int)((idx / a.Nc8) % 4);
  const size_t r = idx / ((size_t)a.Nc8 * 4);
  const float wdp = (float)(a.w[l] * a.pressDrop);
  const int n1 = a.plane_x1[r], nN = a.plane_xN[r];
  if (n1 >= 0) a.h32[hidx(n1, q == 0 ? 0 : q == 1 ? 3 : q == 2 ? 4 : 7, a.Nc8, l)] = a.ghostW32[gbuf][idx] + wdp;
  if (nN >= 0) a.h32[hidx(nN, q == 0 ? 1 : q == 1 ? 2 : q == 2 ? 5 : 6, a.Nc8, l)] = a.ghostE32[gbuf][idx] - wdp;
}

__global__ void k_symmetry32(const DevState a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)a.nsym * a.Nc8) return;
  const int s = (int)(idx / a.Nc8), l = (int)(idx % a.Nc8);
  const uint8_t f = a.sym_flag[s];
  float *hp = a.h32 + (size_t)a.sym_node[s] * 8 * a.Nc8 + l;
  const size_t S = a.Nc8;
  if (f & 1) { hp[1 * S] = hp[2 * S]; hp[0 * S] = hp[3 * S]; hp[5 * S] = hp[6 * S]; hp[4 * S] = hp[7 * S]; }
  if (f & 2) { hp[2 * S] = hp[1 * S]; hp[3 * S] = hp[0 * S]; hp[6 * S] = hp[5 * S]; hp[7 * S] = hp[4 * S]; }
  if (f & 4) { hp[0 * S] = hp[4 * S]; hp[1 * S] = hp[5 * S]; hp[2 * S] = hp[6 * S]; hp[3 * S] = hp[7 * S]; }
  if (f & 8) { hp[4 * S] = hp[0 * S]; hp[5 * S] = hp[1 * S]; hp[6 * S] = hp[2 * S]; hp[7 * S] = hp[3 * S]; }
}

// Moments in FP64 from FP32 values: LANES lanes per node (32 / LANES nodes per warp), VPL
// velocities per lane, partial sums combined with a segment reduction (the FP32 path does
// not follow the reference's order). A whole warp per node measured fastest for 512
// velocities (half a warp with 16-byte rows: 0.40 vs 0.37 ms on a 128^3 pack).
template <int VPL, int LANES>
__global__ void __launch_bounds__(256) k_moments32(const DevState a) {
  const int node = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) / LANES);
  if (node >= a.NF) return;  // whole segment
  const int lane = threadIdx.x % LANES;
  const unsigned seg = LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << (threadIdx.x & 31 & ~(LANES - 1)));
  const int Nc8 = a.Nc8;
  const float *hp = a.h32 + (size_t)node * 8 * Nc8;
  double r = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
  for (int l0 = lane * VPL; l0 < Nc8; l0 += LANES * VPL) {
    float f[8][VPL];
#pragma unroll
    for (int o = 0; o < 8; ++o) {
      if constexpr (VPL == 2) {
        const float2 t = __ldcs(reinterpret_cast<const float2 *>(hp + (size_t)o * Nc8 + l0));
        f[o][0] = t.x; f[o][VPL - 1] = t.y;
      } else {
        f[o][0] = __ldcs(hp + (size_t)o * Nc8 + l0);
      }
    }
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
      const int l = l0 + v;
      const double f1 = f[0][v], f2 = f[1][v], f3 = f[2][v], f4 = f[3][v], f5 = f[4][v], f6 = f[5][v],
                   f7 = f[6][v], f8 = f[7][v];
      r += ((f1 + f2) + (f3 + f4)) + ((f5 + f6) + (f7 + f8));
      ux += __ldg(a.cx + l) * (((f1 - f2) + (f4 - f3)) + ((f5 - f6) + (f8 - f7)));
      uy += __ldg(a.cy + l) * (((f1 + f2) - (f3 + f4)) + ((f5 + f6) - (f7 + f8)));
      uz += __ldg(a.cz + l) * (((f1 + f2) + (f3 + f4)) - ((f5 + f6) + (f7 + f8)));
    }
  }
  for (int off = LANES / 2; off > 0; off >>= 1) {
    r += __shfl_down_sync(seg, r, off, LANES);
    ux += __shfl_down_sync(seg, ux, off, LANES);
    uy += __shfl_down_sync(seg, uy, off, LANES);
    uz += __shfl_down_sync(seg, uz, off, LANES);
  }
  if (lane == 0) {
    double2 *mp = reinterpret_cast<double2 *>(a.mom) + 2 * (size_t)node;
    mp[0] = make_double2(r, ux);
    mp[1] = make_double2(uy, uz);
  }
}

// The same sums for 64 velocities per octant, a warp over two nodes at a time: the sixteen
// row loads of both nodes are in flight together (each node's sums as in k_moments32).
__global__ void __launch_bounds__(256) k_moments32_pair(const DevState a) {
  const int node0 = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 2;
  if (node0 >= a.NF) return;  // whole warp
  const int lane = threadIdx.x & 31;
  const int l0 = lane * 2;
  const bool two = node0 + 1 < a.NF;
  float f[2][8][2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const float *hp = a.h32 + (size_t)(two ? node0 + k : node0) * 8 * 64;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
      const float2 t = __ldcs(reinterpret_cast<const float2 *>(hp + (size_t)o * 64 + l0));
      f[k][o][0] = t.x; f[k][o][1] = t.y;
    }
  }
  const double cx0 = __ldg(a.cx + l0), cx1 = __ldg(a.cx + l0 + 1), cy0 = __ldg(a.cy + l0), cy1 = __ldg(a.cy + l0 + 1),
               cz0 = __ldg(a.cz + l0), cz1 = __ldg(a.cz + l0 + 1);
  double acc[2][4];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    double r = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const double f1 = f[k][0][v], f2 = f[k][1][v], f3 = f[k][2][v], f4 = f[k][3][v], f5 = f[k][4][v],
                   f6 = f[k][5][v], f7 = f[k][6][v], f8 = f[k][7][v];
      r += ((f1 + f2) + (f3 + f4)) + ((f5 + f6) + (f7 + f8));
      ux += (v ? cx1 : cx0) * (((f1 - f2) + (f4 - f3)) + ((f5 - f6) + (f8 - f7)));
      uy += (v ? cy1 : cy0) * (((f1 + f2) - (f3 + f4)) + ((f5 + f6) - (f7 + f8)));
      uz += (v ? cz1 : cz0) * (((f1 + f2) + (f3 + f4)) - ((f5 + f6) + (f7 + f8)));
    }
    acc[k][0] = r; acc[k][1] = ux; acc[k][2] = uy; acc[k][3] = uz;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[k][q] += __shfl_down_sync(0xffffffffu, acc[k][q], off);
  if (lane == 0) {
    for (int k = 0; k < (two ? 2 : 1); ++k) {
      double2 *mp = reinterpret_cast<double2 *>(a.mom) + 2 * (size_t)(node0 + k);
      mp[0] = make_double2(acc[k][0], acc[k][1]);
      mp[1] = make_double2(acc[k][2], acc[k][3]);
    }
  }
}

__global__ void k_widen(const float *src, double *dst, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

__global__ void k_narrow(const double *src, float *dst, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

inline unsigned nblocks(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

void upload_tables_fp32() {
  int8_t prog_of[128];
  WProg progs[26];
  int n = 0;
  for (int lab = 0; lab < 128; ++lab) {
    prog_of[lab] = -1;
    const WProg *p = wall_program(lab);
    if (p) { progs[n] = *p; prog_of[lab] = (int8_t)n; ++n; }
  }
  cudaMemcpyToSymbol(c32_prog_of, prog_of, sizeof prog_of);
  cudaMemcpyToSymbol(c32_prog, progs, sizeof progs);
  cudaMemcpyToSymbol(c32_incoming, kIncoming, sizeof(int) * 24);
  WPlan plans[26];
  int ok = n == 26;
  for (int i = 0; i < n; ++i) ok &= make_wall_plan(progs[i], plans[i]) ? 1 : 0;
  g32_plan_ok = ok != 0;
  cudaMemcpyToSymbol(c32_plan, plans, sizeof plans);
}

void launch_sweep_hyperplane32(const DevState &s, long t0, long ntask, cudaStream_t st) {
  if (ntask <= 0) return;
  if (s.lpt == 32) k_sweep32<32, 2><<<nblocks((size_t)ntask * s.nchunk * 32, 256), 256, 0, st>>>(s, t0, ntask);
  else k_sweep32<8, 1><<<nblocks((size_t)ntask * s.nchunk * 8, 256), 256, 0, st>>>(s, t0, ntask);
}
void launch_commit32(const DevState &s, cudaStream_t st) {
  if (s.ncommit && s.Nc8 % 4 == 0) return launch_commit_rows(s, true, st);
  if (s.ncommit) k_commit32<<<nblocks((size_t)s.ncommit * s.Nc8, 256), 256, 0, st>>>(s);
}
void launch_capture32(const DevState &s, int buf, cudaStream_t st) {
  k_capture32<<<nblocks((size_t)s.Ny * s.Nz * 4 * s.Nc8, 256), 256, 0, st>>>(s, buf);
}
void launch_walls32(const DevState &s, int begin, int end, int gbuf, cudaStream_t st) {
  if (end <= begin) return;
  const size_t walls = (size_t)(end - begin);
  if (g32_plan_ok && (s.Nc8 == 64 || s.Nc8 <= 32)) {
    once_per_device(reinterpret_cast<const void *>(k_walls32_onchip<4, 16>), [](int) {
      cudaFuncSetAttribute(k_walls32_onchip<4, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 16 * 12 * 64 * 4);
    });
    const size_t smem_per_wall = (size_t)12 * s.Nc8 * sizeof(float);
    if (s.Nc8 == 64)
      k_walls32_onchip<4, 16><<<nblocks(walls * 16, 256), 256, 16 * smem_per_wall, st>>>(s, begin, end, gbuf);
    else if (s.Nc8 <= 8)
      k_walls32_onchip<1, 8><<<nblocks(walls * 8, 256), 256, 32 * smem_per_wall, st>>>(s, begin, end, gbuf);
    else k_walls32_onchip<1, 32><<<nblocks(walls * 32, 256), 256, 8 * smem_per_wall, st>>>(s, begin, end, gbuf);
    return;
  }
  if (s.Nc8 % 64 == 0) k_walls32<4, 16><<<nblocks(walls * 16, 256), 256, 0, st>>>(s, begin, end, gbuf);
  else if (s.Nc8 == 8) k_walls32<1, 8><<<nblocks(walls * 8, 256), 256, 0, st>>>(s, begin, end, gbuf);
  else k_walls32<1, 32><<<nblocks(walls * 32, 256), 256, 0, st>>>(s, begin, end, gbuf);
}
void launch_inlet_outlet32(const DevState &s, int buf, cudaStream_t st) {
  k_inlet_outlet32<<<nblocks((size_t)s.Ny * s.Nz * 4 * s.Nc8, 256), 256, 0, st>>>(s, buf);
}
void launch_symmetry32(const DevState &s, cudaStream_t st) {
  if (s.nsym) k_symmetry32<<<nblocks((size_t)s.nsym * s.Nc8, 256), 256, 0, st>>>(s);
}
void launch_moments32(const DevState &s, cudaStream_t st) {
  if (!s.NF) return;
  if (s.Nc8 == 64) k_moments32_pair<<<nblocks((size_t)(s.NF + 1) / 2 * 32, 256), 256, 0, st>>>(s);
  else if (s.Nc8 % 2 == 0) k_moments32<2, 32><<<nblocks((size_t)s.NF * 32, 256), 256, 0, st>>>(s);
  else k_moments32<1, 32><<<nblocks((size_t)s.NF * 32, 256), 256, 0, st>>>(s);
}
template <typename T>
__global__ void __launch_bounds__(256) k_gram(const char *base, size_t stride, int n, size_t count, double *partial) {
  constexpr int kMaxD = kMaxSnapSlots - 1, kMaxPairs = kMaxD * (kMaxD + 1) / 2;
  __shared__ double red[256];
  const int nd = n - 1, npair = nd * (nd + 1) / 2;
  double acc[kMaxPairs];
#pragma unroll
  for (int q = 0; q < kMaxPairs; ++q) acc[q] = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    double x[kMaxSnapSlots], u[kMaxD];
#pragma unroll
    for (int j = 0; j < kMaxSnapSlots; ++j)
      x[j] = j < n ? (double)reinterpret_cast<const T *>(base + (size_t)j * stride)[i] : 0.0;
#pragma unroll
    for (int a = 0; a < kMaxD; ++a) u[a] = x[a + 1] - x[a];
    int q = 0;
#pragma unroll
    for (int a = 0; a < kMaxD; ++a)
#pragma unroll
      for (int b = a; b < kMaxD; ++b, ++q)
        if (b < nd) acc[q] += u[a] * u[b];
  }
  // block sums in a fixed tree order, pair by pair (acc is indexed over the kMaxD triangle,
  // the output over the nd triangle)
  int q = 0;
  for (int a = 0; a < nd; ++a)
    for (int b = a; b < nd; ++b, ++q) {
      const int qa = a * kMaxD - a * (a - 1) / 2 + (b - a);
      double v = 0.0;
#pragma unroll
      for (int k = 0; k < kMaxPairs; ++k)
        if (k == qa) v = acc[k];
      red[threadIdx.x] = v;
      __syncthreads();
      for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
      }
      if (threadIdx.x == 0) partial[(size_t)blockIdx.x * npair + q] = red[0];
      __syncthreads();
    }
}
template <typename T>
void gram_any(const T *base, size_t stride, int n, size_t count, double *partial, cudaStream_t st) {
  const int npair = (n - 1) * n / 2;
  if (!count) {
    cudaMemsetAsync(partial, 0, (size_t)kGramBlocks * npair * sizeof(double), st);
    return;
  }
  k_gram<T><<<kGramBlocks, 256, 0, st>>>(reinterpret_cast<const char *>(base), stride, n, count, partial);
}
void launch_gram(const double *base, size_t stride, int n, size_t count, double *partial, cudaStream_t st) {
  gram_any(base, stride, n, count, partial, st);
}
void launch_gram(const float *base, size_t stride, int n, size_t count, double *partial, cudaStream_t st) {
  gram_any(base, stride, n, count, partial, st);
}

struct Coefs { double c[kMaxSnapSlots]; };
template <typename T>
__global__ void k_combine(T *dst, const char *base, size_t stride, int n, Coefs cf, size_t count) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int j = 0; j < n; ++j) v += cf.c[j] * (double)reinterpret_cast<const T *>(base + (size_t)j * stride)[i];
    dst[i] = (T)v;
  }
}
template <typename T>
void combine_any(T *dst, const T *base, size_t stride, int n, const double *coef, size_t count, cudaStream_t st) {
  if (!count) return;
  Coefs cf{};
  for (int j = 0; j < n && j < kMaxSnapSlots; ++j) cf.c[j] = coef[j];
  k_combine<T><<<148 * 16, 256, 0, st>>>(dst, reinterpret_cast<const char *>(base), stride, n, cf, count);
}
void launch_combine(double *dst, const double *base, size_t stride, int n, const double *coef, size_t count,
                    cudaStream_t st) {
  combine_any(dst, base, stride, n, coef, count, st);
}
void launch_combine(float *dst, const float *base, size_t stride, int n, const double *coef, size_t count,
                    cudaStream_t st) {
  combine_any(dst, base, stride, n, coef, count, st);
}
void launch_widen(const float *src, double *dst, size_t n, cudaStream_t st) {
  if (n) k_widen<<<148 * 16, 256, 0, st>>>(src, dst, n);
}
void launch_narrow(const double *src, float *dst, size_t n, cudaStream_t st) {
  if (n) k_narrow<<<148 * 16, 256, 0, st>>>(src, dst, n);
}

}  // namespace piks
