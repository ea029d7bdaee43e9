// Per-task arithmetic of the octant sweep (solver.F90:205-214), shared by the tile-diagonal
// and the column-march sweep kernels so that both evaluate every value with the same
// operations: FP64 through __dmul_rn / __dadd_rn / __dsub_rn in the reference's order and
// a Markstein-corrected division (bit-identical to the reference's quotient), FP32 with a
// tabulated reciprocal.
//
// Shared-memory rows hold V velocities of one (node, octant); a task is served by V/2
// lanes, two velocities per lane (velocities lp and lp + 1).
#pragma once
#include <cuda_runtime.h>

#include "kernels.h"

namespace piks {
namespace sweep {

constexpr int kFwBit = 1 << 30;

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
// RN(num/den) from y = RN(1/den) with Markstein's correction step (see kernels.cu).
__device__ __forceinline__ double markstein_div(double num, double den, double y) {
  const double q0 = __dmul_rn(num, y);
  const double r = __fma_rn(-q0, den, num);
  return __fma_rn(r, y, q0);
}

template <typename T> struct Pair;
template <> struct Pair<double> { using type = double2; };
template <> struct Pair<float> { using type = float2; };

template <typename T> __device__ __forceinline__ const T *state_h(const DevState &a);
template <> __device__ __forceinline__ const double *state_h<double>(const DevState &a) { return a.h; }
template <> __device__ __forceinline__ const float *state_h<float>(const DevState &a) { return a.h32; }
template <typename T> __device__ __forceinline__ const T *state_fw(const DevState &a);
template <> __device__ __forceinline__ const double *state_fw<double>(const DevState &a) { return a.fw; }
template <> __device__ __forceinline__ const float *state_fw<float>(const DevState &a) { return a.fw32; }

// Octant o's negative-velocity axes (0-based octant = the reference's group o + 1).
__device__ __forceinline__ bool neg_x(int o) { return !(o == 0 || o == 3 || o == 4 || o == 7); }
__device__ __forceinline__ bool neg_y(int o) { return !(o == 0 || o == 1 || o == 4 || o == 5); }
__device__ __forceinline__ bool neg_z(int o) { return o >= 4; }

// The 13 per-velocity constants (cx cy cz w and the nine c*C products) of velocities lp and
// lp + 1.
template <typename T>
__device__ __forceinline__ void load_lane_consts(const DevState &a, int lp, T (&K)[13][2]) {
  if constexpr (sizeof(T) == 8) {
    const double2 *vt = a.vtab2 + (size_t)(lp >> 1) * kVtab;
#pragma unroll
    for (int k = 0; k < 13; ++k) { const double2 t = __ldg(vt + k); K[k][0] = t.x; K[k][1] = t.y; }
  } else {
#pragma unroll
    for (int k = 0; k < 13; ++k) {
      K[k][0] = __ldg(a.vtab32 + (size_t)lp * kVtab + k);
      K[k][1] = __ldg(a.vtab32 + (size_t)(lp + 1) * kVtab + k);
    }
  }
}

// The FP32 arithmetic of one velocity with every rounding explicit (no contraction left to
// the compiler), so that all FP32 sweep kernels give the same values:
// base = mu * (w * (rho + c.u) - f_old / 2), c.u = ((sx cx ux + sy cy uy) + sz cz uz).
__device__ __forceinline__ float base32(const double2 m01, const double2 m23, float fo, float cx, float cy, float cz,
                                        float wl, float mu, bool nx_, bool ny_, bool nz_) {
  const float rho = (float)m01.x, ux = (float)m01.y, uy = (float)m23.x, uz = (float)m23.y;
  float cu = __fmul_rn(nx_ ? -cx : cx, ux);
  cu = __fmaf_rn(ny_ ? -cy : cy, uy, cu);
  cu = __fmaf_rn(nz_ ? -cz : cz, uz, cu);
  const float feq = __fmul_rn(wl, __fadd_rn(rho, cu));
  return __fmul_rn(mu, __fmaf_rn(-0.5f, fo, feq));
}
// num + the upwind terms (x1, x2, y1, y2, z1, z2 in that order; the second-order terms only
// where the axis is not first order), times the reciprocal of the denominator.
__device__ __forceinline__ float update32(float num, float vx1, float vx2, float vy1, float vy2, float vz1, float vz2,
                                          float kx1, float kx2, float ky1, float ky2, float kz1, float kz2, bool fx,
                                          bool fy, bool fz, float rcp) {
  num = __fmaf_rn(kx1, vx1, num);
  if (!fx) num = __fmaf_rn(kx2, vx2, num);
  num = __fmaf_rn(ky1, vy1, num);
  if (!fy) num = __fmaf_rn(ky2, vy2, num);
  num = __fmaf_rn(kz1, vz1, num);
  if (!fz) num = __fmaf_rn(kz2, vz2, num);
  return __fmul_rn(num, rcp);
}

// mu * (fEq - f_old / 2) of one velocity with constants Kq (cx cy cz w ...) and the node's
// moments (rho, ux | uy, uz).
template <typename T>
__device__ __forceinline__ T base_value(const DevState &a, const double2 m01, const double2 m23, T fo, const T *Kq,
                                        bool nx_, bool ny_, bool nz_) {
  if constexpr (sizeof(T) == 8) {
    const double rho = m01.x, ux = m01.y, uy = m23.x, uz = m23.y;
    const double cx = Kq[0], cy = Kq[1], cz = Kq[2], wl = Kq[3];
    const double ex = dmul(nx_ ? -cx : cx, ux), ey = dmul(ny_ ? -cy : cy, uy), ez = dmul(nz_ ? -cz : cz, uz);
    const double feq = dmul(wl, dadd(rho, dadd(dadd(ex, ey), ez)));
    return dmul(a.mu, dsub(feq, dmul(0.5, fo)));
  } else {
    return base32(m01, m23, fo, Kq[0], Kq[1], Kq[2], Kq[3], (float)a.mu, nx_, ny_, nz_);
  }
}

// The part of an update that does not depend on this sweep's values, mu * (fEq - f_old / 2),
// replaces f_old in the task's own row (S + own * V, this lane's two velocities).
template <typename T, int V>
__device__ __forceinline__ void base_task(const DevState &a, const double2 m01, const double2 m23, T *S, int own,
                                          int sub, const T (&K)[13][2], bool nx_, bool ny_, bool nz_) {
  using T2 = typename Pair<T>::type;
  T2 *p = reinterpret_cast<T2 *>(S + (size_t)own * V + 2 * sub);
  const T2 fold = *p;
  const T fo[2] = {fold.x, fold.y};
  T base[2];
  if constexpr (sizeof(T) == 8) {
    const double rho = m01.x, ux = m01.y, uy = m23.x, uz = m23.y;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const double cx = K[0][q], cy = K[1][q], cz = K[2][q], wl = K[3][q];
      const double ex = dmul(nx_ ? -cx : cx, ux), ey = dmul(ny_ ? -cy : cy, uy), ez = dmul(nz_ ? -cz : cz, uz);
      const double feq = dmul(wl, dadd(rho, dadd(dadd(ex, ey), ez)));
      base[q] = dmul(a.mu, dsub(feq, dmul(0.5, fo[q])));
    }
  } else {
#pragma unroll
    for (int q = 0; q < 2; ++q)
      base[q] = base32(m01, m23, fo[q], K[0][q], K[1][q], K[2][q], K[3][q], (float)a.mu, nx_, ny_, nz_);
  }
  T2 bv;
  bv.x = base[0];
  bv.y = base[1];
  *p = bv;
}

// The first-order-class tables of the chunk of V velocities from l0 in shared memory,
// written by the V/2 lanes of one task group (lane sub: velocities l0 + 2 sub, + 1):
// ctab[cls * V + l - l0] = reciprocal of the denominator, and for FP64 also
// ctab[(8 + cls) * V + l - l0] = the denominator (class cls = fx | fy << 1 | fz << 2).
template <typename T, int V>
__device__ __forceinline__ void load_class_table(const DevState &a, int l0, int sub, T *ctab) {
#pragma unroll
  for (int cls = 0; cls < 8; ++cls)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int l = l0 + 2 * sub + q;
      if constexpr (sizeof(T) == 8) {
        ctab[cls * V + 2 * sub + q] = a.vtab[(size_t)l * kVtab + 21 + cls];
        ctab[(8 + cls) * V + 2 * sub + q] = a.vtab[(size_t)l * kVtab + 13 + cls];
      } else {
        ctab[cls * V + 2 * sub + q] = a.vtab32[(size_t)l * kVtab + 21 + cls];
      }
    }
}

// The base pass of one task group: base_task for tasks grp, grp + G, ... < ntask, two tasks
// at a time with both tasks' loads before either's stores (their own rows are distinct).
template <typename T, int V, int G>
__device__ __forceinline__ void base_pass(const DevState &a, const double2 *Mom, T *S, int own0, int ntask, int grp,
                                          int sub, const T (&K)[13][2], bool nx_, bool ny_, bool nz_) {
  using T2 = typename Pair<T>::type;
  int t = grp;
  for (; t + G < ntask; t += 2 * G) {
    T2 *p0 = reinterpret_cast<T2 *>(S + (size_t)(own0 + t) * V + 2 * sub);
    T2 *p1 = reinterpret_cast<T2 *>(S + (size_t)(own0 + t + G) * V + 2 * sub);
    const T2 f0 = *p0, f1 = *p1;
    const double2 a0 = Mom[2 * t], b0 = Mom[2 * t + 1], a1 = Mom[2 * (t + G)], b1 = Mom[2 * (t + G) + 1];
    T2 r0, r1;
    if constexpr (sizeof(T) == 8) {
      const T fo0[2] = {f0.x, f0.y}, fo1[2] = {f1.x, f1.y};
      T o0[2], o1[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const T Kq[4] = {K[0][q], K[1][q], K[2][q], K[3][q]};
        o0[q] = base_value<T>(a, a0, b0, fo0[q], Kq, nx_, ny_, nz_);
        o1[q] = base_value<T>(a, a1, b1, fo1[q], Kq, nx_, ny_, nz_);
      }
      r0.x = o0[0]; r0.y = o0[1]; r1.x = o1[0]; r1.y = o1[1];
    } else {
      r0.x = base32(a0, b0, f0.x, K[0][0], K[1][0], K[2][0], K[3][0], (float)a.mu, nx_, ny_, nz_);
      r0.y = base32(a0, b0, f0.y, K[0][1], K[1][1], K[2][1], K[3][1], (float)a.mu, nx_, ny_, nz_);
      r1.x = base32(a1, b1, f1.x, K[0][0], K[1][0], K[2][0], K[3][0], (float)a.mu, nx_, ny_, nz_);
      r1.y = base32(a1, b1, f1.y, K[0][1], K[1][1], K[2][1], K[3][1], (float)a.mu, nx_, ny_, nz_);
    }
    *p0 = r0;
    *p1 = r1;
  }
  if (t < ntask) base_task<T, V>(a, Mom[2 * t], Mom[2 * t + 1], S, own0 + t, sub, K, nx_, ny_, nz_);
}

// One update: the upwind terms read from the slots of record `rec` (x1 | x2 << 16, y..., z...)
// added to the base in the task's own slot in the reference's order, then the division;
// the result replaces the base. The reciprocal (and FP64 denominator) of the task's class
// come from the shared-memory class table when `ctab` is given, else from the global
// per-velocity table.
template <typename T, int V>
__device__ __forceinline__ void update_core(const DevState &a, T *S, const int4 rec, int own, int sub, int lp,
                                            const T (&K)[13][2], const T *ctab, const T (&bs)[2]) {
  using T2 = typename Pair<T>::type;
  const bool fx = (rec.x >> 27) & 1, fy = (rec.x >> 28) & 1, fz = (rec.x >> 29) & 1;
  const int cls = (fx ? 1 : 0) | (fy ? 2 : 0) | (fz ? 4 : 0);
  auto ld = [&](int slot) { return *reinterpret_cast<const T2 *>(S + (size_t)slot * V + 2 * sub); };
  const T2 x1 = ld(rec.y & 0xffff), y1 = ld(rec.z & 0xffff), z1 = ld(rec.w & 0xffff);
  T2 x2{}, y2{}, z2{};
  if (!fx) x2 = ld((unsigned)rec.y >> 16);
  if (!fy) y2 = ld((unsigned)rec.z >> 16);
  if (!fz) z2 = ld((unsigned)rec.w >> 16);
  const T vx1[2] = {x1.x, x1.y}, vx2[2] = {x2.x, x2.y}, vy1[2] = {y1.x, y1.y}, vy2[2] = {y2.x, y2.y},
          vz1[2] = {z1.x, z1.y}, vz2[2] = {z2.x, z2.y};
  T out[2];
  if constexpr (sizeof(T) == 8) {
    double2 dn, rc;
    if (ctab) {
      rc = *reinterpret_cast<const double2 *>(ctab + cls * V + 2 * sub);
      dn = *reinterpret_cast<const double2 *>(ctab + (8 + cls) * V + 2 * sub);
    } else {
      dn = __ldg(a.vtab2 + (size_t)(lp >> 1) * kVtab + 13 + cls);
      rc = __ldg(a.vtab2 + (size_t)(lp >> 1) * kVtab + 21 + cls);
    }
    const double den[2] = {dn.x, dn.y}, rcp[2] = {rc.x, rc.y};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      double num = bs[q];
      num = dadd(num, dmul(fx ? K[5][q] : K[4][q], vx1[q]));
      if (!fx) num = dadd(num, dmul(K[6][q], vx2[q]));
      num = dadd(num, dmul(fy ? K[8][q] : K[7][q], vy1[q]));
      if (!fy) num = dadd(num, dmul(K[9][q], vy2[q]));
      num = dadd(num, dmul(fz ? K[11][q] : K[10][q], vz1[q]));
      if (!fz) num = dadd(num, dmul(K[12][q], vz2[q]));
      out[q] = markstein_div(num, den[q], rcp[q]);
    }
  } else {
    float rc2[2];
    if (ctab) {
      const float2 r = *reinterpret_cast<const float2 *>(ctab + cls * V + 2 * sub);
      rc2[0] = r.x;
      rc2[1] = r.y;
    } else {
      rc2[0] = __ldg(a.vtab32 + (size_t)lp * kVtab + 21 + cls);
      rc2[1] = __ldg(a.vtab32 + (size_t)(lp + 1) * kVtab + 21 + cls);
    }
#pragma unroll
    for (int q = 0; q < 2; ++q)
      out[q] = update32(bs[q], vx1[q], vx2[q], vy1[q], vy2[q], vz1[q], vz2[q], fx ? K[5][q] : K[4][q], K[6][q],
                        fy ? K[8][q] : K[7][q], K[9][q], fz ? K[11][q] : K[10][q], K[12][q], fx, fy, fz, rc2[q]);
  }
  T2 res;
  res.x = out[0];
  res.y = out[1];
  *reinterpret_cast<T2 *>(S + (size_t)own * V + 2 * sub) = res;
}

// The base is read from the own row (written there by base_task).
template <typename T, int V>
__device__ __forceinline__ void update_task(const DevState &a, T *S, const int4 rec, int own, int sub, int lp,
                                            const T (&K)[13][2], const T *ctab = nullptr) {
  using T2 = typename Pair<T>::type;
  const T2 b2 = *reinterpret_cast<const T2 *>(S + (size_t)own * V + 2 * sub);
  const T bs[2] = {b2.x, b2.y};
  update_core<T, V>(a, S, rec, own, sub, lp, K, ctab, bs);
}

// ---- mbarriers and bulk asynchronous copies (shared by the tile and column kernels) ----
// Longest wait on an mbarrier phase or a flag before a kernel gives up and reports (2 s).
constexpr unsigned long long kWaitNs = 2000000000ull;
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_arrive(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void *src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
}  // namespace sweep
}  // namespace piks
