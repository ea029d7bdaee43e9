// Device classification of the preprocessed voxel box (physicalGrid.F90:546-936): labels,
// the node map, the 3-fold corner numbers and the wall list, identical to classify_host.
//
// The box (ghosted (Nx+4)(Ny+4)(Nz+4) bytes after the drill / thin passes, which stay on the
// host because their result depends on the raster order of their in-place updates) is
// uploaded once; then, one thread per voxel:
//  1. k_labels: the wall label of each solid voxel from which face neighbours are fluid;
//  2. k_flags: fluid node, solid node read by the solver (within two cells of a fluid voxel
//     along an axis), wall, 3-fold corner;
//  3. a three-phase exclusive scan over the raster order (per-block counts, block offsets,
//     per-block ranks with warp ballots) numbers the fluid nodes, the read solid nodes (after
//     all fluid nodes), the walls and the corners exactly in the raster order the host uses;
//  4. k_walls: each wall's record (node, label, corner, extrapolation coefficients, face
//     neighbours) at its number.
// The results are copied back into the Geometry, where the host finishes the schedule.
#include <cuda_runtime.h>

#include <vector>

#include "kernels.h"
#include "piks_internal.h"

namespace piks {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;                          // voxels per thread
constexpr int kScanTile = kScanThreads * kScanItems;   // voxels per block
constexpr int kFlags = 4;                              // fluid node, read solid node, wall, corner

struct ClassTables {
  uint8_t face[128];       // fluid-side bits of a label
  int8_t side_label[64];   // label of a solid voxel by fluid sides (-1: plain solid)
  uint8_t nface[128];      // wall program: faces
  uint8_t dir[128][3];     // ... and their directions (DIR_PX ..)
};
__constant__ ClassTables c_ct;

struct BoxDims {
  int Nx, Ny, Nz, GX, GY;
  long long NG;
};

__device__ __forceinline__ void decode(const BoxDims &d, long long v, int &i, int &j, int &k) {
  i = (int)(v % d.GX) - 1;
  j = (int)((v / d.GX) % d.GY) - 1;
  k = (int)(v / ((long long)d.GX * d.GY)) - 1;
}
__device__ __forceinline__ long long gidx(const BoxDims &d, int i, int j, int k) {
  return (long long)(i + 1) + (long long)(j + 1) * d.GX + (long long)(k + 1) * d.GX * d.GY;
}
__device__ __forceinline__ bool real_voxel(const BoxDims &d, int i, int j, int k) {
  return i >= 1 && i <= d.Nx && j >= 1 && j <= d.Ny && k >= 1 && k <= d.Nz;
}

__global__ void k_labels(BoxDims d, const uint8_t *box, uint8_t *label) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= d.NG) return;
  int i, j, k;
  decode(d, v, i, j, k);
  if (!real_voxel(d, i, j, k)) { label[v] = L_GHOST; return; }
  const uint8_t c = box[v];
  int lab = c;
  if (c == L_SOLID) {
    unsigned sides = 0;
    if (box[gidx(d, i + 1, j, k)] == L_FLUID) sides |= FACE_E;
    if (box[gidx(d, i - 1, j, k)] == L_FLUID) sides |= FACE_W;
    if (box[gidx(d, i, j + 1, k)] == L_FLUID) sides |= FACE_N;
    if (box[gidx(d, i, j - 1, k)] == L_FLUID) sides |= FACE_S;
    if (box[gidx(d, i, j, k + 1)] == L_FLUID) sides |= FACE_F;
    if (box[gidx(d, i, j, k - 1)] == L_FLUID) sides |= FACE_B;
    const int t = c_ct.side_label[sides & 63];
    lab = t < 0 ? L_SOLID : t;
  }
  label[v] = (uint8_t)lab;
}

__device__ __forceinline__ bool is_corner3(int lab) { return lab >= 60 && lab <= 73 && (lab % 10) <= 3; }

// bit 0 fluid node, bit 1 read solid node, bit 2 wall, bit 3 3-fold corner
__global__ void k_flags(BoxDims d, const uint8_t *label, uint8_t *flags) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= d.NG) return;
  int i, j, k;
  decode(d, v, i, j, k);
  uint8_t f = 0;
  if (real_voxel(d, i, j, k)) {
    const int lab = label[v];
    if (lab == L_FLUID) {
      f = 1;
    } else {
      bool keep = false;
      for (int q = -2; q <= 2 && !keep; ++q) {
        if (q == 0) continue;
        if (real_voxel(d, i + q, j, k) && label[gidx(d, i + q, j, k)] == L_FLUID) keep = true;
        if (real_voxel(d, i, j + q, k) && label[gidx(d, i, j + q, k)] == L_FLUID) keep = true;
        if (real_voxel(d, i, j, k + q) && label[gidx(d, i, j, k + q)] == L_FLUID) keep = true;
      }
      if (keep) f |= 2;
      if (c_ct.face[lab]) f |= 4;
      if (c_ct.face[lab] && is_corner3(lab)) f |= 8;
    }
  }
  flags[v] = f;
}

// Phase 1: per-block counts of the four flags.
__global__ void __launch_bounds__(kScanThreads) k_scan_count(long long NG, const uint8_t *flags, int *counts) {
  __shared__ int red[kFlags][kScanThreads / 32];
  const long long base = (long long)blockIdx.x * kScanTile;
  int c[kFlags] = {0, 0, 0, 0};
  for (int e = 0; e < kScanItems; ++e) {
    const long long v = base + (long long)e * kScanThreads + threadIdx.x;
    const uint8_t f = v < NG ? flags[v] : 0;
#pragma unroll
    for (int b = 0; b < kFlags; ++b) c[b] += (f >> b) & 1;
  }
#pragma unroll
  for (int b = 0; b < kFlags; ++b) {
    int x = c[b];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if ((threadIdx.x & 31) == 0) red[b][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < kFlags) {
    int t = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) t += red[threadIdx.x][w];
    counts[(size_t)blockIdx.x * kFlags + threadIdx.x] = t;
  }
}

// Phase 2: exclusive offsets of the blocks and the totals (one block; warp w scans flag w
// over the blocks, 32 blocks per step).
__global__ void k_scan_offsets(int nblocks, const int *counts, int *offsets, int *totals) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w >= kFlags) return;
  int acc = 0;
  for (int b0 = 0; b0 < nblocks; b0 += 32) {
    const int b = b0 + lane;
    const int c = b < nblocks ? counts[(size_t)b * kFlags + w] : 0;
    int x = c;
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, off);
      if (lane >= off) x += y;
    }
    if (b < nblocks) offsets[(size_t)b * kFlags + w] = acc + x - c;
    acc += __shfl_sync(0xffffffffu, x, 31);
  }
  if (lane == 0) totals[w] = acc;
}

// Phase 3: each voxel's rank in the raster order for its flags; node map, inverse map, wall
// and corner numbers.
__global__ void __launch_bounds__(kScanThreads)
k_scan_write(BoxDims d, const uint8_t *flags, const int *offsets, const int *totals, int32_t *nodemap,
             int32_t *node_g, int32_t *wall_of, int32_t *corner_of) {
  __shared__ int warp_sum[kFlags][kScanThreads / 32];
  __shared__ int running[kFlags];
  const long long base = (long long)blockIdx.x * kScanTile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x < kFlags) running[threadIdx.x] = offsets[(size_t)blockIdx.x * kFlags + threadIdx.x];
  const int NF = totals[0];
  __syncthreads();
  for (int e = 0; e < kScanItems; ++e) {
    const long long v = base + (long long)e * kScanThreads + threadIdx.x;
    const uint8_t f = v < d.NG ? flags[v] : 0;
    int rank[kFlags];
#pragma unroll
    for (int b = 0; b < kFlags; ++b) {
      const unsigned m = __ballot_sync(0xffffffffu, (f >> b) & 1);
      rank[b] = __popc(m & ((1u << lane) - 1u));
      if (lane == 0) warp_sum[b][warp] = __popc(m);
    }
    __syncthreads();
    int before[kFlags];
#pragma unroll
    for (int b = 0; b < kFlags; ++b) {
      int x = running[b];
      for (int w = 0; w < warp; ++w) x += warp_sum[b][w];
      before[b] = x + rank[b];
    }
    if (v < d.NG) {
      int i, j, k;
      decode(d, v, i, j, k);
      int32_t nm = real_voxel(d, i, j, k) ? -1 : -2;
      if (f & 1) nm = before[0];
      else if (f & 2) nm = NF + before[1];
      nodemap[v] = nm;
      if (nm >= 0) node_g[nm] = (int32_t)v;
      wall_of[v] = (f & 4) ? before[2] : -1;
      corner_of[v] = (f & 8) ? before[3] : -1;
    }
    __syncthreads();
    if (threadIdx.x < kFlags) {
      int t = 0;
      for (int w = 0; w < kScanThreads / 32; ++w) t += warp_sum[threadIdx.x][w];
      running[threadIdx.x] += t;
    }
    __syncthreads();
  }
}

// Wall records at their numbers (classify_host's wall loop, wall_extrapolation,
// wall_neighbours).
__global__ void k_walls(BoxDims d, int ext_order, int NF, const uint8_t *label, const int32_t *nodemap,
                        const int32_t *wall_of, const int32_t *corner_of, int32_t *w_node, int32_t *w_label,
                        int32_t *w_corner, double *w_e, int32_t *w_nb, int32_t *bcorner) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= d.NG) return;
  const int q = wall_of[v];
  if (q < 0) return;
  int i, j, k;
  decode(d, v, i, j, k);
  const int lab = label[v];
  const int node = nodemap[v];
  const int corner = corner_of[v];
  if (node >= NF) bcorner[node - NF] = corner;
  double e1 = 2.0, e2 = -1.0;
  if (ext_order == 1) {
    e1 = 1.0; e2 = 0.0;
  } else if (ext_order != 2) {
    // reference local id and its decode (physicalGrid.F90:895-936), as written there
    const long long NXT = d.Nx + 4, NXYT = (long long)(d.Nx + 4) * (d.Ny + 4);
    const long long localid = (long long)(i + 2) + (long long)(j + 1) * NXT + (long long)(k + 1) * NXYT;
    const int kd = -1 + (int)(localid / NXYT);
    const int jd = -1 + (int)((localid - (long long)(kd + 1) * NXYT) / NXT);
    const int id = -1 + (int)(localid - (long long)(kd + 1) * NXYT - (long long)(jd + 1) * NXT);
    const uint8_t fm = c_ct.face[label[gidx(d, id, jd, kd)]];
    auto LAB = [&](int ii, int jj, int kk) { return (int)label[gidx(d, ii, jj, kk)]; };
    bool first = false;
    if ((fm & FACE_W) && id == 2 && LAB(1, jd, kd) == L_FLUID) first = true;
    if ((fm & FACE_E) && id == d.Nx - 1 && LAB(d.Nx, jd, kd) == L_FLUID) first = true;
    if ((fm & FACE_S) && jd == 2 && LAB(id, 1, kd) == L_FLUID) first = true;
    if ((fm & FACE_N) && jd == d.Ny - 1 && LAB(id, d.Ny, kd) == L_FLUID) first = true;
    if ((fm & FACE_B) && kd == 2 && LAB(id, jd, 1) == L_FLUID) first = true;
    if ((fm & FACE_F) && kd == d.Nz - 1 && LAB(id, jd, d.Nz) == L_FLUID) first = true;
    if (first) { e1 = 1.0; e2 = 0.0; }
  }
  int32_t nb[6] = {-1, -1, -1, -1, -1, -1};
  for (int fi = 0; fi < c_ct.nface[lab]; ++fi) {
    const int dir = c_ct.dir[lab][fi];
    const int dx = dir == DIR_PX ? 1 : dir == DIR_MX ? -1 : 0;
    const int dy = dir == DIR_PY ? 1 : dir == DIR_MY ? -1 : 0;
    const int dz = dir == DIR_PZ ? 1 : dir == DIR_MZ ? -1 : 0;
    nb[2 * fi] = nodemap[gidx(d, i + dx, j + dy, k + dz)];
    const int i2 = i + 2 * dx, j2 = j + 2 * dy, k2 = k + 2 * dz;
    int32_t code;
    if (real_voxel(d, i2, j2, k2)) code = nodemap[gidx(d, i2, j2, k2)];
    else if (i2 == 0 && j2 >= 1 && j2 <= d.Ny && k2 >= 1 && k2 <= d.Nz) code = -(2 + 2 * ((k2 - 1) * d.Ny + (j2 - 1)));
    else if (i2 == d.Nx + 1 && j2 >= 1 && j2 <= d.Ny && k2 >= 1 && k2 <= d.Nz) code = -(3 + 2 * ((k2 - 1) * d.Ny + (j2 - 1)));
    else code = -1;
    nb[2 * fi + 1] = code;
  }
  w_node[q] = node;
  w_label[q] = lab;
  w_corner[q] = corner;
  w_e[2 * (size_t)q] = e1;
  w_e[2 * (size_t)q + 1] = e2;
  for (int t = 0; t < 6; ++t) w_nb[6 * (size_t)q + t] = nb[t];
}

// Device buffers of one classification, freed on every return path.
struct Scratch {
  std::vector<void *> ptrs;
  template <typename T>
  cudaError_t alloc(T **p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, (n ? n : 1) * sizeof(T));
    if (e == cudaSuccess) { ptrs.push_back(q); *p = static_cast<T *>(q); }
    return e;
  }
  ~Scratch() {
    for (void *p : ptrs) cudaFree(p);
  }
};

unsigned blocks_of(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

piks_status classify_device(const Setup &s, const std::vector<uint8_t> &box, Geometry &g, void *stream,
                            std::string &err) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  BoxDims d;
  d.Nx = s.Nx; d.Ny = s.Ny; d.Nz = s.Nz; d.GX = s.Nx + 4; d.GY = s.Ny + 4;
  d.NG = (long long)d.GX * d.GY * (s.Nz + 4);
  if ((long long)box.size() != d.NG) { err = "classify: box size"; return PIKS_ERR_ARG; }
  // label tables from the host definitions
  ClassTables ct{};
  for (int lab = 0; lab < 128; ++lab) {
    ct.face[lab] = face_mask(lab);
    const WProg *P = wall_program(lab);
    ct.nface[lab] = P ? (uint8_t)P->nface : 0;
    for (int f = 0; f < 3; ++f) ct.dir[lab][f] = P && f < P->nface ? (uint8_t)P->face[f].dir : 0;
  }
  for (int sides = 0; sides < 64; ++sides) ct.side_label[sides] = -1;
  for (int lab = 0; lab < 128; ++lab)
    if (is_wall_label(lab)) ct.side_label[face_mask(lab)] = (int8_t)lab;
  auto cuda = [&](cudaError_t e, const char *what) -> bool {
    if (e == cudaSuccess) return true;
    err = std::string("classify: ") + what + ": " + cudaGetErrorString(e);
    return false;
  };
  Scratch sc;
  uint8_t *dbox = nullptr, *dlabel = nullptr, *dflags = nullptr;
  int32_t *dnodemap = nullptr, *dnode_g = nullptr, *dwall_of = nullptr, *dcorner_of = nullptr;
  int *dcounts = nullptr, *doffsets = nullptr, *dtotals = nullptr;
  const unsigned nscan = blocks_of(d.NG, kScanTile);
  if (!cuda(sc.alloc(&dbox, (size_t)d.NG), "alloc") || !cuda(sc.alloc(&dlabel, (size_t)d.NG), "alloc") ||
      !cuda(sc.alloc(&dflags, (size_t)d.NG), "alloc") || !cuda(sc.alloc(&dnodemap, (size_t)d.NG), "alloc") ||
      !cuda(sc.alloc(&dnode_g, (size_t)d.NG), "alloc") || !cuda(sc.alloc(&dwall_of, (size_t)d.NG), "alloc") ||
      !cuda(sc.alloc(&dcorner_of, (size_t)d.NG), "alloc") || !cuda(sc.alloc(&dcounts, (size_t)nscan * kFlags), "alloc") ||
      !cuda(sc.alloc(&doffsets, (size_t)nscan * kFlags), "alloc") || !cuda(sc.alloc(&dtotals, (size_t)kFlags), "alloc"))
    return PIKS_ERR_OOM;
  if (!cuda(cudaMemcpyToSymbolAsync(c_ct, &ct, sizeof ct, 0, cudaMemcpyHostToDevice, st), "tables") ||
      !cuda(cudaMemcpyAsync(dbox, box.data(), (size_t)d.NG, cudaMemcpyHostToDevice, st), "box upload"))
    return PIKS_ERR_CUDA;
  k_labels<<<blocks_of(d.NG, 256), 256, 0, st>>>(d, dbox, dlabel);
  k_flags<<<blocks_of(d.NG, 256), 256, 0, st>>>(d, dlabel, dflags);
  k_scan_count<<<nscan, kScanThreads, 0, st>>>(d.NG, dflags, dcounts);
  k_scan_offsets<<<1, 32 * kFlags, 0, st>>>((int)nscan, dcounts, doffsets, dtotals);
  k_scan_write<<<nscan, kScanThreads, 0, st>>>(d, dflags, doffsets, dtotals, dnodemap, dnode_g, dwall_of, dcorner_of);
  int totals[kFlags] = {0, 0, 0, 0};
  if (!cuda(cudaGetLastError(), "launch") ||
      !cuda(cudaMemcpyAsync(totals, dtotals, sizeof totals, cudaMemcpyDeviceToHost, st), "totals") ||
      !cuda(cudaStreamSynchronize(st), "sync"))
    return PIKS_ERR_CUDA;
  const int NF = totals[0], NB = totals[1], nWall = totals[2], nCorner = totals[3];
  int32_t *w_node = nullptr, *w_label = nullptr, *w_corner = nullptr, *w_nb = nullptr, *dbcorner = nullptr;
  double *w_e = nullptr;
  if (!cuda(sc.alloc(&w_node, (size_t)nWall), "alloc") || !cuda(sc.alloc(&w_label, (size_t)nWall), "alloc") ||
      !cuda(sc.alloc(&w_corner, (size_t)nWall), "alloc") || !cuda(sc.alloc(&w_nb, (size_t)nWall * 6), "alloc") ||
      !cuda(sc.alloc(&w_e, (size_t)nWall * 2), "alloc") || !cuda(sc.alloc(&dbcorner, (size_t)NB), "alloc"))
    return PIKS_ERR_OOM;
  if (!cuda(cudaMemsetAsync(dbcorner, 0xff, (size_t)(NB ? NB : 1) * sizeof(int32_t), st), "memset")) return PIKS_ERR_CUDA;
  k_walls<<<blocks_of(d.NG, 256), 256, 0, st>>>(d, s.p.wallExtOrder, NF, dlabel, dnodemap, dwall_of, dcorner_of, w_node,
                                                  w_label, w_corner, w_e, w_nb, dbcorner);
  g.Nx = s.Nx; g.Ny = s.Ny; g.Nz = s.Nz; g.GX = d.GX; g.GY = d.GY; g.GZ = s.Nz + 4;
  g.xl = 1; g.xu = s.Nx; g.wglob = g.eglob = true;  // one rank: the whole box
  g.NF = NF; g.NB = NB; g.nWall = nWall; g.nCorner = nCorner;
  g.label.resize((size_t)d.NG);
  g.nodemap.resize((size_t)d.NG);
  g.node_g.resize((size_t)NF + NB);
  g.bcorner.resize((size_t)NB);
  g.wall_node.resize((size_t)nWall); g.wall_label.resize((size_t)nWall); g.wall_corner.resize((size_t)nWall);
  g.wall_e.resize((size_t)nWall * 2); g.wall_nb.resize((size_t)nWall * 6);
  auto down = [&](void *dst, const void *src, size_t bytes) {
    return !bytes || cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st), "download");
  };
  if (!cuda(cudaGetLastError(), "launch") || !down(g.label.data(), dlabel, (size_t)d.NG) ||
      !down(g.nodemap.data(), dnodemap, (size_t)d.NG * 4) || !down(g.node_g.data(), dnode_g, g.node_g.size() * 4) ||
      !down(g.bcorner.data(), dbcorner, g.bcorner.size() * 4) || !down(g.wall_node.data(), w_node, (size_t)nWall * 4) ||
      !down(g.wall_label.data(), w_label, (size_t)nWall * 4) || !down(g.wall_corner.data(), w_corner, (size_t)nWall * 4) ||
      !down(g.wall_e.data(), w_e, (size_t)nWall * 16) || !down(g.wall_nb.data(), w_nb, (size_t)nWall * 24) ||
      !cuda(cudaStreamSynchronize(st), "sync"))
    return PIKS_ERR_CUDA;
  return PIKS_OK;
}

}  // namespace piks
