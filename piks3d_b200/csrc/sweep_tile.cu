// Tile-wavefront octant sweep (solver.F90:176-526) over the TileJobs schedule.
//
// One CTA runs one job (a tile of the box for one octant) for one chunk of V velocities:
//  1. it copies every row the job touches (its own rows, the upwind rows of neighbouring
//     tiles, the wall rows seen by its readers) into shared memory with cp.async, V
//     velocities (one 128-byte segment for V*sizeof(T) = 128) per row;
//  2. it replaces each own row by the part of its update that depends only on the previous
//     iteration (mu * (fEq - f_old / 2)), for all tasks at once;
//  3. it sweeps the tile's local hyperplanes in order, a group of V/2 lanes per task with
//     two velocities per lane, adding the upwind terms read from shared memory in the
//     reference's order and writing the new value to the task's own slot (one barrier per
//     non-empty hyperplane);
//  4. it writes the own rows back.
// Jobs of one diagonal run in one launch; rows a job reads from another tile were written
// by an earlier launch. Each update applies the same operations to the same operands as
// the per-node FP64 kernel, so the FP64 result is unchanged by the schedule.
#include <cuda_runtime.h>

#include "kernels.h"
#include "sweep_core.cuh"

namespace piks {

namespace {

using namespace sweep;

// Task groups per CTA (tasks of one local hyperplane in flight): FP64 CTAs of 64 threads
// (8 groups of 8 lanes for 16 velocities), FP32 6 groups of 16 lanes (32 velocities).
// Measured on B200 (128^3 pack, 512 velocities, sweep per iteration): FP64 with 8x4x4 tiles
// and two chunks per CTA 4 / 6 / 8 / 12 / 16 groups 6.15 / 5.84 / 5.42 / 5.41 / 5.77 ms
// (4x4x4 tiles: 5.32 / 5.63 / 5.46 / 6.19 / 7.01); FP32 4 groups 2.76 ms, 6: 2.69, 8: 2.74,
// 12: 3.39.
template <typename T, int V> constexpr int groups_of() { return sizeof(T) == 8 ? 64 / (V / 2) : 6; }
template <typename T, int V> constexpr int threads_of() { return V / 2 * groups_of<T, V>(); }

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Shared-memory layout of one CTA: [slots][V] rows, the job's task records (int4), the
// moments of each task's node (two double2), the row codes (int32) and the step offsets.
__host__ __device__ inline size_t tile_smem_bytes(int slots, int ntask, int steps_stride, int row_bytes) {
  return (size_t)slots * row_bytes + (size_t)ntask * 48 + ((size_t)slots * 4 + 15) / 16 * 16 +
         (size_t)steps_stride * 2;
}

// Synchronisation of the threads sweeping one job: the whole CTA (bar 0) or the half of a
// pair CTA (named barrier `bar` of N threads).
// The barrier number is a compile-time constant (a register operand would make the kernel
// reserve every hardware barrier and cut its residency); pairs exist only for teams of
// whole warps.
template <int N, int BAR>
__device__ __forceinline__ void team_sync() {
  if constexpr (BAR == 0 || N % 32 != 0) __syncthreads();
  else asm volatile("bar.sync %0, %1;" ::"n"(BAR), "n"(N) : "memory");
}
template <int N, int BAR>
__device__ __forceinline__ bool team_or(bool v) {
  if constexpr (BAR == 0 || N % 32 != 0) {
    return __syncthreads_or(v) != 0;
  } else {
    unsigned r;
    asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
                 : "=r"(r)
                 : "r"((unsigned)v), "n"(BAR), "n"(N)
                 : "memory");
    return r != 0;
  }
}

// One job (tile, octant) for the velocity chunks chunk0 .. chunk0 + nch - 1, by one team
// (thread `tid` of THREADS, synchronised through `bar`): the job's row codes, task records,
// steps and moments are staged once, then each chunk's rows are staged, swept and written
// back in turn.
// With `meta_bar` (an mbarrier in shared memory, initialised, phase 0) the three contiguous
// metadata arrays arrive by bulk asynchronous copies issued by one thread; without it (the
// persistent kernels, which run many jobs per CTA) every thread copies 16-byte pieces.
template <typename T, int V, int NCH = 1, int BAR = 0>
__device__ __forceinline__ void tile_job(const DevState &a, int job, int chunk0, int slots_cap, int tasks_cap,
                                         unsigned char *smem_raw, unsigned long long *meta_bar = nullptr,
                                         int tid = (int)threadIdx.x) {
  constexpr int LPT = V / 2;                        // lanes per task
  constexpr int THREADS = LPT * groups_of<T, V>();
  constexpr int GROUPS = groups_of<T, V>();            // tasks in flight per pass
  constexpr int EPP = 16 / (int)sizeof(T);          // elements per 16-byte piece
  constexpr int PIECES = V / EPP;                   // pieces per row
  using T2 = typename Pair<T>::type;
  T *S = reinterpret_cast<T *>(smem_raw);

  const TileView &tv = a.tv;
  const int Nc8 = a.Nc8;
  const int64_t rb = tv.row_begin[job];
  const int nrows = tv.row_count[job];
  const int64_t tb = tv.task_begin[job];
  const int ntask = (int)(tv.task_begin[job + 1] - tb);
  const int nsteps = tv.nsteps;
  int4 *Trec = reinterpret_cast<int4 *>(smem_raw + (size_t)slots_cap * V * sizeof(T));
  double2 *Mom = reinterpret_cast<double2 *>(Trec + tasks_cap);
  int *Codes = reinterpret_cast<int *>(Mom + 2 * (size_t)tasks_cap);
  uint16_t *Steps = reinterpret_cast<uint16_t *>(Codes + ((size_t)slots_cap + 3) / 4 * 4);
  const T *h = state_h<T>(a);
  const T *fw = state_fw<T>(a);
  // the next tile diagonal (launched as a programmatic dependent) may start its first round
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  // 1a. row codes, task records and step offsets -> shared memory (row lists start at a
  //     multiple of four entries, records are 16 bytes, the step stride a multiple of eight)
  if (meta_bar) {
    const unsigned bar = smem_u32(meta_bar);
    if (tid == 0) {
      const unsigned b_codes = (unsigned)((nrows + 3) / 4) * 16u, b_trec = (unsigned)ntask * 16u,
                     b_steps = (unsigned)tv.steps_stride * 2u;
      mbar_expect_arrive(bar, b_codes + b_trec + b_steps);
      bulk_g2s(smem_u32(Codes), tv.rows + rb, b_codes, bar);
      bulk_g2s(smem_u32(Trec), tv.tasks + tb, b_trec, bar);
      bulk_g2s(smem_u32(Steps), tv.steps + (size_t)job * tv.steps_stride, b_steps, bar);
    }
    // bounded wait: a phase that never completes marks the sweep failed and skips the job
    bool ok = mbar_try(bar, 0);
    if (!ok) {
      const unsigned long long t0 = gtimer();
      while (!(ok = mbar_try(bar, 0)) && gtimer() - t0 < kWaitNs) {
      }
    }
    if (team_or<THREADS, BAR>(!ok)) {
      if (tid == 0) atomicExch(tv.err, 1);
      return;
    }
  } else {
    for (int i = tid; i < (nrows + 3) / 4; i += THREADS)
      cp_async16(Codes + 4 * i, tv.rows + rb + 4 * i);
    for (int i = tid; i < ntask; i += THREADS) cp_async16(Trec + i, tv.tasks + tb + i);
    for (int i = tid; i < tv.steps_stride / 8; i += THREADS)
      cp_async16(Steps + 8 * i, tv.steps + (size_t)job * tv.steps_stride + 8 * i);
    cp_async_wait_all();
    team_sync<THREADS, BAR>();
  }
  // 1b. the moments of the tasks' nodes (FP64 Rho, Ux | Uy, Uz; written by the previous
  //     iteration), then, once the previous diagonal's rows are visible, the rows
  for (int i = tid; i < 2 * ntask; i += THREADS) {
    const int m = Trec[i >> 1].x & ((1 << 27) - 1);
    cp_async16(Mom + i, reinterpret_cast<const double2 *>(a.mom) + 2 * (size_t)m + (i & 1));
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (tid < PIECES) *reinterpret_cast<int4 *>(S + tid * EPP) = make_int4(0, 0, 0, 0);
  const int grp = tid / LPT, sub = tid % LPT;
  const int o = Codes[0] & 7;                       // own row code = node * 8 + octant
  const bool nx_ = neg_x(o), ny_ = neg_y(o), nz_ = neg_z(o);
  T *hw = const_cast<T *>(h);

#pragma unroll 1
  for (int c = 0; c < NCH; ++c) {
    const int l0 = (chunk0 + c) * V;
    if (c > 0) team_sync<THREADS, BAR>();                     // the previous chunk's write-back read S
    for (int i = tid; i < nrows * PIECES; i += THREADS) {
      const int r = i / PIECES, pc = i - r * PIECES;
      const int code = Codes[r];
      const T *src = ((code & kFwBit) ? fw : h) + (size_t)(code & ~kFwBit) * (size_t)Nc8 + l0 + pc * EPP;
      cp_async16(S + (size_t)(1 + r) * V + pc * EPP, src);
    }

    // per-lane constants of its two velocities
    const int lp = l0 + 2 * sub;
    T K[13][2];
    load_lane_consts<T>(a, lp, K);

    cp_async_wait_all();
    team_sync<THREADS, BAR>();

    // 2. the part of every update that does not depend on this sweep's values,
    //    mu * (fEq - f_old / 2) (solver.F90:205-214), replaces f_old in the task's own slot
    base_pass<T, V, GROUPS>(a, Mom, S, 1, ntask, grp, sub, K, nx_, ny_, nz_);
    team_sync<THREADS, BAR>();

    // 3. local hyperplanes: the upwind terms in the reference's order, then the division
    for (int s = 0; s < nsteps; ++s) {
      const int t0 = Steps[s], t1 = Steps[s + 1];
      if (t0 == t1) continue;
      for (int t = t0 + grp; t < t1; t += GROUPS) update_task<T, V>(a, S, Trec[t], 1 + t, sub, lp, K);
      team_sync<THREADS, BAR>();
    }

    // 4. own rows -> global
    for (int i = tid; i < ntask * PIECES; i += THREADS) {
      const int r = i / PIECES, pc = i - r * PIECES;
      const int code = Codes[r];
      *reinterpret_cast<int4 *>(hw + (size_t)code * Nc8 + l0 + pc * EPP) =
          *reinterpret_cast<const int4 *>(S + (size_t)(1 + r) * V + pc * EPP);
    }
  }
}

// Velocity chunks one CTA of a diagonal launch sweeps (when they divide the chunk count;
// otherwise one). Measured on B200 (128^3 pack, 512 velocities, sweep per iteration): FP64
// one / two / four chunks of 16 per CTA 6.03 / 5.73 / 5.90 ms; FP32 one / two chunks of 32:
// 2.79 / 2.94 ms.
template <typename T> constexpr int kChunksPerCta = sizeof(T) == 8 ? 2 : 1;
// Whether a diagonal launch's CTAs take their job metadata by bulk copies: measured on the
// same workload, FP64 5.96 ms with them against 6.03 without, FP32 2.85 against 2.79.
template <typename T> constexpr bool kBulkMeta = sizeof(T) == 8;

template <typename T, int V, int CPB>
__global__ void __launch_bounds__(threads_of<T, V>())
k_tile_sweep(const DevState a, int job0, int slots_cap, int tasks_cap) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long meta_bar;
  if (kBulkMeta<T>) {
    if (threadIdx.x == 0) {
      mbar_init(smem_u32(&meta_bar), 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
  }
  const int per_job = a.Nc8 / V / CPB;              // CTAs per job
  tile_job<T, V, CPB>(a, a.tv.job_list[job0 + (int)(blockIdx.x / per_job)], (int)(blockIdx.x % per_job) * CPB,
                      slots_cap, tasks_cap, smem_raw, kBulkMeta<T> ? &meta_bar : nullptr);
}

// A pair of jobs per CTA: two teams of threads_of<T, V>() threads, each sweeping one job in
// its own part of the shared memory (the first job's part, sized for it, then the second's),
// so that a large job and a small one share one CTA's allocation instead of each CTA
// reserving room for the diagonal's largest job. Pairs are job_list[job0 + 2p, +1].
__host__ __device__ inline size_t job_smem_bytes(int nrows, int ntask, int steps_stride, int row_bytes) {
  return tile_smem_bytes(nrows + 1, ntask, steps_stride, row_bytes);
}
template <typename T, int V, int CPB>
__global__ void __launch_bounds__(2 * threads_of<T, V>())
k_tile_sweep_pairs(const DevState a, int job0, int njobs, unsigned smem_bytes) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long meta_bar[2];
  constexpr int TH = threads_of<T, V>();
  if (kBulkMeta<T>) {
    if (threadIdx.x == 0) {
      mbar_init(smem_u32(&meta_bar[0]), 1);
      mbar_init(smem_u32(&meta_bar[1]), 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
  }
  const TileView &tv = a.tv;
  const int per_pair = a.Nc8 / V / CPB;             // CTAs per pair
  const int pr = (int)(blockIdx.x / per_pair), chunk0 = (int)(blockIdx.x % per_pair) * CPB;
  const int half = (int)threadIdx.x / TH, tid = (int)threadIdx.x % TH;
  const int q = 2 * pr + half;
  if (q >= njobs) return;                           // the lone job of an odd count: one team
  const int ja = tv.job_list[job0 + 2 * pr], job = tv.job_list[job0 + q];
  const int rb = V * (int)sizeof(T);
  const size_t off = half ? job_smem_bytes(tv.row_count[ja], (int)(tv.task_begin[ja + 1] - tv.task_begin[ja]),
                                           tv.steps_stride, rb)
                          : 0;
  const int nrows = tv.row_count[job], ntask = (int)(tv.task_begin[job + 1] - tv.task_begin[job]);
  if (off + job_smem_bytes(nrows, ntask, tv.steps_stride, rb) > smem_bytes) {
    if (tid == 0) atomicExch(tv.err, 1);            // the plan's bound was exceeded: report, skip
    return;
  }
  if (half == 0)
    tile_job<T, V, CPB, 1>(a, job, chunk0, nrows + 1, ntask, smem_raw, kBulkMeta<T> ? &meta_bar[0] : nullptr, tid);
  else
    tile_job<T, V, CPB, 2>(a, job, chunk0, nrows + 1, ntask, smem_raw + off, kBulkMeta<T> ? &meta_bar[1] : nullptr,
                           tid);
}

// Lets `fn` use all the shared memory a block may opt into, less its static shared memory.
void allow_dynamic_smem(const void *fn, int dev) {
  cudaFuncAttributes fa{};
  int optin = 0;
  if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Waits until *flag == epoch. Gives up after about a second (kMaxPolls polls) or as soon
// as another CTA has given up, and then returns false with *err set.
constexpr int kMaxPolls = 1 << 21;
__device__ bool wait_flag(const int *flag, int epoch, int *err) {
  for (int it = 0; it < kMaxPolls; ++it) {
    if (ld_acquire(flag) == epoch) return true;
    if ((it & 63) == 63 && ld_acquire(err) != 0) return false;
    __nanosleep(256);
  }
  atomicExch(err, 1);
  return false;
}

// Dataflow form of the sweep: one launch per iteration. Work items (job, chunk) are taken
// in the launch plan's order (diagonal by diagonal) from a global counter; an item first
// waits until the items of its upstream tiles (same octant, same chunk) carry this
// iteration's epoch, and publishes its own epoch after its rows are written. Items are
// claimed in an order in which every upstream item comes first, by CTAs that are running,
// so the earliest unfinished claimed item can always proceed.
template <typename T, int V>
__global__ void __launch_bounds__(threads_of<T, V>())
k_tile_sweep_dataflow(const DevState a, int epoch, int slots_cap, int tasks_cap) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int item_s, skip_s;
  const TileView &tv = a.tv;
  const int nchunk = a.Nc8 / V;
  const int nitems = tv.njobs * nchunk;
  for (;;) {
    if (threadIdx.x == 0) { item_s = atomicAdd(tv.counter, 1); skip_s = 0; }
    __syncthreads();
    const int item = item_s;
    if (item >= nitems) break;
    const int job = tv.job_list[item / nchunk], chunk = item % nchunk;
    if (threadIdx.x < 3) {
      const int u = tv.up[4 * job + threadIdx.x];
      if (u >= 0 && !wait_flag(tv.flags + (size_t)u * nchunk + chunk, epoch, tv.err)) skip_s = 1;
    }
    __syncthreads();
    if (!skip_s) tile_job<T, V>(a, job, chunk, slots_cap, tasks_cap, smem_raw);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      st_release(tv.flags + (size_t)job * nchunk + chunk, epoch);
    }
  }
}

// Batched dataflow sweep: the work items of several solves (one DevState each, in device
// memory) in one launch. items[i] = (member | chunk << 12, job), ordered so that every
// item's upstream items (same member, same chunk) come first. A member's flags are cleared
// before the launch and hold 1 once an item is done.
template <typename T, int V>
__global__ void __launch_bounds__(threads_of<T, V>())
k_tile_sweep_batch(const DevState *states, const int2 *items, int nitems, int slots_cap, int tasks_cap, int *counter,
                   int *err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int item_s, skip_s;
  for (;;) {
    if (threadIdx.x == 0) { item_s = atomicAdd(counter, 1); skip_s = 0; }
    __syncthreads();
    const int item = item_s;
    if (item >= nitems) break;
    const int2 it = items[item];
    const int member = it.x & 4095, chunk = it.x >> 12, job = it.y;
    const DevState &a = states[member];
    const int nchunk = a.Nc8 / V;
    if (threadIdx.x < 3) {
      const int u = a.tv.up[4 * job + threadIdx.x];
      if (u >= 0 && !wait_flag(a.tv.flags + (size_t)u * nchunk + chunk, 1, err)) skip_s = 1;
    }
    __syncthreads();
    if (!skip_s) tile_job<T, V>(a, job, chunk, slots_cap, tasks_cap, smem_raw);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      st_release(a.tv.flags + (size_t)job * nchunk + chunk, 1);
    }
  }
}

template <typename T, int V>
void launch_batch(const DevState *states, const int2 *items, int nitems, int slots, int tasks, int stride,
                  int *counter, int *err, cudaStream_t st) {
  const void *fn = reinterpret_cast<const void *>(k_tile_sweep_batch<T, V>);
  once_per_device(fn, [](int dev) { allow_dynamic_smem(reinterpret_cast<const void *>(k_tile_sweep_batch<T, V>), dev); });
  const size_t smem = tile_smem_bytes(slots, tasks, stride, V * (int)sizeof(T));
  long grid = resident_blocks(fn, threads_of<T, V>(), smem);
  if (grid > nitems) grid = nitems;
  if (grid < 1) return;
  cudaMemsetAsync(counter, 0, sizeof(int), st);
  k_tile_sweep_batch<T, V><<<(unsigned)grid, threads_of<T, V>(), smem, st>>>(states, items, nitems, slots, tasks, counter,
                                                                         err);
}

template <typename T, int V>
void launch_dataflow(const DevState &s, int epoch, int slots, int tasks, cudaStream_t st) {
  const void *fn = reinterpret_cast<const void *>(k_tile_sweep_dataflow<T, V>);
  once_per_device(fn, [](int dev) { allow_dynamic_smem(reinterpret_cast<const void *>(k_tile_sweep_dataflow<T, V>), dev); });
  const size_t smem = tile_smem_bytes(slots, tasks, s.tv.steps_stride, V * (int)sizeof(T));
  const long items = (long)s.tv.njobs * (s.Nc8 / V);
  long grid = resident_blocks(fn, threads_of<T, V>(), smem);
  if (grid > items) grid = items;
  if (grid < 1) return;
  cudaMemsetAsync(s.tv.counter, 0, sizeof(int), st);
  k_tile_sweep_dataflow<T, V><<<(unsigned)grid, threads_of<T, V>(), smem, st>>>(s, epoch, slots, tasks);
}

template <typename T, int V, int CPB>
void launch_cpb(const DevState &s, int job0, int njobs, int slots, int tasks, bool pdl, cudaStream_t st) {
  once_per_device(reinterpret_cast<const void *>(k_tile_sweep<T, V, CPB>),
                  [](int dev) { allow_dynamic_smem(reinterpret_cast<const void *>(k_tile_sweep<T, V, CPB>), dev); });
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)((size_t)njobs * (s.Nc8 / V / CPB)));
  cfg.blockDim = dim3(threads_of<T, V>());
  cfg.dynamicSmemBytes = tile_smem_bytes(slots, tasks, s.tv.steps_stride, V * (int)sizeof(T));
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k_tile_sweep<T, V, CPB>, s, job0, slots, tasks);
}

// A launch of job pairs; slots / tasks are the largest sums of a pair (TileJobs::paired).
template <typename T, int V, int CPB>
void launch_pairs(const DevState &s, int job0, int njobs, int slots, int tasks, bool pdl, cudaStream_t st) {
  once_per_device(reinterpret_cast<const void *>(k_tile_sweep_pairs<T, V, CPB>), [](int dev) {
    allow_dynamic_smem(reinterpret_cast<const void *>(k_tile_sweep_pairs<T, V, CPB>), dev);
  });
  // both parts' layouts: the pair's slot and task sums, a second step array and the
  // rounding of two code arrays
  const size_t bytes = tile_smem_bytes(slots, tasks, s.tv.steps_stride, V * (int)sizeof(T)) +
                       (size_t)s.tv.steps_stride * 2 + 32;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)((size_t)(njobs + 1) / 2 * (s.Nc8 / V / CPB)));
  cfg.blockDim = dim3(2 * threads_of<T, V>());
  cfg.dynamicSmemBytes = bytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k_tile_sweep_pairs<T, V, CPB>, s, job0, njobs, (unsigned)bytes);
}

template <typename T, int V>
void launch_one(const DevState &s, int job0, int njobs, int slots, int tasks, bool pdl, cudaStream_t st) {
  constexpr int C = kChunksPerCta<T>;
  const bool cpb = C > 1 && (s.Nc8 / V) % C == 0;
  if constexpr (threads_of<T, V>() % 32 == 0) {
    if (s.tv.paired) {
      if (cpb) launch_pairs<T, V, C>(s, job0, njobs, slots, tasks, pdl, st);
      else launch_pairs<T, V, 1>(s, job0, njobs, slots, tasks, pdl, st);
      return;
    }
  }
  {
    if (cpb) launch_cpb<T, V, C>(s, job0, njobs, slots, tasks, pdl, st);
    else launch_cpb<T, V, 1>(s, job0, njobs, slots, tasks, pdl, st);
  }
}

}  // namespace

// Velocities per CTA: 128-byte rows where the octant has enough velocities.
int tile_sweep_velocities(int Nc8, bool fp32) {
  if (fp32) return Nc8 % 32 == 0 ? 32 : Nc8 % 16 == 0 ? 16 : 8;
  return Nc8 % 16 == 0 ? 16 : 8;
}

int tile_sweep_max_slots(int Nc8, bool fp32, int tile_voxels, int nsteps) {
  const int row = tile_sweep_velocities(Nc8, fp32) * (fp32 ? 4 : 8);
  const size_t fixed = tile_smem_bytes(0, tile_voxels, (nsteps + 1 + 7) / 8 * 8, row) + 16;
  const size_t cap = 227 * 1024 - 256;  // less the kernels' static shared memory
  return fixed >= cap ? 0 : (int)((cap - fixed) / (row + 4));
}

void launch_tile_sweep(const DevState &s, bool fp32, int job0, int njobs, int slots, int tasks, bool pdl,
                       cudaStream_t st) {
  if (njobs <= 0) return;
  const int V = tile_sweep_velocities(s.Nc8, fp32);
  if (fp32) {
    if (V == 32) launch_one<float, 32>(s, job0, njobs, slots, tasks, pdl, st);
    else if (V == 16) launch_one<float, 16>(s, job0, njobs, slots, tasks, pdl, st);
    else launch_one<float, 8>(s, job0, njobs, slots, tasks, pdl, st);
  } else {
    if (V == 16) launch_one<double, 16>(s, job0, njobs, slots, tasks, pdl, st);
    else launch_one<double, 8>(s, job0, njobs, slots, tasks, pdl, st);
  }
}

}  // namespace piks

namespace piks {

void launch_tile_sweep_dataflow(const DevState &s, bool fp32, int epoch, int slots, int tasks, cudaStream_t st) {
  if (s.tv.njobs <= 0) return;
  const int V = tile_sweep_velocities(s.Nc8, fp32);
  if (fp32) {
    if (V == 32) launch_dataflow<float, 32>(s, epoch, slots, tasks, st);
    else if (V == 16) launch_dataflow<float, 16>(s, epoch, slots, tasks, st);
    else launch_dataflow<float, 8>(s, epoch, slots, tasks, st);
  } else {
    if (V == 16) launch_dataflow<double, 16>(s, epoch, slots, tasks, st);
    else launch_dataflow<double, 8>(s, epoch, slots, tasks, st);
  }
}

}  // namespace piks

namespace piks {

void launch_tile_sweep_batch(const DevState *states, const int2 *items, int nitems, bool fp32, int V, int slots,
                             int tasks, int stride, int *counter, int *err, cudaStream_t st) {
  if (nitems <= 0) return;
  if (fp32) {
    if (V == 32) launch_batch<float, 32>(states, items, nitems, slots, tasks, stride, counter, err, st);
    else if (V == 16) launch_batch<float, 16>(states, items, nitems, slots, tasks, stride, counter, err, st);
    else launch_batch<float, 8>(states, items, nitems, slots, tasks, stride, counter, err, st);
  } else {
    if (V == 16) launch_batch<double, 16>(states, items, nitems, slots, tasks, stride, counter, err, st);
    else launch_batch<double, 8>(states, items, nitems, slots, tasks, stride, counter, err, st);
  }
}

}  // namespace piks
