// Persistent producer / consumer octant sweeps (solver.F90:176-526) over the split forms of
// TileJobs: a producer warp stages tile jobs into shared memory with bulk asynchronous
// copies (cp.async.bulk completing on mbarriers) while consumer warps sweep jobs staged
// earlier. Two variants share the producer:
//  * column march (k_column_sweep<COL = true>): work items are columns (one octant's tiles
//    at one (x, y) tile position, in the octant's z order); the consumer warps of a CTA
//    sweep each job together, task groups of V/2 lanes with two velocities per lane, one
//    named barrier per local hyperplane, and carry the tile's last two z layers to the next
//    tile of the column on chip;
//  * pipelined dataflow, cooperative (k_column_sweep<COL = false>): work items are single
//    jobs in the diagonal launch order, all upwind rows staged from HBM; consumers as above;
// The producer of a job copies, per metadata slot: its task records, row codes, step offsets
// and carry lists; then into a region of a shared-memory row arena: a zero row, the job's own
// rows (previous iteration's values), the static rows (solid, corner and inflow-plane rows,
// never written by the sweep) and the moments of its nodes; and, once the upwind tiles' jobs
// have published their flags, the dependent rows those jobs wrote. It claims work in
// dependency order and runs ahead of the consumers as far as the metadata slots and the
// arena allow (regions are allocated in order and reclaimed in order).
// The per-task arithmetic is the tile-diagonal kernel's (sweep_core.cuh), so the FP64 values
// are the reference's bit for bit whatever the schedule, and the FP32 values equal the tile
// kernel's.
//
// Waits are bounded by the global timer (about two seconds): a dependency wait that gives
// up sets the error flag and the job still runs (on stale upwind rows) and publishes its
// flag, so nothing downstream waits longer; an mbarrier wait that gives up sets the error
// flag and an abort flag, on which every warp stops, the producer after waiting (bounded)
// for the copies it issued.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"
#include "sweep_core.cuh"

namespace piks {

namespace {

using namespace sweep;


// 256 zero bytes: the source of every region's zero row (slot 0).
__device__ __align__(128) unsigned char g_zero_row[256] = {0};

// Shared-memory layout of one CTA (byte offsets; every region 16-byte aligned).
struct ColLayout {
  int rb;            // bytes per row: V * sizeof(T)
  int arena_rows;    // rows in the arena
  int kmeta;         // metadata slots
  int max_tasks, max_codes, steps_stride, max_carry, ncells, nctab;
  unsigned off_carrybuf, off_arena, off_meta, meta_bytes;
  unsigned m_trec, m_mom, m_codes, m_steps, m_carry;   // offsets inside one metadata slot
  unsigned off_ctab;  // nctab class tables of 16 rows (rb bytes each)
  unsigned off_desc, off_bar, total;
};

struct Desc {
  int job, chunk, base, ntask, ncin, ncout, fresh, pad;
};

// Waits for the phase of `parity` to complete; gives up (false, *abort and *err set) after
// kWaitNs or as soon as another warp of the CTA has aborted.
__device__ bool mbar_wait(unsigned bar, unsigned parity, volatile int *abort, int *err) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = gtimer();
  for (int it = 1;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 31) == 0) {
      if (*abort) return false;
      if (gtimer() - t0 > kWaitNs) {
        *abort = 1;
        atomicExch(err, 1);
        return false;
      }
    }
  }
}
// 16 bytes global -> shared through L2 (LSU path); completion is tracked per thread.
__device__ __forceinline__ void cp16(unsigned dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
// Arrives on the mbarrier once all of this thread's earlier cp.async copies are complete
// (counted as one of the barrier's expected arrivals).
__device__ __forceinline__ void cp_async_arrive(unsigned bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Waits until *flag == epoch; gives up (false, *err set) after kWaitNs or once *err is set.
__device__ bool wait_flag(const int *flag, int epoch, int *err) {
  if (ld_acquire(flag) == epoch) return true;
  const unsigned long long t0 = gtimer();
  for (int it = 1;; ++it) {
    if (ld_acquire(flag) == epoch) return true;
    if ((it & 63) == 0) {
      if (ld_acquire(err) != 0) return false;
      if (gtimer() - t0 > kWaitNs) {
        atomicExch(err, 1);
        return false;
      }
    }
    __nanosleep(128);
  }
}
__device__ __forceinline__ void consumer_bar(int nthreads) {
  asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}
// Barrier 1 over the consumer threads that also returns whether `ok` holds in all of them.
__device__ __forceinline__ bool consumer_all(int nthreads, bool ok) {
  unsigned r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, 1, %2, p;\n selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((unsigned)ok), "r"(nthreads)
      : "memory");
  return r != 0;
}

// A job and its header (hdr: row_begin, task_begin, carry_begin, nrows, ntask, first
// dependent row, ncin, ncout), lane-uniform in the producer warp.
struct Pending {
  int job, chunk, fresh;
  int4 h0, h1;
};

// The shared-memory pipeline state of a CTA with KM metadata slots.
template <int KM>
struct Pipe {
  unsigned char *smem;
  const ColLayout *L;
  Desc *desc;
  unsigned long long *bars;
  volatile int *abort;
  int *reg_base;
  __device__ Pipe(unsigned char *sm, const ColLayout &l) : smem(sm), L(&l) {
    desc = reinterpret_cast<Desc *>(sm + l.off_desc);
    bars = reinterpret_cast<unsigned long long *>(sm + l.off_bar);
    int *ctl = reinterpret_cast<int *>(bars + 3 * KM);
    abort = ctl;
    reg_base = ctl + 1;
  }
  __device__ unsigned full(int s) const { return smem_u32(bars + s); }
  __device__ unsigned empty(int s) const { return smem_u32(bars + KM + s); }
  __device__ unsigned metab(int s) const { return smem_u32(bars + 2 * KM + s); }
  __device__ unsigned char *slot(int s) const { return smem + L->off_meta + (size_t)s * L->meta_bytes; }
  __device__ void init() {
    for (int s = 0; s < KM; ++s) {
      mbar_init(full(s), 33);   // the 32 producer lanes' copy completions and lane 0's descriptor
      mbar_init(empty(s), 1);
      mbar_init(empty(s), 1);
      mbar_init(metab(s), 1);
    }
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
};

// The producer warp. COL: items are columns (jobs in z order), dependent rows come from the
// x- and y-upwind tiles only; else items are single jobs in the diagonal launch order and
// the z-upwind tile's rows are dependent rows too. Metadata of tile k + AHEAD is requested
// while the rows of tile k are staged. After the last job it stages one end marker per
// consumer team (NTEAM teams take tiles round robin).
template <typename T, int V, bool COL, int KM, int AHEAD, int NTEAM>
__device__ void run_producer(const DevState &a, const ColLayout &L, int epoch, Pipe<KM> &P) {
  static_assert(AHEAD >= 1 && AHEAD < KM, "metadata lookahead must leave a slot for the rows being staged");
  const TileView &tv = a.tv;
  const int lane = threadIdx.x & 31;
  const int nchunk = a.Nc8 / V;
  const T *h = state_h<T>(a);
  const T *fw = state_fw<T>(a);
  T *arena = reinterpret_cast<T *>(P.smem + L.off_arena);
  const long nitems = COL ? (long)tv.ncols * nchunk : (long)tv.njobs * nchunk;
  int q = 0, qend = 0, chunk = 0;
  int rel = 0, tail = 0;          // tiles known released; arena end of the last region
  // dataflow claims run two calls ahead in lane 0: claim_a (counter value of an atomic
  // issued one call earlier), claim_b and job_b (its item and the job_list entry loaded)
  int claim_a = 0, claim_b = 0, job_b = -1;
  if (!COL && lane == 0) {
    claim_b = atomicAdd(tv.counter, 1);
    claim_a = atomicAdd(tv.counter, 1);
    job_b = claim_b < nitems ? __ldg(tv.job_list + claim_b / nchunk) : -1;
  }
  bool ended = false;             // the last claim returned no work
  auto next_job = [&]() {
    Pending p;
    p.fresh = 0;
    p.job = -1;
    p.chunk = 0;
    if (ended) return p;
    if (!COL) {
      const int it = __shfl_sync(0xffffffffu, claim_b, 0);
      const int jb = __shfl_sync(0xffffffffu, job_b, 0);
      if (lane == 0) {
        claim_b = claim_a;
        job_b = claim_b < nitems ? __ldg(tv.job_list + claim_b / nchunk) : -1;
        claim_a = atomicAdd(tv.counter, 1);
      }
      if (it >= nitems) { ended = true; return p; }
      p.job = jb;
      p.chunk = it % nchunk;
      p.fresh = 1;
    } else {
      if (q >= qend) {
        int it = 0;
        if (lane == 0) it = atomicAdd(tv.counter, 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nitems) { ended = true; return p; }
        const int col = tv.col_list[it / nchunk];
        chunk = it % nchunk;
        q = tv.col_begin[col];
        qend = tv.col_begin[col + 1];
        p.fresh = 1;
      }
      p.job = tv.col_jobs[q++];
      p.chunk = chunk;
    }
    const int4 *hp = reinterpret_cast<const int4 *>(tv.hdr) + 2 * (size_t)p.job;
    p.h0 = __ldg(hp);
    p.h1 = __ldg(hp + 1);
    return p;
  };
  auto wait_release = [&]() -> bool {
    const bool ok =
        __all_sync(0xffffffffu, mbar_wait(P.empty(rel % KM), (unsigned)((rel / KM) & 1), P.abort, tv.err));
    if (ok) ++rel;
    return ok;
  };
  // task records, row codes, step offsets and carry lists of tile k
  auto stage_meta = [&](int k, const Pending &p) -> bool {
    const int s = k % KM;
    while (rel <= k - KM)
      if (!wait_release()) return false;
    if (lane == 0) {
      Desc &d = P.desc[s];
      d.job = p.job; d.chunk = p.chunk; d.fresh = p.fresh;
      d.ntask = p.job >= 0 ? p.h1.x : 0;
      d.ncin = p.job >= 0 ? p.h1.z : 0;
      d.ncout = p.job >= 0 ? p.h1.w : 0;
    }
    __syncwarp();
    if (p.job < 0) return true;
    const int nrows = p.h0.w, ntask = p.h1.x, ncarry = p.h1.z + p.h1.w;
    const unsigned b_trec = (unsigned)ntask * 16, b_codes = (unsigned)((nrows + 3) / 4) * 16,
                   b_steps = (unsigned)tv.steps_stride * 2, b_carry = (unsigned)((ncarry + 3) / 4) * 16;
    if (lane == 0) mbar_expect_arrive(P.metab(s), b_trec + b_codes + b_steps + b_carry);
    __syncwarp();
    unsigned char *m = P.slot(s);
    if (lane == 0 && b_trec) bulk_g2s(smem_u32(m + L.m_trec), tv.tasks + p.h0.y, b_trec, P.metab(s));
    if (lane == 1 && b_codes) bulk_g2s(smem_u32(m + L.m_codes), tv.rows + p.h0.x, b_codes, P.metab(s));
    if (lane == 2) bulk_g2s(smem_u32(m + L.m_steps), tv.steps + (size_t)p.job * tv.steps_stride, b_steps, P.metab(s));
    if (lane == 3 && b_carry) bulk_g2s(smem_u32(m + L.m_carry), tv.carry + p.h0.z, b_carry, P.metab(s));
    return true;
  };
  // the rows and moments of tile k into a region of the arena; an end marker for no job.
  // Rows and moments move in 16-byte cp.async pieces (a warp instruction moves 512 bytes);
  // each lane's completion arrives on the tile's full barrier, and lane 0 arrives once the
  // descriptor is written.
  auto stage_rows = [&](int k, const Pending &p) -> bool {
    constexpr int EPP = 16 / (int)sizeof(T);     // elements per 16-byte piece
    constexpr int PIECES = V / EPP;              // pieces per row
    const int s = k % KM;
    if (p.job < 0) {                             // end of work
      cp_async_arrive(P.full(s));
      __syncwarp();
      if (lane == 0) mbar_arrive(P.full(s));
      return true;
    }
    if (!__all_sync(0xffffffffu, mbar_wait(P.metab(s), (unsigned)((k / KM) & 1), P.abort, tv.err))) return false;
    const int nrows = p.h0.w, ntask = p.h1.x, dep0 = p.h1.y, ncin = p.h1.z;
    const int n = 1 + ncin + nrows;
    int base = -1;
    for (;;) {                     // contiguous room for n rows after the live regions
      if (rel == k) { base = 0; break; }
      const int head = P.reg_base[rel % KM];
      if (tail > head) {
        if (L.arena_rows - tail >= n) { base = tail; break; }
        if (head >= n) { base = 0; break; }
      } else if (head - tail >= n) {
        base = tail;
        break;
      }
      if (!wait_release()) return false;
    }
    tail = base + n;
    unsigned char *m = P.slot(s);
    const int *codes = reinterpret_cast<const int *>(m + L.m_codes);
    const int4 *trec = reinterpret_cast<const int4 *>(m + L.m_trec);
    const unsigned mom = smem_u32(m + L.m_mom);
    const unsigned R0 = smem_u32(arena) + (unsigned)base * (unsigned)L.rb;
    const unsigned RS = R0 + (unsigned)(1 + ncin) * (unsigned)L.rb;   // first job row
    const size_t l0 = (size_t)p.chunk * V;
    for (int i = lane; i < PIECES; i += 32) cp16(R0 + 16u * i, g_zero_row + 16 * i);
    for (int i = lane; i < dep0 * PIECES; i += 32) {
      const int r = i / PIECES, pc = i - r * PIECES;
      const int code = codes[r];
      const T *src = ((code & kFwBit) ? fw : h) + (size_t)(code & ~kFwBit) * (size_t)a.Nc8 + l0 + pc * EPP;
      cp16(RS + (unsigned)r * (unsigned)L.rb + 16u * pc, src);
    }
    for (int i = lane; i < 2 * ntask; i += 32) {
      const int node = trec[i >> 1].x & ((1 << 27) - 1);
      cp16(mom + 16u * i, a.mom + (size_t)node * 4 + 2 * (i & 1));
    }
    if (dep0 < nrows) {
      // the rows of the upwind tiles' jobs (x and y; z too without carried layers), once
      // those are done
      if (lane < (COL ? 2 : 3)) {
        const int u = tv.up[4 * (size_t)p.job + lane];
        if (u >= 0) wait_flag(tv.flags + (size_t)u * nchunk + p.chunk, epoch, tv.err);
      }
      __syncwarp();
      for (int i = dep0 * PIECES + lane; i < nrows * PIECES; i += 32) {
        const int r = i / PIECES, pc = i - r * PIECES;
        const T *src = h + (size_t)codes[r] * (size_t)a.Nc8 + l0 + pc * EPP;
        cp16(RS + (unsigned)r * (unsigned)L.rb + 16u * pc, src);
      }
    }
    cp_async_arrive(P.full(s));
    if (lane == 0) {
      P.desc[s].base = base;
      P.reg_base[s] = base;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(P.full(s));
    return true;
  };

  // pend[i] = job of tile k + i (its metadata requested for i < AHEAD)
  Pending pend[AHEAD + 1];
#pragma unroll
  for (int i = 0; i <= AHEAD; ++i) pend[i] = next_job();
  bool ok = true;
#pragma unroll
  for (int i = 0; i < AHEAD; ++i)
    if (ok) ok = stage_meta(i, pend[i]);
  int k = 0, rows_issued = 0, ends = 0;
  while (ok) {
    ok = stage_meta(k + AHEAD, pend[AHEAD]);
    if (ok) ok = stage_rows(k, pend[0]);
    if (!ok) break;
    rows_issued = k + 1;
    if (pend[0].job < 0 && ++ends == NTEAM) break;    // every team has its end marker
#pragma unroll
    for (int i = 0; i < AHEAD; ++i) pend[i] = pend[i + 1];
    pend[AHEAD] = next_job();
    ++k;
  }
  if (!ok) {
    // aborted: wait (bounded) for the copies of staged tiles before the CTA exits
    for (int m = rel; m < rows_issued; ++m) {
      const unsigned long long t0 = gtimer();
      while (!mbar_try(P.full(m % KM), (unsigned)((m / KM) & 1)) && gtimer() - t0 < kWaitNs) {
      }
    }
    for (int m = std::max(rel, rows_issued); m <= k + AHEAD; ++m) {
      const unsigned long long t0 = gtimer();
      while (!mbar_try(P.metab(m % KM), (unsigned)((m / KM) & 1)) && gtimer() - t0 < kWaitNs) {
      }
    }
  }
}

// ------------------------------------------------------------------- cooperative consumers
// COL: column march (items are columns, jobs in z order, z layers carried on chip); else
// pipelined dataflow (items are single jobs in the diagonal launch order, every upwind row
// staged from HBM once its job has published its flag).
template <typename T, int V, int NCW, bool COL>
__global__ void __launch_bounds__((NCW + 1) * 32)
k_column_sweep(const DevState a, const ColLayout L, int epoch) {
  constexpr int KM = 4;
  constexpr int NCT = NCW * 32;                  // consumer threads
  constexpr int LPT = V / 2;                     // lanes per task
  constexpr int GROUPS = NCT / LPT;              // tasks in flight per pass
  constexpr int EPP = 16 / (int)sizeof(T);       // elements per 16-byte piece
  constexpr int PIECES = V / EPP;                // pieces per row
  extern __shared__ __align__(128) unsigned char smem[];
  const TileView &tv = a.tv;
  Pipe<KM> P(smem, L);
  T *arena = reinterpret_cast<T *>(smem + L.off_arena);
  T *carrybuf = reinterpret_cast<T *>(smem + L.off_carrybuf);
  T *ctab = reinterpret_cast<T *>(smem + L.off_ctab);
  const int warp = threadIdx.x >> 5;
  const int nchunk = a.Nc8 / V;
  if (threadIdx.x == 0) P.init();
  __syncthreads();
  if (warp == NCW) {
    run_producer<T, V, COL, KM, 1, 1>(a, L, epoch, P);
    return;
  }
  const int ct = threadIdx.x;
  const int grp = ct / LPT, sub = ct % LPT;
  T K[13][2];
  bool nx_ = false, ny_ = false, nz_ = false;
  int kchunk = -1;
  T *hw = const_cast<T *>(state_h<T>(a));
  for (int k = 0;; ++k) {
    const int s = k % KM;
    // every consumer thread leaves together when any wait gave up
    if (!consumer_all(NCT, mbar_wait(P.full(s), (unsigned)((k / KM) & 1), P.abort, tv.err))) break;
    const Desc d = P.desc[s];
    if (d.job < 0) break;
    unsigned char *m = P.slot(s);
    const int4 *trec = reinterpret_cast<const int4 *>(m + L.m_trec);
    const double2 *mom = reinterpret_cast<const double2 *>(m + L.m_mom);
    const int *codes = reinterpret_cast<const int *>(m + L.m_codes);
    const uint16_t *steps = reinterpret_cast<const uint16_t *>(m + L.m_steps);
    const int *carry = reinterpret_cast<const int *>(m + L.m_carry);
    const int l0 = d.chunk * V;
    const int lp = l0 + 2 * sub;
    if (d.fresh) {
      const int o = codes[0] & 7;
      nx_ = neg_x(o); ny_ = neg_y(o); nz_ = neg_z(o);
      if (d.chunk != kchunk) {
        load_lane_consts<T>(a, lp, K);
        if (grp == 0) load_class_table<T, V>(a, l0, sub, ctab);
      }
      kchunk = d.chunk;
    }
    T *S = arena + (size_t)d.base * V;
    const int own0 = 1 + d.ncin;
    // rows carried from the previous tile of the column
    for (int i = ct; i < d.ncin * PIECES; i += NCT) {
      const int e = i / PIECES, pc = i - e * PIECES;
      const int cell = carry[e] & 0xffff, slot = carry[e] >> 16;
      *reinterpret_cast<int4 *>(S + (size_t)slot * V + pc * EPP) =
          *reinterpret_cast<const int4 *>(carrybuf + (size_t)cell * V + pc * EPP);
    }
    base_pass<T, V, GROUPS>(a, mom, S, own0, d.ntask, grp, sub, K, nx_, ny_, nz_);
    // the bases, the carried rows and (on a new chunk) the class table are read after this
    consumer_bar(NCT);
    for (int st = 0; st < tv.nsteps; ++st) {
      const int t0 = steps[st], t1 = steps[st + 1];
      if (t0 == t1) continue;
      for (int t = t0 + grp; t < t1; t += GROUPS) update_task<T, V>(a, S, trec[t], own0 + t, sub, lp, K, ctab);
      consumer_bar(NCT);
    }
    // own rows -> HBM; this tile's last two z layers -> the carried rows
    for (int i = ct; i < d.ntask * PIECES; i += NCT) {
      const int r = i / PIECES, pc = i - r * PIECES;
      *reinterpret_cast<int4 *>(hw + (size_t)codes[r] * a.Nc8 + l0 + pc * EPP) =
          *reinterpret_cast<const int4 *>(S + (size_t)(own0 + r) * V + pc * EPP);
    }
    for (int i = ct; i < d.ncout * PIECES; i += NCT) {
      const int e = i / PIECES, pc = i - e * PIECES;
      const int r = carry[d.ncin + e] & 0xffff, cell = carry[d.ncin + e] >> 16;
      *reinterpret_cast<int4 *>(carrybuf + (size_t)cell * V + pc * EPP) =
          *reinterpret_cast<const int4 *>(S + (size_t)(own0 + r) * V + pc * EPP);
    }
    consumer_bar(NCT);
    if (ct == 0) {
      mbar_arrive(P.empty(s));
      // the release orders every consumer's stores above (the barrier) before the flag
      st_release(tv.flags + (size_t)d.job * nchunk + d.chunk, epoch);
    }
  }
}

// Layout for row size rb, `kmeta` metadata slots and `nctab` class tables; the arena holds
// arena_rows rows.
ColLayout make_layout(const TileView &tv, int rb, int arena_rows, int kmeta, int nctab) {
  ColLayout L{};
  L.rb = rb;
  L.kmeta = kmeta;
  L.nctab = nctab;
  L.max_tasks = tv.max_tasks;
  L.max_codes = (tv.max_nrows + 3) / 4 * 4;
  L.steps_stride = tv.steps_stride;
  L.max_carry = (tv.max_carry + 3) / 4 * 4;
  L.ncells = tv.ncells;
  L.arena_rows = arena_rows;
  auto up16 = [](unsigned x) { return (x + 15u) / 16u * 16u; };
  unsigned off = 0;
  L.off_carrybuf = off;
  off += up16((unsigned)L.ncells * rb);
  off = (off + 127u) / 128u * 128u;
  L.off_arena = off;
  off += (unsigned)arena_rows * rb;
  L.off_meta = off;
  L.m_trec = 0;
  L.m_mom = up16((unsigned)L.max_tasks * 16);
  L.m_codes = L.m_mom + up16((unsigned)L.max_tasks * 32);
  L.m_steps = L.m_codes + up16((unsigned)L.max_codes * 4);
  L.m_carry = L.m_steps + up16((unsigned)L.steps_stride * 2);
  L.meta_bytes = L.m_carry + up16((unsigned)L.max_carry * 4);
  off += L.meta_bytes * kmeta;
  L.off_ctab = off;
  off += up16(16u * (unsigned)rb) * (unsigned)nctab;
  L.off_desc = off;
  off += (unsigned)sizeof(Desc) * kmeta;
  L.off_bar = off;
  off += 8u * 3 * kmeta + 4u * (1 + kmeta);
  L.total = up16(off);
  return L;
}

constexpr unsigned kSmemCap = 227u * 1024u;

// The arena size: the most CTAs per SM whose arena still holds the largest region plus
// `extra` mean regions (so that later jobs can be staged while the current ones run), else
// the largest arena that fits one CTA per SM.
ColLayout choose_layout(const TileView &tv, int rb, int kmeta, int nctab, float extra) {
  const int need = tv.max_region;
  const int want = tv.max_region + (int)(extra * tv.mean_region + 0.5f);
  for (int per_sm = 8; per_sm >= 1; --per_sm) {
    const unsigned budget = (228u * 1024u) / per_sm - 1024u;
    const ColLayout base = make_layout(tv, rb, 0, kmeta, nctab);
    if (base.total + (unsigned)need * rb > budget || base.total + (unsigned)need * rb > kSmemCap) continue;
    const int rows = (int)((std::min(budget, kSmemCap) - base.total) / (unsigned)rb);
    if (rows >= want || per_sm == 1) return make_layout(tv, rb, rows, kmeta, nctab);
  }
  return make_layout(tv, rb, need, kmeta, nctab);
}

void allow_smem(const void *fn, unsigned bytes) {
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename T, int V, int NCW, bool COL>
void launch_columns(const DevState &s, int epoch, cudaStream_t st) {
  const TileView &tv = s.tv;
  const ColLayout L = choose_layout(tv, V * (int)sizeof(T), 4, 1, 1.0f);
  const void *fn = reinterpret_cast<const void *>(k_column_sweep<T, V, NCW, COL>);
  once_per_device(fn, [](int) {
    allow_smem(reinterpret_cast<const void *>(k_column_sweep<T, V, NCW, COL>), kSmemCap);
  });
  const int threads = (NCW + 1) * 32;
  const long items = (COL ? (long)tv.ncols : (long)tv.njobs) * (s.Nc8 / V);
  long grid = resident_blocks(fn, threads, L.total);
  if (grid > items) grid = items;
  if (grid < 1) return;
  cudaMemsetAsync(tv.counter, 0, sizeof(int), st);
  cudaMemsetAsync(tv.flags, 0, (size_t)tv.njobs * (s.Nc8 / V) * sizeof(int), st);
  k_column_sweep<T, V, NCW, COL><<<(unsigned)grid, threads, L.total, st>>>(s, L, epoch);
}

}  // namespace

bool column_sweep_fits(const TileView &tv, int Nc8, bool fp32) {
  const int V = tile_sweep_velocities(Nc8, fp32);
  return make_layout(tv, V * (fp32 ? 4 : 8), tv.max_region, 4, 1).total <= kSmemCap;
}

void launch_tile_sweep_columns(const DevState &s, bool fp32, int epoch, cudaStream_t st) {
  if (s.tv.njobs <= 0 || s.tv.ncols <= 0) return;
  const int V = tile_sweep_velocities(s.Nc8, fp32);
  if (fp32) {
    if (V == 32) launch_columns<float, 32, 2, true>(s, epoch, st);
    else if (V == 16) launch_columns<float, 16, 2, true>(s, epoch, st);
    else launch_columns<float, 8, 2, true>(s, epoch, st);
  } else {
    if (V == 16) launch_columns<double, 16, 2, true>(s, epoch, st);
    else launch_columns<double, 8, 2, true>(s, epoch, st);
  }
}

void launch_tile_sweep_pipelined(const DevState &s, bool fp32, int epoch, cudaStream_t st) {
  if (s.tv.njobs <= 0) return;
  const int V = tile_sweep_velocities(s.Nc8, fp32);
  if (fp32) {
    if (V == 32) launch_columns<float, 32, 2, false>(s, epoch, st);
    else if (V == 16) launch_columns<float, 16, 2, false>(s, epoch, st);
    else launch_columns<float, 8, 2, false>(s, epoch, st);
  } else {
    if (V == 16) launch_columns<double, 16, 2, false>(s, epoch, st);
    else launch_columns<double, 8, 2, false>(s, epoch, st);
  }
}

}  // namespace piks
