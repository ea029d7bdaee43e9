// C ABI of libpiks3d_b200 (include/piks3d_gpu.h): context life cycle, device memory,
// the per-iteration launch schedule and the host-facing getters / writers.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <future>
#include <mutex>
#include <string>
#include <vector>

#include "context.h"

namespace piks {
void write_fields(const Setup &s, const Geometry &g, const double *rho, const double *ux,
                  const double *uy, const double *uz, const char *dir, int format, std::string &err, bool &ok);
}

using namespace piks;

namespace {
thread_local std::string g_last_error;
const char kKernelNames[] = "sweep,commit,capture,walls,inlet_outlet,symmetry,moments,flux";
}  // namespace

namespace piks {

piks_status fail(piks_status st, const std::string &msg) {
  g_last_error = msg;
  return st;
}

piks_status cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return PIKS_OK;
  if (e == cudaErrorMemoryAllocation) return fail(PIKS_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e));
  return fail(PIKS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace piks


namespace {

template <typename T, typename A>
piks_status upload(piks_ctx *c, const std::vector<T, A> &v, T **out, size_t min_count = 1) {
  size_t n = v.size() < min_count ? min_count : v.size();
  void *p = nullptr;
  piks_status st = cuda_check(cudaMalloc(&p, n * sizeof(T)), "cudaMalloc");
  if (st) return st;
  c->allocations.push_back({p, n * sizeof(T)});
  c->dev_bytes += n * sizeof(T);
  if (!v.empty()) {
    st = cuda_check(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream), "upload");
    if (st) return st;
  }
  *out = static_cast<T *>(p);
  return PIKS_OK;
}

template <typename T>
piks_status zeros(piks_ctx *c, size_t n, T **out) {
  void *p = nullptr;
  piks_status st = cuda_check(cudaMalloc(&p, (n ? n : 1) * sizeof(T)), "cudaMalloc");
  if (st) return st;
  c->allocations.push_back({p, (n ? n : 1) * sizeof(T)});
  c->dev_bytes += (n ? n : 1) * sizeof(T);
  st = cuda_check(cudaMemsetAsync(p, 0, (n ? n : 1) * sizeof(T), c->stream), "memset");
  if (st) return st;
  *out = static_cast<T *>(p);
  return PIKS_OK;
}

void drop_graphs(piks_ctx *c);

void free_device(piks_ctx *c) {
  drop_graphs(c);
  for (auto &a : c->allocations) cudaFree(a.first);
  c->allocations.clear();
  c->dev_bytes = 0;
  c->have_geometry = false;
  c->snap = nullptr;
  c->snap_bytes = 0;
}

void release(piks_ctx *c, void *p) {
  for (size_t i = 0; i < c->allocations.size(); ++i)
    if (c->allocations[i].first == p) {
      cudaFree(p);
      c->dev_bytes -= c->allocations[i].second;
      c->allocations.erase(c->allocations.begin() + (long)i);
      return;
    }
}

// Sizes of the precision-dependent state: f, fw and one ghost plane (in elements).
struct StateSizes { size_t h, fw, plane, hsend[2], hrecv[2]; };
StateSizes state_sizes(const piks_ctx *c) {
  const Geometry &g = c->geo;
  const size_t Nc8 = (size_t)c->vel.Nc8;
  return {((size_t)g.NF + g.NB) * 8 * Nc8, (size_t)g.nCorner * 8 * Nc8, (size_t)g.Ny * g.Nz * 4 * Nc8,
          {g.halo_send[0].size() * 4 * Nc8, g.halo_send[1].size() * 4 * Nc8},
          {g.halo_recv[0].size() * 4 * Nc8, g.halo_recv[1].size() * 4 * Nc8}};
}

// Allocates (zeroed) f, fw and the two pairs of ghost planes in precision `prec`
// (flow.F90:92 f = 0, physicalGrid.F90:1624 fw = 0, flow.F90:151-162 ghosts = 0).
piks_status alloc_state(piks_ctx *c, int prec) {
  DevState &s = c->ds;
  const StateSizes z = state_sizes(c);
  piks_status st;
  if (prec == PIKS_PREC_FP64) {
    if ((st = zeros(c, z.h, &s.h))) return st;
    if ((st = zeros(c, z.fw, &s.fw))) return st;
    for (int b = 0; b < 2; ++b) {
      if ((st = zeros(c, z.plane, &s.ghostW[b]))) return st;
      if ((st = zeros(c, z.plane, &s.ghostE[b]))) return st;
    }
  } else {
    if ((st = zeros(c, z.h, &s.h32))) return st;
    if ((st = zeros(c, z.fw, &s.fw32))) return st;
    for (int b = 0; b < 2; ++b) {
      if ((st = zeros(c, z.plane, &s.ghostW32[b]))) return st;
      if ((st = zeros(c, z.plane, &s.ghostE32[b]))) return st;
    }
  }
  // the x messages of a slab start as zeros (flow.F90:115-163 allocate the buffers zeroed)
  for (int side = 0; side < 2; ++side) {
    if (!z.hsend[side] && !z.hrecv[side]) continue;
    for (int b = 0; b < 2; ++b)
      if ((st = prec == PIKS_PREC_FP64 ? zeros(c, z.hsend[side], &s.hsend[side][b])
                                       : zeros(c, z.hsend[side], &s.hsend32[side][b]))) return st;
    if ((st = prec == PIKS_PREC_FP64 ? zeros(c, z.hrecv[side], &s.hrecv[side]) : zeros(c, z.hrecv[side], &s.hrecv32[side])))
      return st;
  }
  return PIKS_OK;
}

void free_state(piks_ctx *c, int prec) {
  DevState &s = c->ds;
  if (prec == PIKS_PREC_FP64) {
    release(c, s.h); release(c, s.fw);
    for (int b = 0; b < 2; ++b) { release(c, s.ghostW[b]); release(c, s.ghostE[b]); s.ghostW[b] = s.ghostE[b] = nullptr; }
    s.h = s.fw = nullptr;
    for (int side = 0; side < 2; ++side) {
      for (int b = 0; b < 2; ++b) { release(c, s.hsend[side][b]); s.hsend[side][b] = nullptr; }
      release(c, s.hrecv[side]);
      s.hrecv[side] = nullptr;
    }
  } else {
    release(c, s.h32); release(c, s.fw32);
    for (int b = 0; b < 2; ++b) { release(c, s.ghostW32[b]); release(c, s.ghostE32[b]); s.ghostW32[b] = s.ghostE32[b] = nullptr; }
    s.h32 = s.fw32 = nullptr;
    for (int side = 0; side < 2; ++side) {
      for (int b = 0; b < 2; ++b) { release(c, s.hsend32[side][b]); s.hsend32[side][b] = nullptr; }
      release(c, s.hrecv32[side]);
      s.hrecv32[side] = nullptr;
    }
  }
}

// Event-timed launch of one kernel group when timing is on.
struct Timed {
  piks_ctx *c;
  int k;
  cudaEvent_t a = nullptr, b = nullptr;
  Timed(piks_ctx *cc, int kk) : c(cc), k(kk) {
    if (!c->timing) return;
    if (c->ev_next + 2 > c->ev_pool.size()) {
      for (int i = 0; i < 64; ++i) { cudaEvent_t e; cudaEventCreate(&e); c->ev_pool.push_back(e); }
    }
    a = c->ev_pool[c->ev_next++];
    b = c->ev_pool[c->ev_next++];
    cudaEventRecord(a, c->stream);
  }
  ~Timed() {
    if (!c->timing) return;
    cudaEventRecord(b, c->stream);
    c->pending.push_back({k, {a, b}});
  }
};

void drain_timing(piks_ctx *c) {
  if (c->pending.empty()) return;
  cudaStreamSynchronize(c->stream);
  for (auto &p : c->pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.second.first, p.second.second);
    c->kt_ms[p.first] += ms;
    c->kt_n[p.first] += 1;
  }
  c->pending.clear();
  c->ev_next = 0;
}

// The tile sweeps' error flag: set when a dependency wait or a staging wait gave up (the
// values of that sweep are then not the solver's).
piks_status check_sweep_error(piks_ctx *c) {
  if (!c->use_tiles || !c->ds.tv.err) return PIKS_OK;
  int e = 0;
  piks_status st = cuda_check(cudaMemcpyAsync(&e, c->ds.tv.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "err D2H");
  if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "err sync");
  if (st) return st;
  if (e) return fail(PIKS_ERR_CUDA, "tile sweep: a dependency wait timed out");
  return PIKS_OK;
}

// The boundary part of iteration n (solver.F90:535-1938): switch commits, halo capture,
// walls, inlet/outlet, symmetry, moments, on stream st.
void enqueue_boundaries_timed(piks_ctx *c, cudaStream_t st, int n) {
  DevState &s = c->ds;
  const int cap = n & 1, prev = (n - 1) & 1;
  const bool f32 = c->prec == PIKS_PREC_FP32;
  { Timed t(c, KT_COMMIT); f32 ? launch_commit32(s, st) : launch_commit(s, st); }
  {
    Timed t(c, KT_CAPTURE);
    f32 ? launch_capture32(s, cap, st) : launch_capture(s, cap, st);
    if (c->setup.nranks > 1) launch_halo(s, f32, cap, st);  // solver.F90:535-560 on a slab
  }
  {
    Timed t(c, KT_WALLS);
    const auto &ls = c->geo.level_start;
    for (size_t L = 0; L + 1 < ls.size(); ++L) {
      if (f32) launch_walls32(s, ls[L], ls[L + 1], prev, st);
      else launch_walls(s, ls[L], ls[L + 1], prev, st);
    }
  }
  { Timed t(c, KT_INLET); f32 ? launch_inlet_outlet32(s, prev, st) : launch_inlet_outlet(s, prev, st); }
  { Timed t(c, KT_SYM); f32 ? launch_symmetry32(s, st) : launch_symmetry(s, st); }
  { Timed t(c, KT_MOM); f32 ? launch_moments32(s, st) : launch_moments(s, st); }
}

// The eight octant sweeps (solver.F90:176-526) of iteration n on stream st.
void enqueue_sweep(piks_ctx *c, cudaStream_t st, int n) {
  DevState &s = c->ds;
  const bool f32 = c->prec == PIKS_PREC_FP32;
  {
    Timed t(c, KT_SWEEP);
    if (c->use_tiles && c->tiles.split) {
      if (c->tiles.columns) launch_tile_sweep_columns(s, f32, 1, st);
      else launch_tile_sweep_pipelined(s, f32, 1, st);
    } else if (c->use_tiles && c->schedule == PIKS_SCHED_TILE_DATAFLOW) {
      launch_tile_sweep_dataflow(s, f32, n, c->tiles.max_rows, c->tiles.max_tasks, st);
    } else if (c->use_tiles) {
      const auto &L = c->tiles.launches;
      for (size_t k = 0; k + 3 < L.size(); k += 4)
        launch_tile_sweep(s, f32, L[k], L[k + 1], L[k + 2], L[k + 3], k > 0, st);
    } else {
      const auto &hs = c->geo.hyper_start;
      for (size_t h = 0; h + 1 < hs.size(); ++h) {
        if (f32) launch_sweep_hyperplane32(s, hs[h], hs[h + 1] - hs[h], st);
        else launch_sweep_hyperplane(s, hs[h], hs[h + 1] - hs[h], st);
      }
    }
  }
}

void drop_graphs(piks_ctx *c) {
  for (auto &g : c->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  c->graph_key = -1;
  c->graph_warm = 0;
}

// One source iteration (solver.F90:111-1940) as a launch sequence on the context stream.
void enqueue_iteration(piks_ctx *c) {
  const int n = c->iStep + 1;          // the iteration being run (1-based)
  enqueue_sweep(c, c->stream, n);
  enqueue_boundaries_timed(c, c->stream, n);
  c->iStep = n;
  if (c->timing && c->pending.size() > 4096) drain_timing(c);
}

// Tile schedule of the context's tile_dims on the host (false: not usable, e.g. a job needs
// more shared memory than a block has).
// Shared-memory rows a tile job may use: what both precisions' sweep kernels can hold.
int tile_slots(const piks_ctx *c, const int *dims) {
  const int vox = dims[0] * dims[1] * dims[2];
  const int nst = dims[0] + dims[1] + dims[2] - 2;
  return std::min(tile_sweep_max_slots(c->vel.Nc8, false, vox, nst), tile_sweep_max_slots(c->vel.Nc8, true, vox, nst));
}

// Default tile shape of a precision, measured fastest on B200 for 512 velocities: 8x4x4
// for the FP64 sweep, 4x4x4 for the FP32 sweep (whose CTAs carry twice the velocities per row).
void default_tile_dims(int prec, int *dims) {
  dims[0] = prec == PIKS_PREC_FP32 ? 4 : 8;
  dims[1] = 4;
  dims[2] = 4;
}

// Waits for a background tile build and drops its result.
void drop_tiles_next(piks_ctx *c) {
  if (c->tiles_next_ready.valid()) c->tiles_next_ready.wait();
  c->tiles_next_ready = std::future<bool>();
  c->tiles_next = TileJobs{};
  c->tiles_next_dims[0] = c->tiles_next_dims[1] = c->tiles_next_dims[2] = 0;
}

// TileView fields of the column form that size the column kernel's shared memory.
TileView column_sizes(const TileJobs &tj) {
  TileView tv{};
  tv.max_tasks = tj.max_tasks;
  tv.max_nrows = tj.max_rows - 1;
  tv.steps_stride = tj.steps_stride;
  tv.max_carry = tj.max_carry;
  tv.ncells = tj.ncells;
  tv.max_region = tj.max_region;
  tv.mean_region = tj.row_count.empty() ? 0.f : (float)((double)tj.sum_region / (double)tj.row_count.size());
  return tv;
}

// Form of the tile jobs a launch schedule reads.
int tile_form(int schedule) {
  return schedule == PIKS_SCHED_TILE_COLUMNS ? TILE_FORM_COLUMNS
         : schedule == PIKS_SCHED_TILE_PIPELINED ? TILE_FORM_SPLIT
                                                  : TILE_FORM_SLOTS;
}

// Tile jobs for a tile shape in the given form (the split forms fall back to the slot form
// when the producer / consumer kernel cannot hold the largest job in shared memory).
bool build_tiles_for(const piks_ctx *c, const int *dims, int form, TileJobs &tj, int prec) {
  tj = TileJobs{};
  if (dims[0] <= 0) return false;
  if (form != TILE_FORM_SLOTS) {
    if (build_tile_jobs(c->geo, dims[0], dims[1], dims[2], 65535, tj, form) &&
        column_sweep_fits(column_sizes(tj), c->vel.Nc8, false) && column_sweep_fits(column_sizes(tj), c->vel.Nc8, true))
      return true;
    tj = TileJobs{};
  }
  const bool ok = build_tile_jobs(c->geo, dims[0], dims[1], dims[2], tile_slots(c, dims), tj);
  if (!ok) tj = TileJobs{};
  else plan_for_precision(tj, prec);
  return ok;
}

bool build_tiles(piks_ctx *c) {
  c->use_tiles = build_tiles_for(c, c->tile_dims, tile_form(c->schedule), c->tiles, c->prec);
  return c->use_tiles;
}

// Device copy of the tile schedule (replacing an earlier one), with zeroed dataflow flags.
piks_status upload_tiles(piks_ctx *c) {
  DevState &s = c->ds;
  TileView &tv = s.tv;
  for (const void *p : {(const void *)tv.rows, (const void *)tv.row_begin, (const void *)tv.row_count,
                        (const void *)tv.tasks, (const void *)tv.task_begin, (const void *)tv.steps,
                        (const void *)tv.job_list, (const void *)tv.up, (const void *)tv.flags,
                        (const void *)tv.counter, (const void *)tv.hdr, (const void *)tv.carry,
                        (const void *)tv.col_jobs, (const void *)tv.col_begin, (const void *)tv.col_list})
    if (p) release(c, const_cast<void *>(p));
  tv = TileView{};
  piks_status st;
  if (!c->use_tiles) {
    // the per-node hyperplane sweep reads the task list (uploaded once, only if needed)
    if (!c->ds.tasks) {
      int32_t *pt = nullptr;
      if ((st = upload(c, c->geo.tasks, &pt))) return st;
      c->ds.tasks = pt;
    }
    return PIKS_OK;
  }
  const TileJobs &tj = c->tiles;
  int32_t *pi = nullptr;
  int64_t *p64 = nullptr;
  uint16_t *p16 = nullptr;
#define UPT(vec, field, ptr) do { if ((st = upload(c, vec, &ptr))) return st; tv.field = ptr; } while (0)
  UPT(tj.rows, rows, pi);
  UPT(tj.row_begin, row_begin, p64);
  UPT(tj.row_count, row_count, pi);
  if ((st = upload(c, tj.tasks, &pi))) return st;
  tv.tasks = reinterpret_cast<const int4 *>(pi);
  UPT(tj.task_begin, task_begin, p64);
  UPT(tj.steps, steps, p16);
  UPT(tj.job_list, job_list, pi);
  UPT(tj.up, up, pi);
#undef UPT
  tv.njobs = (int)(tj.row_count.size());
  int *pw = nullptr;
  // one more job's worth of flags than jobs: that job never publishes (wait self-test)
  if ((st = zeros(c, (size_t)(tv.njobs + 1) * (size_t)(c->vel.Nc8 / 8 > 0 ? c->vel.Nc8 / 8 : 1), &pw))) return st;
  tv.flags = pw;
  if ((st = zeros(c, (size_t)2, &pw))) return st;
  tv.counter = pw;
  tv.err = pw + 1;
  tv.nsteps = tj.nsteps;
  tv.steps_stride = tj.steps_stride;
  tv.paired = tj.paired ? 1 : 0;
  if (tj.split) {
    const TileView sz = column_sizes(tj);
    tv.max_tasks = sz.max_tasks; tv.max_nrows = sz.max_nrows; tv.max_carry = sz.max_carry;
    tv.ncells = sz.ncells; tv.max_region = sz.max_region; tv.mean_region = sz.mean_region;
#define UPC(vec, field) do { if ((st = upload(c, vec, &pi))) return st; tv.field = pi; } while (0)
    UPC(tj.hdr, hdr);
    UPC(tj.carry, carry);
    UPC(tj.col_jobs, col_jobs);
    UPC(tj.col_begin, col_begin);
    UPC(tj.col_list, col_list);
#undef UPC
    tv.ncols = (int)tj.col_list.size();
  }
  return PIKS_OK;
}

}  // namespace

namespace piks {

void enqueue_boundaries(piks_ctx *c, cudaStream_t st, int n) {
  const bool timing = c->timing;
  c->timing = false;
  enqueue_boundaries_timed(c, st, n);
  c->timing = timing;
}

void launch_check(piks_ctx *c, cudaStream_t st) {
  const double inv = 1.0 / c->setup.p.Ref_L;
  launch_flux(c->ds, c->setup.ds, std::sqrt(1.0 / 2.0), inv * inv, st);
}

// output.F90:151-155
void finish_check(piks_ctx *c, double m2) {
  const double kPi = std::atan(1.0) * 4.0;
  c->error = std::fabs(1.0 - m2 / c->mass) / (double)c->setup.p.chkConvergeStep;
  c->mass = m2;
  c->permeability = c->mass * c->setup.p.Kn * std::sqrt(4.0 / kPi);
}

}  // namespace piks

extern "C" {

const char *piks_last_error(void) { return g_last_error.c_str(); }
const char *piks_kernel_names(void) { return kKernelNames; }

piks_status piks_params_default(piks_params *p) {
  if (!p) return fail(PIKS_ERR_ARG, "null params");
  std::memset(p, 0, sizeof *p);
  // parameters.F90:91-98
  p->block_repx = p->block_repy = p->block_repz = 1;
  p->wallExtOrder = 2;
  p->fluidlayer = 0;
  p->Ref_L = 1.0;
  p->saveLast = 1;
  p->saveFormat = 1;
  p->halfRange = 1;
  p->mpi_xdim = p->mpi_ydim = p->mpi_zdim = 1;
  p->accom = 1.0;
  p->chkConvergeStep = 10;
  p->saveStep = 1 << 30;
  p->maxStep = 1000;
  p->eps = 1e-8;
  return PIKS_OK;
}

piks_status piks_read_params(const char *path, piks_params *p, char *image_file, int32_t len) {
  if (!path || !p) return fail(PIKS_ERR_ARG, "null argument");
  std::string img, err;
  piks_status st = read_namelist(path, *p, img, err);
  if (st) return fail(st, err);
  if (image_file && len > 0) {
    std::strncpy(image_file, img.c_str(), (size_t)len - 1);
    image_file[len - 1] = 0;
  }
  return PIKS_OK;
}

piks_status piks_create(const piks_params *p, int32_t device, piks_ctx **out) {
  if (!p || !out) return fail(PIKS_ERR_ARG, "null argument");
  *out = nullptr;
  if (device < -1) return fail(PIKS_ERR_ARG, "device index out of range");
  if (device >= 0) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PIKS_ERR_NOT_FOUND, "no CUDA device");
    if (device >= ndev) return fail(PIKS_ERR_ARG, "device index out of range");
  }
  auto *c = new piks_ctx();
  std::string err;
  piks_status st = make_setup(*p, c->setup, err);
  if (!st) st = make_velocity(*p, c->vel, err);
  if (st) { delete c; return fail(st, err); }
  c->device = device;
  if (device < 0) { *out = c; return PIKS_OK; }  // host-only context: preprocessing and getters
  st = cuda_check(cudaSetDevice(device), "cudaSetDevice");
  if (!st) st = cuda_check(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  if (st) { delete c; return st; }
  c->stream = c->own_stream;
  {
    // the wall programs in constant memory are the same for every context: once per device
    static std::mutex mu;
    static unsigned long long uploaded = 0;
    std::lock_guard<std::mutex> lock(mu);
    if (!(uploaded >> (device & 63) & 1ull)) {
      upload_tables();
      upload_tables_fp32();
      st = cuda_check(cudaGetLastError(), "upload_tables");
      if (st) { cudaStreamDestroy(c->own_stream); delete c; return st; }
      uploaded |= 1ull << (device & 63);
    }
  }
  *out = c;
  return PIKS_OK;
}

piks_status piks_setup_physical_grid(piks_ctx *c, const uint8_t *raw, int64_t nbytes) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  const auto t_setup = std::chrono::steady_clock::now();
  drop_tiles_next(c);
  if (c->device >= 0) { cudaSetDevice(c->device); free_device(c); }
  c->have_host_geometry = false;
  std::string err;
  piks_status st;
  {
    // the box on the host (its drill / thin passes depend on the raster order), the voxel
    // classification on the device when the context has one, the rest on the host
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    std::vector<uint8_t> box;
    st = preprocess_box(c->setup, raw, nbytes, box, err);
    if (st) return fail(st, err);
    const auto t1 = clk::now();
    // (a slab of an x-decomposed box is classified on the host: its node set includes the
    // read voxels of the neighbour ranks' planes)
    if (c->device >= 0 && c->prep == PIKS_PREP_DEVICE && c->setup.nranks == 1) {
      st = classify_device(c->setup, box, c->geo, c->stream, err);
      if (st) return fail(st, err);
    } else {
      classify_host(c->setup, box, c->geo);
    }
    const auto t2 = clk::now();
    st = finish_geometry(c->setup, c->geo, err);
    if (st) return fail(st, err);
    const auto t3 = clk::now();
    c->setup_seconds[0] = std::chrono::duration<double>(t1 - t0).count();
    c->setup_seconds[1] = std::chrono::duration<double>(t2 - t1).count();
    c->setup_seconds[2] = std::chrono::duration<double>(t3 - t2).count();
  }
  c->have_host_geometry = true;
  c->tiles_tuned = false;
  if (!c->tiles_explicit) default_tile_dims(c->prec, c->tile_dims);
  build_tiles(c);
  if (c->device < 0) {
    c->setup_seconds[3] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_setup).count();
    return PIKS_OK;
  }
  const Geometry &g = c->geo;
  const Velocity &v = c->vel;
  DevState &s = c->ds;
  s = DevState{};
  s.Nx = g.Nx; s.Ny = g.Ny; s.Nz = g.Nz; s.GX = g.GX; s.GXY = g.GX * g.GY;
  s.NF = g.NF; s.NB = g.NB; s.Nc8 = v.Nc8;
  s.lpt = v.Nc8 >= 32 ? 32 : 8;   // lanes per sweep task (2 velocities per lane when 32)
  s.nchunk = s.lpt == 32 ? (v.Nc8 + 63) / 64 : (v.Nc8 + 7) / 8;
  const double ds = c->setup.ds;
  s.mu = c->setup.mu;
  s.c15 = 1.5 / ds; s.c20 = 2.0 / ds; s.c05 = -0.5 / ds; s.c10 = 1.0 / ds;
  s.accom = c->setup.p.accom; s.pressDrop = c->setup.p.pressDrop; s.DiffFlux = v.DiffFlux;
  const size_t nnodes = (size_t)g.NF + g.NB;
  int32_t *pi = nullptr; uint8_t *pu8 = nullptr; uint16_t *pu16 = nullptr; double *pd = nullptr;
#define UP(vec, field, ptr) do { st = upload(c, vec, &ptr); if (st) return st; s.field = ptr; } while (0)
  UP(g.nodemap, nodemap, pi);
  UP(g.label, label, pu8);
  UP(g.bcorner, bcorner, pi);
  UP(g.roles, roles, pu16);
  UP(v.cx, cx, pd); UP(v.cy, cy, pd); UP(v.cz, cz, pd); UP(v.w, w, pd);
  UP(g.wall_node, wall_node, pi); UP(g.wall_label, wall_label, pi); UP(g.wall_corner, wall_corner, pi);
  UP(g.wall_nb, wall_nb, pi); UP(g.wall_order, wall_order, pi); UP(g.wall_e, wall_e, pd);
  {
    std::vector<int32_t> rec(g.wall_order.size() * 16, 0);
    for (size_t w = 0; w < g.wall_order.size(); ++w) {
      const size_t q = (size_t)g.wall_order[w];
      int32_t *r = &rec[w * 16];
      r[0] = g.wall_node[q]; r[1] = g.wall_corner[q]; r[2] = g.wall_label[q];
      std::memcpy(r + 4, &g.wall_e[2 * q], 2 * sizeof(double));
      for (int k = 0; k < 6; ++k) r[8 + k] = g.wall_nb[6 * q + k];
    }
    if ((st = upload(c, rec, &pi))) return st;
    s.wall_rec = reinterpret_cast<const int4 *>(pi);
  }
  UP(g.commit, commit, pi);
  UP(g.plane_x1, plane_x1, pi); UP(g.plane_xN, plane_xN, pi);
  UP(g.sym_node, sym_node, pi); UP(g.sym_flag, sym_flag, pu8);
  UP(g.flux_list, flux_list, pi);
  for (int side = 0; side < 2; ++side) {
    s.nhalo_send[side] = (int)g.halo_send[side].size();
    s.nhalo_recv[side] = (int)g.halo_recv[side].size();
    if (s.nhalo_send[side]) UP(g.halo_send[side], halo_send[side], pi);
    if (s.nhalo_recv[side]) UP(g.halo_recv[side], halo_recv[side], pi);
  }
  {
    // per-velocity sweep constants: cx cy cz w; the products c*C of the upwind terms
    // (C1 = 2/ds second order, 1/ds first order; C2 = -0.5/ds) for x, y, z; the
    // denominators 0.5*mu + cx*C0x + cy*C0y + cz*C0z (solver.F90:214) by first-order
    // class (C0 = 1.5/ds or 1/ds) and their correctly rounded reciprocals
    std::vector<double> vt((size_t)kVtab * v.Nc8);
    const double c15 = 1.5 / ds, c20 = 2.0 / ds, c05 = -0.5 / ds, c10 = 1.0 / ds;
    for (int l = 0; l < v.Nc8; ++l) {
      double *t = &vt[(size_t)l * kVtab];
      t[0] = v.cx[l]; t[1] = v.cy[l]; t[2] = v.cz[l]; t[3] = v.w[l];
      t[4] = v.cx[l] * c20; t[5] = v.cx[l] * c10; t[6] = v.cx[l] * c05;
      t[7] = v.cy[l] * c20; t[8] = v.cy[l] * c10; t[9] = v.cy[l] * c05;
      t[10] = v.cz[l] * c20; t[11] = v.cz[l] * c10; t[12] = v.cz[l] * c05;
      for (int cls = 0; cls < 8; ++cls) {
        double den = 0.5 * s.mu;
        den = den + v.cx[l] * ((cls & 1) ? c10 : c15);
        den = den + v.cy[l] * ((cls & 2) ? c10 : c15);
        den = den + v.cz[l] * ((cls & 4) ? c10 : c15);
        t[13 + cls] = den;
        t[21 + cls] = 1.0 / den;
      }
    }
    UP(vt, vtab, pd);
    {
      std::vector<float> v32(vt.begin(), vt.end());
      float *pf = nullptr;
      if ((st = upload(c, v32, &pf))) return st;
      s.vtab32 = pf;
    }
    if (v.Nc8 % 2 == 0) {
      std::vector<double> v2((size_t)kVtab * v.Nc8);
      for (int l = 0; l < v.Nc8; l += 2)
        for (int k = 0; k < kVtab; ++k) {
          v2[((size_t)(l / 2) * kVtab + k) * 2 + 0] = vt[(size_t)l * kVtab + k];
          v2[((size_t)(l / 2) * kVtab + k) * 2 + 1] = vt[(size_t)(l + 1) * kVtab + k];
        }
      const double *pv2 = nullptr;
      st = upload(c, v2, &pd);
      if (st) return st;
      pv2 = pd;
      s.vtab2 = reinterpret_cast<const double2 *>(pv2);
    }
  }
#undef UP
  if ((st = upload_tiles(c))) return st;
  s.nWall = g.nWall;
  s.ncommit = (int)(g.commit.size() / 3);
  s.nsym = (int)g.sym_node.size();
  for (int i = 0; i < 10; ++i) s.flux_groups[i] = g.flux_groups[i];
  (void)nnodes;
  if ((st = alloc_state(c, c->prec))) return st;
  if ((st = zeros(c, (size_t)g.NF * 4, &s.mom))) return st;                      // flow.F90:93-96
  if ((st = zeros(c, (size_t)1, &s.flux_out))) return st;
  st = cuda_check(cudaStreamSynchronize(c->stream), "setup");
  if (st) return st;
  c->have_geometry = true;
  c->version += 1;
  c->iStep = 0;
  if (c->prec == PIKS_PREC_FP32 && c->use_tiles && !c->tiles_explicit) {
    // a refined solve switches to FP64 later: its schedule is built meanwhile
    default_tile_dims(PIKS_PREC_FP64, c->tiles_next_dims);
    const int slots = tile_slots(c, c->tiles_next_dims);
    (void)slots;
    const int form = tile_form(c->schedule);
    c->tiles_next_ready = std::async(std::launch::async, [c, form] {
      return build_tiles_for(c, c->tiles_next_dims, form, c->tiles_next, PIKS_PREC_FP64);
    });
  }
  c->mass = 1.0;  // flow.F90:97
  c->error = 1.0;
  c->permeability = 0.0;
  c->setup_seconds[3] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_setup).count();
  return PIKS_OK;
}

piks_status piks_iterate(piks_ctx *c, int32_t nsteps) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  if (c->device < 0) return fail(PIKS_ERR_NOT_FOUND, "host-only context (device -1) cannot iterate");
  if (!c->have_geometry) return fail(PIKS_ERR_STATE, "piks_setup_physical_grid has not been called");
  if (nsteps < 0) return fail(PIKS_ERR_ARG, "nsteps < 0");
  if (c->setup.nranks > 1 && nsteps > 1)
    return fail(PIKS_ERR_ARG, "a slab context iterates one step per call (its halos are exchanged between calls)");
  cudaSetDevice(c->device);
  // The dataflow sweep takes the iteration number as its epoch and per-kernel timing records
  // events, so both launch plainly; otherwise one graph launch per iteration replaces about
  // a hundred kernel launches (the host would otherwise leave the GPU idle after every
  // convergence check while it re-fills the stream).
  const bool graphs = !c->graph_failed && !c->timing && !(c->use_tiles && c->schedule == PIKS_SCHED_TILE_DATAFLOW);
  for (int n = 0; n < nsteps; ++n) {
    if (!graphs) { enqueue_iteration(c); continue; }
    const int key = c->version * 8 + c->schedule;
    if (key != c->graph_key) { drop_graphs(c); c->graph_key = key; }
    if (c->graph_warm < 2) { enqueue_iteration(c); ++c->graph_warm; continue; }
    const int it = c->iStep + 1;
    const int par = it & 1;
    if (!c->graph[par]) {
      if (!c->cap_stream && cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        c->graph_failed = true;
        enqueue_iteration(c);
        continue;
      }
      cudaGraph_t g = nullptr;
      bool ok = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
        enqueue_sweep(c, c->cap_stream, it);
        enqueue_boundaries_timed(c, c->cap_stream, it);
        ok = cudaStreamEndCapture(c->cap_stream, &g) == cudaSuccess && g;
      }
      if (ok) ok = cudaGraphInstantiate(&c->graph[par], g, 0) == cudaSuccess;
      if (g) cudaGraphDestroy(g);
      if (!ok) {  // plain launches from here on
        cudaGetLastError();
        c->graph[par] = nullptr;
        c->graph_failed = true;
        enqueue_iteration(c);
        continue;
      }
    }
    piks_status st = cuda_check(cudaGraphLaunch(c->graph[par], c->stream), "iteration graph launch");
    if (st) return st;
    c->iStep = it;
  }
  return cuda_check(cudaGetLastError(), "iterate launch");
}

piks_status piks_chk_converge(piks_ctx *c, double *mass, double *perm, double *err) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  if (!c->have_geometry) return fail(PIKS_ERR_STATE, "piks_setup_physical_grid has not been called");
  cudaSetDevice(c->device);
  if (!c->geo.wglob) {
    // output.F90:89: only the west-most slab computes the check; the others keep their values
    piks_status st = check_sweep_error(c);
    if (st) return st;
    if (mass) *mass = c->mass;
    if (perm) *perm = c->permeability;
    if (err) *err = c->error;
    return PIKS_OK;
  }
  {
    Timed t(c, KT_FLUX);
    launch_check(c, c->stream);
  }
  double m2 = 0.0;
  piks_status st = cuda_check(cudaMemcpyAsync(&m2, c->ds.flux_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "flux D2H");
  if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "flux sync");
  if (!st) st = check_sweep_error(c);
  if (st) return st;
  finish_check(c, m2);
  if (mass) *mass = c->mass;
  if (perm) *perm = c->permeability;
  if (err) *err = c->error;
  return PIKS_OK;
}

piks_status piks_get_macro(piks_ctx *c, double *rho, double *ux, double *uy, double *uz) {
  if (!c || !c->have_geometry) return fail(PIKS_ERR_STATE, "no geometry");
  cudaSetDevice(c->device);
  const Geometry &g = c->geo;
  std::vector<double> tmp((size_t)g.NF * 4);
  double *dst[4] = {rho, ux, uy, uz};
  const size_t box = (size_t)g.Nx * g.Ny * g.Nz;
  piks_status st = cuda_check(cudaMemcpyAsync(tmp.data(), c->ds.mom, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "macro D2H");
  if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "macro sync");
  if (st) return st;
  for (int q = 0; q < 4; ++q) {
    if (!dst[q]) continue;
    std::memset(dst[q], 0, box * sizeof(double));
    for (int32_t n = 0; n < g.NF; ++n) {
      int64_t gi = g.node_g[n];
      int i = (int)(gi % g.GX) - 1, j = (int)((gi / g.GX) % g.GY) - 1, k = (int)(gi / ((int64_t)g.GX * g.GY)) - 1;
      dst[q][(size_t)(i - 1) + (size_t)(j - 1) * g.Nx + (size_t)(k - 1) * g.Nx * g.Ny] = tmp[(size_t)n * 4 + q];
    }
  }
  return PIKS_OK;
}

piks_status piks_get_labels(piks_ctx *c, int32_t *labels) {
  if (!c || !c->have_host_geometry || !labels) return fail(PIKS_ERR_STATE, "no geometry");
  const Geometry &g = c->geo;
  for (int k = 1; k <= g.Nz; ++k)
    for (int j = 1; j <= g.Ny; ++j)
      for (int i = 1; i <= g.Nx; ++i)
        labels[(size_t)(i - 1) + (size_t)(j - 1) * g.Nx + (size_t)(k - 1) * g.Nx * g.Ny] = g.label[g.ghost_index(i, j, k)];
  return PIKS_OK;
}

piks_status piks_get_info(piks_ctx *c, int64_t *info, int32_t n) {
  if (!c || !info) return fail(PIKS_ERR_ARG, "null argument");
  const Geometry &g = c->geo;
  int64_t v[11] = {c->setup.Nx, c->setup.Ny, c->setup.Nz, c->vel.Nc8, g.NF, g.nWall, g.nCorner,
                   (int64_t)g.NF + g.NB, c->iStep, (int64_t)(g.level_start.empty() ? 0 : g.level_start.size() - 1),
                   (int64_t)c->dev_bytes};
  for (int i = 0; i < n && i < 11; ++i) info[i] = v[i];
  return PIKS_OK;
}

piks_status piks_get_f(piks_ctx *c, double *f_ref, double *fw) {
  if (!c || !c->have_geometry) return fail(PIKS_ERR_STATE, "no geometry");
  cudaSetDevice(c->device);
  const Geometry &g = c->geo;
  const int Nc8 = c->vel.Nc8;
  const size_t nnodes = (size_t)g.NF + g.NB;
  piks_status st;
  const bool f32 = c->prec == PIKS_PREC_FP32;
  if (f_ref) {
    std::vector<double> h(nnodes * 8 * Nc8);
    if (f32) {
      std::vector<float> h32(h.size());
      st = cuda_check(cudaMemcpyAsync(h32.data(), c->ds.h32, h32.size() * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "f D2H");
      if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "f sync");
      if (st) return st;
      std::copy(h32.begin(), h32.end(), h.begin());
    } else {
      st = cuda_check(cudaMemcpyAsync(h.data(), c->ds.h, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "f D2H");
      if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "f sync");
      if (st) return st;
    }
    const size_t Ntot = (size_t)g.GX * g.GY * g.GZ;
    std::memset(f_ref, 0, Ntot * Nc8 * 8 * sizeof(double));
    for (size_t n = 0; n < nnodes; ++n)
      for (int o = 0; o < 8; ++o)
        for (int l = 0; l < Nc8; ++l)
          f_ref[(size_t)g.node_g[n] + (size_t)l * Ntot + (size_t)o * Ntot * Nc8] = h[(n * 8 + o) * Nc8 + l];
  }
  if (fw && g.nCorner > 0) {
    std::vector<double> t((size_t)g.nCorner * 8 * Nc8);
    if (f32) {
      std::vector<float> t32(t.size());
      st = cuda_check(cudaMemcpyAsync(t32.data(), c->ds.fw32, t32.size() * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "fw D2H");
      if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "fw sync");
      if (st) return st;
      std::copy(t32.begin(), t32.end(), t.begin());
    } else {
      st = cuda_check(cudaMemcpyAsync(t.data(), c->ds.fw, t.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "fw D2H");
      if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "fw sync");
      if (st) return st;
    }
    for (int cc = 0; cc < g.nCorner; ++cc)
      for (int o = 0; o < 8; ++o)
        for (int l = 0; l < Nc8; ++l)
          fw[(size_t)cc + (size_t)l * g.nCorner + (size_t)o * g.nCorner * Nc8] = t[((size_t)cc * 8 + o) * Nc8 + l];
  }
  return PIKS_OK;
}

piks_status piks_get_f_nodes(piks_ctx *c, const int32_t *nodes, int32_t n, double *out) {
  if (!c || !c->have_geometry) return fail(PIKS_ERR_STATE, "no geometry");
  if (n < 0 || (n > 0 && (!nodes || !out))) return fail(PIKS_ERR_ARG, "bad node list");
  cudaSetDevice(c->device);
  const Geometry &g = c->geo;
  const size_t row = (size_t)8 * c->vel.Nc8;
  const bool f32 = c->prec == PIKS_PREC_FP32;
  std::vector<float> t32(f32 ? row : 0);
  for (int32_t q = 0; q < n; ++q) {
    if (nodes[q] < 0 || (int64_t)nodes[q] >= (int64_t)g.NF + g.NB) return fail(PIKS_ERR_ARG, "node index out of range");
    piks_status st;
    if (f32) {
      st = cuda_check(cudaMemcpyAsync(t32.data(), c->ds.h32 + (size_t)nodes[q] * row, row * sizeof(float),
                                      cudaMemcpyDeviceToHost, c->stream), "f rows D2H");
      if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "f rows sync");
      if (!st) std::copy(t32.begin(), t32.end(), out + (size_t)q * row);
    } else {
      st = cuda_check(cudaMemcpyAsync(out + (size_t)q * row, c->ds.h + (size_t)nodes[q] * row, row * sizeof(double),
                                      cudaMemcpyDeviceToHost, c->stream), "f rows D2H");
    }
    if (st) return st;
  }
  return cuda_check(cudaStreamSynchronize(c->stream), "f rows sync");
}

piks_status piks_save_fields(piks_ctx *c, const char *dir, int32_t format) {
  if (!c || !c->have_geometry) return fail(PIKS_ERR_STATE, "no geometry");
  const Geometry &g = c->geo;
  const size_t box = (size_t)g.Nx * g.Ny * g.Nz;
  std::vector<double> r(box), u(box), v(box), w(box);
  piks_status st = piks_get_macro(c, r.data(), u.data(), v.data(), w.data());
  if (st) return st;
  std::string err;
  bool ok = true;
  write_fields(c->setup, g, r.data(), u.data(), v.data(), w.data(), dir ? dir : ".", format, err, ok);
  if (!ok) return fail(PIKS_ERR_IO, err);
  return PIKS_OK;
}

}  // extern "C"

namespace {

// chkConverge at `step` with main.F90's stdout line (:104-107) and Results.dat line
// (output.F90:157-159).
piks_status check_and_report(piks_ctx *c, int step, const char *results_path, int verbose) {
  const piks_params &p = c->setup.p;
  piks_status st = piks_chk_converge(c, nullptr, nullptr, nullptr);
  if (st) return st;
  if (verbose)
    std::printf("%10d%s%s%s\n", step, fortran_es15_6(c->mass).c_str(), fortran_es15_6(c->permeability).c_str(),
                fortran_es15_6(c->error).c_str());
  if (results_path && results_path[0]) {
    FILE *fh = std::fopen(results_path, "a");
    if (!fh) return fail(PIKS_ERR_IO, std::string("cannot open ") + results_path);
    std::fprintf(fh, "%s%s%s%s%15d\n", fortran_es15_6(p.Kn).c_str(), fortran_es15_6(c->mass).c_str(),
                 fortran_es15_6(c->permeability).c_str(), fortran_es15_6(c->error).c_str(), step);
    std::fclose(fh);
  }
  return PIKS_OK;
}

// main.F90:98-121 from iteration first_step on; stops at error <= eps, at maxStep, or (when
// stop_on_stall) once the error has gone 5 checks without a new minimum. Returns the last
// iteration run in *last.
piks_status run_loop(piks_ctx *c, int first_step, double eps, bool stop_on_stall, const char *results_path,
                     const char *out_dir, int verbose, int *last) {
  if (c->setup.nranks > 1)
    return fail(PIKS_ERR_STATE, "a slab context is driven by its host (one iteration and one halo exchange at a time)");
  const piks_params &p = c->setup.p;
  piks_status st;
  double best = HUGE_VAL;
  int since_best = 0;
  int step = first_step;
  for (; step <= p.maxStep; ++step) {
    if ((st = piks_iterate(c, 1))) return st;
    if (step % p.chkConvergeStep == 0) {
      if ((st = check_and_report(c, step, results_path, verbose))) return st;
      if (c->error < best) { best = c->error; since_best = 0; } else ++since_best;
    }
    if (out_dir && p.saveStep > 0 && step % p.saveStep == 0)
      if ((st = piks_save_fields(c, out_dir, p.saveFormat))) return st;
    if (c->error <= eps) {
      if (step < p.chkConvergeStep) {
        if ((st = piks_chk_converge(c, nullptr, nullptr, nullptr))) return st;
      }
      break;
    }
    if (stop_on_stall && since_best >= 5) break;
  }
  *last = step > p.maxStep ? p.maxStep : step;
  return PIKS_OK;
}

}  // namespace

extern "C" {

piks_status piks_run(piks_ctx *c, const char *results_path, const char *out_dir, int32_t verbose,
                     int32_t *steps, double *perm, double *seconds) {
  if (!c || !c->have_geometry) return fail(PIKS_ERR_STATE, "no geometry");
  const piks_params &p = c->setup.p;
  c->error = 1.0;  // main.F90:95
  auto t0 = std::chrono::steady_clock::now();
  int step = 0;
  piks_status st = run_loop(c, 1, p.eps, false, results_path, out_dir, verbose, &step);
  if (st) return st;
  // the reference's loop variable ends one past maxStep when the loop runs out
  if (c->error > p.eps) step = p.maxStep + 1;
  cudaStreamSynchronize(c->stream);
  double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (verbose) {
    char wt[32];
    std::snprintf(wt, sizeof wt, "%11.3E", secs);
    std::printf("Walltime= %s, Steps= %6d, K= %s\n", wt, step, fortran_es15_6(c->permeability).c_str());
  }
  if (out_dir && p.saveLast)
    if ((st = piks_save_fields(c, out_dir, p.saveFormat))) return st;
  if (steps) *steps = step;
  if (perm) *perm = c->permeability;
  if (seconds) *seconds = secs;
  return PIKS_OK;
}

// After a precision switch: the new precision's default tile shape, from the background
// build when it made that shape, else built now (the schedule does not change any value).
static piks_status retile_for_precision(piks_ctx *c) {
  int d[3];
  default_tile_dims(c->prec, d);
  if (d[0] == c->tile_dims[0] && d[1] == c->tile_dims[1] && d[2] == c->tile_dims[2]) return PIKS_OK;
  TileJobs tj;
  bool ok = false;
  if (c->tiles_next_ready.valid() && d[0] == c->tiles_next_dims[0] && d[1] == c->tiles_next_dims[1] &&
      d[2] == c->tiles_next_dims[2]) {
    ok = c->tiles_next_ready.get();
    if (ok) tj = std::move(c->tiles_next);
  } else {
    ok = build_tiles_for(c, d, tile_form(c->schedule), tj, c->prec);
  }
  drop_tiles_next(c);
  if (!ok) return PIKS_OK;  // keep the current schedule
  c->tiles = std::move(tj);
  c->tile_dims[0] = d[0]; c->tile_dims[1] = d[1]; c->tile_dims[2] = d[2];
  piks_status st = upload_tiles(c);
  if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "retile");
  return st;
}

piks_status piks_set_precision(piks_ctx *c, int32_t precision) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  if (precision != PIKS_PREC_FP64 && precision != PIKS_PREC_FP32) return fail(PIKS_ERR_ARG, "unknown precision");
  if (c->device < 0 || !c->have_geometry || precision == c->prec) { c->prec = precision; return PIKS_OK; }
  cudaSetDevice(c->device);
  piks_status st = cuda_check(cudaStreamSynchronize(c->stream), "precision sync");
  if (st) return st;
  if (c->snap) {  // snapshots of the other precision are of no further use: free them first
    release(c, c->snap);
    c->snap = nullptr;
    c->snap_bytes = 0;
  }
  if ((st = alloc_state(c, precision))) { free_state(c, precision); return st; }
  DevState &s = c->ds;
  const StateSizes z = state_sizes(c);
  if (precision == PIKS_PREC_FP64) {
    launch_widen(s.h32, s.h, z.h, c->stream);
    launch_widen(s.fw32, s.fw, z.fw, c->stream);
    for (int b = 0; b < 2; ++b) {
      launch_widen(s.ghostW32[b], s.ghostW[b], z.plane, c->stream);
      launch_widen(s.ghostE32[b], s.ghostE[b], z.plane, c->stream);
      for (int side = 0; side < 2; ++side) launch_widen(s.hsend32[side][b], s.hsend[side][b], z.hsend[side], c->stream);
    }
  } else {
    launch_narrow(s.h, s.h32, z.h, c->stream);
    launch_narrow(s.fw, s.fw32, z.fw, c->stream);
    for (int b = 0; b < 2; ++b) {
      launch_narrow(s.ghostW[b], s.ghostW32[b], z.plane, c->stream);
      launch_narrow(s.ghostE[b], s.ghostE32[b], z.plane, c->stream);
      for (int side = 0; side < 2; ++side) launch_narrow(s.hsend[side][b], s.hsend32[side][b], z.hsend[side], c->stream);
    }
  }
  st = cuda_check(cudaGetLastError(), "precision convert");
  if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "precision convert");
  if (st) return st;
  free_state(c, c->prec);
  c->prec = precision;
  if (c->use_tiles && !c->tiles_explicit && !c->tiles_tuned && (st = retile_for_precision(c))) return st;
  if (c->use_tiles && !c->tiles.split && c->tiles.plan_prec != precision) {
    // the schedule stayed: its launch plan becomes the new precision's
    plan_for_precision(c->tiles, precision);
    if ((st = upload_tiles(c))) return st;
    if ((st = cuda_check(cudaStreamSynchronize(c->stream), "replan"))) return st;
  }
  c->version += 1;
  return PIKS_OK;
}

piks_status piks_set_tiles(piks_ctx *c, int32_t tx, int32_t ty, int32_t tz) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  if (tx < 0 || ty < 0 || tz < 0 || (tx > 0 && (ty < 2 || tz < 2 || tx < 2)) || (int64_t)tx * ty * tz > 65535)
    return fail(PIKS_ERR_ARG, "tile extents must be 0 (per-node schedule) or >= 2 with at most 65535 voxels");
  c->tile_dims[0] = tx; c->tile_dims[1] = tx ? ty : 0; c->tile_dims[2] = tx ? tz : 0;
  c->tiles_explicit = true;
  return PIKS_OK;
}

piks_status piks_set_schedule(piks_ctx *c, int32_t schedule) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  if (schedule < PIKS_SCHED_TILE_DATAFLOW || schedule > PIKS_SCHED_TILE_PIPELINED)
    return fail(PIKS_ERR_ARG, "unknown schedule");
  const int old_form = tile_form(c->schedule);
  c->schedule = schedule;
  if (old_form == tile_form(schedule) || !c->have_host_geometry) return PIKS_OK;
  // the new launch schedule reads another form of the tile jobs: rebuild them
  drop_tiles_next(c);
  if (c->device >= 0 && c->have_geometry) {
    cudaSetDevice(c->device);
    piks_status st = cuda_check(cudaStreamSynchronize(c->stream), "schedule sync");
    if (st) return st;
  }
  build_tiles(c);
  if (c->device >= 0 && c->have_geometry) {
    piks_status st = upload_tiles(c);
    if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "schedule upload");
    if (st) return st;
    c->version += 1;
  }
  return PIKS_OK;
}

piks_status piks_get_schedule(piks_ctx *c, int32_t *out, int32_t n) {
  if (!c || !out) return fail(PIKS_ERR_ARG, "null argument");
  const int32_t v[7] = {c->use_tiles ? 1 : 0, c->tiles.TX, c->tiles.TY, c->tiles.TZ, c->tiles.max_rows,
                        c->schedule, (int32_t)c->tiles.row_count.size()};
  for (int i = 0; i < n && i < 7; ++i) out[i] = v[i];
  return PIKS_OK;
}

piks_status piks_autotune(piks_ctx *c, const int32_t *cand, int32_t ncand, int32_t sweeps, int32_t *chosen,
                          double *ms_out) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  if (c->device < 0 || !c->have_geometry) return fail(PIKS_ERR_STATE, "piks_autotune needs a device state");
  if (c->iStep != 0) return fail(PIKS_ERR_STATE, "piks_autotune must run before the first iteration");
  static const int32_t kDefault[] = {8, 4, 4, PIKS_SCHED_TILE_DIAGONALS, 8, 4, 4, PIKS_SCHED_TILE_DATAFLOW,
                                     4, 4, 4, PIKS_SCHED_TILE_DIAGONALS, 4, 4, 4, PIKS_SCHED_TILE_DATAFLOW,
                                     8, 8, 4, PIKS_SCHED_TILE_DIAGONALS};
  if (!cand || ncand <= 0) { cand = kDefault; ncand = 5; }
  if (sweeps < 1) sweeps = 1;
  cudaSetDevice(c->device);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const bool timing = c->timing;
  c->timing = false;
  double best = 1e300;
  int bi = -1;
  piks_status st = PIKS_OK;
  int epoch = 1;
  for (int i = 0; i < ncand && !st; ++i) {
    const int32_t *k = cand + 4 * i;
    if (ms_out) ms_out[i] = -1.0;
    if (k[0] < 2 || k[1] < 2 || k[2] < 2 || (int64_t)k[0] * k[1] * k[2] > 65535) continue;
    if (k[3] < PIKS_SCHED_TILE_DATAFLOW || k[3] > PIKS_SCHED_TILE_PIPELINED) continue;
    c->tile_dims[0] = k[0]; c->tile_dims[1] = k[1]; c->tile_dims[2] = k[2];
    c->schedule = k[3];
    if (!build_tiles(c)) continue;
    if ((st = upload_tiles(c))) break;
    enqueue_sweep(c, c->stream, epoch++);  // warm-up
    cudaEventRecord(e0, c->stream);
    for (int r = 0; r < sweeps; ++r) enqueue_sweep(c, c->stream, epoch++);
    cudaEventRecord(e1, c->stream);
    if ((st = cuda_check(cudaEventSynchronize(e1), "autotune"))) break;
    if ((st = check_sweep_error(c))) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double per = ms / sweeps;
    if (ms_out) ms_out[i] = per;
    if (per < best) { best = per; bi = i; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->timing = timing;
  if (st) return st;
  if (bi < 0) return fail(PIKS_ERR_ARG, "no usable tile candidate");
  const int32_t *k = cand + 4 * bi;
  c->tile_dims[0] = k[0]; c->tile_dims[1] = k[1]; c->tile_dims[2] = k[2];
  c->schedule = k[3];
  build_tiles(c);
  if ((st = upload_tiles(c))) return st;
  c->tiles_tuned = true;
  // the trial sweeps changed f: back to the state of setupFlow (all zero)
  const StateSizes z = state_sizes(c);
  DevState &s = c->ds;
  const size_t e = c->prec == PIKS_PREC_FP32 ? sizeof(float) : sizeof(double);
  void *hs = c->prec == PIKS_PREC_FP32 ? (void *)s.h32 : (void *)s.h;
  void *fws = c->prec == PIKS_PREC_FP32 ? (void *)s.fw32 : (void *)s.fw;
  cudaMemsetAsync(hs, 0, z.h * e, c->stream);
  if (z.fw) cudaMemsetAsync(fws, 0, z.fw * e, c->stream);
  for (int b = 0; b < 2; ++b) {
    cudaMemsetAsync(c->prec == PIKS_PREC_FP32 ? (void *)s.ghostW32[b] : (void *)s.ghostW[b], 0, z.plane * e, c->stream);
    cudaMemsetAsync(c->prec == PIKS_PREC_FP32 ? (void *)s.ghostE32[b] : (void *)s.ghostE[b], 0, z.plane * e, c->stream);
  }
  cudaMemsetAsync(s.mom, 0, (size_t)c->geo.NF * 4 * sizeof(double), c->stream);
  c->version += 1;
  if (chosen) for (int j = 0; j < 4; ++j) chosen[j] = k[j];
  return cuda_check(cudaStreamSynchronize(c->stream), "autotune reset");
}

piks_status piks_get_precision(piks_ctx *c, int32_t *precision) {
  if (!c || !precision) return fail(PIKS_ERR_ARG, "null argument");
  *precision = c->prec;
  return PIKS_OK;
}

piks_status piks_run_refined(piks_ctx *c, const char *results_path, const char *out_dir, int32_t verbose,
                             double switch_eps, int32_t *steps32, int32_t *steps, double *perm, double *seconds) {
  if (!c || !c->have_geometry) return fail(PIKS_ERR_STATE, "no geometry");
  if (!(switch_eps >= 0.0)) return fail(PIKS_ERR_ARG, "switch_eps < 0");
  const piks_params &p = c->setup.p;
  c->error = 1.0;
  auto t0 = std::chrono::steady_clock::now();
  piks_status st = piks_set_precision(c, PIKS_PREC_FP32);
  if (st) return st;
  int last32 = 0, step = 0;
  const int first = c->iStep + 1;
  if ((st = run_loop(c, first, std::max(switch_eps, p.eps), true, results_path, out_dir, verbose, &last32))) return st;
  const int n32 = last32 - first + 1;
  if ((st = piks_set_precision(c, PIKS_PREC_FP64))) return st;
  step = last32;
  if (last32 < p.maxStep) {
    // the FP64 phase starts from the widened FP32 iterate and applies the reference's test
    if ((st = run_loop(c, last32 + 1, p.eps, false, results_path, out_dir, verbose, &step))) return st;
  }
  cudaStreamSynchronize(c->stream);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (verbose) {
    char wt[32];
    std::snprintf(wt, sizeof wt, "%11.3E", secs);
    std::printf("Walltime= %s, Steps= %6d, K= %s\n", wt, step, fortran_es15_6(c->permeability).c_str());
  }
  if (out_dir && p.saveLast)
    if ((st = piks_save_fields(c, out_dir, p.saveFormat))) return st;
  if (steps32) *steps32 = n32;
  if (steps) *steps = step;
  if (perm) *perm = c->permeability;
  if (seconds) *seconds = secs;
  return PIKS_OK;
}

piks_status piks_geometry_array(piks_ctx *c, const char *name, void *out, int64_t capacity, int64_t *count) {
  if (!c || !name) return fail(PIKS_ERR_ARG, "null argument");
  const bool velocity = !std::strcmp(name, "cx") || !std::strcmp(name, "cy") || !std::strcmp(name, "cz") ||
                        !std::strcmp(name, "w");
  if (!velocity && !c->have_host_geometry) return fail(PIKS_ERR_STATE, "no geometry");
  const Geometry &g = c->geo;
  const void *src = nullptr;
  size_t n = 0, esz = 0;
  std::string nm(name);
#define ARR(key, vec) if (nm == key) { src = vec.data(); n = vec.size(); esz = sizeof(vec[0]); }
  ARR("nodemap", g.nodemap) ARR("label", g.label) ARR("node_g", g.node_g) ARR("wall_node", g.wall_node)
  ARR("wall_label", g.wall_label) ARR("wall_e", g.wall_e) ARR("wall_corner", g.wall_corner)
  ARR("wall_nb", g.wall_nb) ARR("wall_order", g.wall_order) ARR("level_start", g.level_start)
  ARR("bcorner", g.bcorner) ARR("roles", g.roles) ARR("commit", g.commit) ARR("plane_x1", g.plane_x1)
  ARR("plane_xN", g.plane_xN) ARR("sym_node", g.sym_node) ARR("sym_flag", g.sym_flag)
  ARR("flux_list", g.flux_list) ARR("tasks", g.tasks) ARR("hyper_start", g.hyper_start) ARR("cx", c->vel.cx) ARR("cy", c->vel.cy) ARR("cz", c->vel.cz) ARR("w", c->vel.w)
  ARR("halo_send_w", g.halo_send[0]) ARR("halo_send_e", g.halo_send[1])
  ARR("halo_recv_w", g.halo_recv[0]) ARR("halo_recv_e", g.halo_recv[1])
  const TileJobs &tj = c->tiles;
  ARR("tile_rows", tj.rows) ARR("tile_row_begin", tj.row_begin) ARR("tile_row_count", tj.row_count)
  ARR("tile_tasks", tj.tasks)
  ARR("tile_task_begin", tj.task_begin) ARR("tile_steps", tj.steps) ARR("tile_diag_begin", tj.diag_begin)
  ARR("tile_diag_rows", tj.diag_rows) ARR("tile_job_list", tj.job_list) ARR("tile_launches", tj.launches)
  ARR("tile_up", tj.up) ARR("tile_hdr", tj.hdr) ARR("tile_carry", tj.carry) ARR("tile_carry_begin", tj.carry_begin)
  ARR("tile_col_jobs", tj.col_jobs) ARR("tile_col_begin", tj.col_begin) ARR("tile_col_list", tj.col_list)
#undef ARR
  if (nm == "flux_groups") { src = g.flux_groups; n = 10; esz = sizeof(int32_t); }
  int32_t colinfo[5] = {tj.columns ? 1 : tj.split ? 2 : 0, tj.ncells, tj.max_region, tj.max_carry, tj.max_tasks};
  if (nm == "tile_column_info") { src = colinfo; n = 5; esz = sizeof(int32_t); }
  if (!esz) return fail(PIKS_ERR_ARG, "unknown geometry array " + nm);
  if (count) *count = (int64_t)n;
  if (out) {
    if (capacity < (int64_t)(n * esz)) return fail(PIKS_ERR_ARG, "buffer too small for " + nm);
    std::memcpy(out, src, n * esz);
  }
  return PIKS_OK;
}

piks_status piks_selftest_division(int32_t device, int64_t samples, uint64_t seed, int64_t *mismatches) {
  if (!mismatches || samples <= 0) return fail(PIKS_ERR_ARG, "bad argument");
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) { cudaGetLastError(); prev = -1; }
  piks_status st = cuda_check(cudaSetDevice(device), "cudaSetDevice");
  if (st) return st;
  unsigned long long *d = nullptr;
  if (!(st = cuda_check(cudaMalloc(&d, sizeof(unsigned long long)), "cudaMalloc"))) {
    st = cuda_check(cudaMemset(d, 0, sizeof(unsigned long long)), "selftest memset");
    if (!st) {
      launch_division_selftest(samples, seed, d);
      st = cuda_check(cudaGetLastError(), "selftest launch");
    }
    unsigned long long h = 0;
    if (!st) st = cuda_check(cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost), "selftest");
    cudaFree(d);
    if (!st) *mismatches = (int64_t)h;
  }
  if (prev >= 0) cudaSetDevice(prev);
  return st;
}

piks_status piks_selftest_division_noalloc(int32_t device, int64_t samples, uint64_t seed, int64_t *mismatches) {
  if (!mismatches) return fail(PIKS_ERR_ARG, "null mismatches");
  const char *err = "";
  const int rc = division_selftest_noalloc(device, samples, seed, mismatches, &err);
  if (rc == 1) return fail(PIKS_ERR_ARG, err);
  if (rc) return fail(PIKS_ERR_CUDA, err);
  return PIKS_OK;
}

piks_status piks_set_preprocessing(piks_ctx *c, int32_t where) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  if (where != PIKS_PREP_HOST && where != PIKS_PREP_DEVICE) return fail(PIKS_ERR_ARG, "unknown preprocessing place");
  c->prep = where;
  return PIKS_OK;
}

piks_status piks_setup_seconds(piks_ctx *c, double *out) {
  if (!c || !out) return fail(PIKS_ERR_ARG, "null argument");
  for (int i = 0; i < 4; ++i) out[i] = c->setup_seconds[i];
  return PIKS_OK;
}

// Regions of the iteration state, in snapshot order: f, fw (state precision), moments (FP64),
// the west and east ghost planes the next iteration reads (state precision).
struct StateRegion { void *p; size_t bytes; };
static int state_regions(piks_ctx *c, StateRegion *r) {
  const StateSizes z = state_sizes(c);
  DevState &s = c->ds;
  const bool f32 = c->prec == PIKS_PREC_FP32;
  const size_t e = f32 ? sizeof(float) : sizeof(double);
  const int par = c->iStep & 1;
  r[0] = {f32 ? (void *)s.h32 : (void *)s.h, z.h * e};
  r[1] = {f32 ? (void *)s.fw32 : (void *)s.fw, z.fw * e};
  r[2] = {(void *)s.mom, (size_t)c->geo.NF * 4 * sizeof(double)};
  r[3] = {f32 ? (void *)s.ghostW32[par] : (void *)s.ghostW[par], z.plane * e};
  r[4] = {f32 ? (void *)s.ghostE32[par] : (void *)s.ghostE[par], z.plane * e};
  return 5;
}

// Bytes of one snapshot slot (each region rounded up to 256 bytes).
static size_t slot_bytes(piks_ctx *c) {
  StateRegion r[5];
  const int n = state_regions(c, r);
  size_t b = 0;
  for (int i = 0; i < n; ++i) b += (r[i].bytes + 255) / 256 * 256;
  return b;
}

piks_status piks_snapshot_slot(piks_ctx *c, int32_t slot, int32_t nslots) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  if (c->device < 0 || !c->have_geometry) return fail(PIKS_ERR_STATE, "snapshots need a device state");
  if (c->setup.nranks > 1) return fail(PIKS_ERR_STATE, "snapshots cover single-box contexts");
  if (nslots < 1 || nslots > kMaxSnapSlots || slot < 0 || slot >= nslots) return fail(PIKS_ERR_ARG, "bad snapshot slot");
  cudaSetDevice(c->device);
  const size_t sb = slot_bytes(c);
  piks_status st;
  if (c->snap && (c->snap_bytes < sb * (size_t)nslots || c->snap_prec != c->prec || c->snap_version != c->version)) {
    release(c, c->snap);
    c->snap = nullptr;
    c->snap_bytes = 0;
  }
  if (!c->snap) {
    void *p = nullptr;
    const size_t need = sb * (size_t)nslots;
    if ((st = cuda_check(cudaMalloc(&p, need), "snapshot slots"))) return st;
    c->allocations.push_back({p, need});
    c->dev_bytes += need;
    c->snap = p;
    c->snap_bytes = need;
    c->snap_prec = c->prec;
    c->snap_version = c->version;
    for (auto &v : c->snap_steps) v = -1;
  }
  StateRegion r[5];
  const int n = state_regions(c, r);
  size_t off = sb * (size_t)slot;
  for (int i = 0; i < n; ++i) {
    if (r[i].bytes && (st = cuda_check(cudaMemcpyAsync(static_cast<char *>(c->snap) + off, r[i].p, r[i].bytes,
                                                      cudaMemcpyDeviceToDevice, c->stream), "snapshot copy")))
      return st;
    off += (r[i].bytes + 255) / 256 * 256;
  }
  c->snap_steps[slot] = c->iStep;
  return cuda_check(cudaStreamSynchronize(c->stream), "snapshot");
}

// Slots 0 .. n-1 hold states of this context's current allocation, all an even number of
// iterations apart from each other and from the current state (their ghost planes are the
// ones the next iteration reads).
static piks_status check_slots(piks_ctx *c, int n) {
  if (!c->have_geometry || !c->snap || c->snap_prec != c->prec || c->snap_version != c->version)
    return fail(PIKS_ERR_STATE, "no snapshots of this state");
  if (n < 1 || n > kMaxSnapSlots || slot_bytes(c) * (size_t)n > c->snap_bytes) return fail(PIKS_ERR_ARG, "bad slot count");
  for (int j = 0; j < n; ++j)
    if (c->snap_steps[j] < 0 || ((c->iStep - c->snap_steps[j]) & 1))
      return fail(PIKS_ERR_STATE, "snapshot slot empty or an odd number of iterations away");
  return PIKS_OK;
}

piks_status piks_snapshot_gram(piks_ctx *c, int32_t n, double *gram) {
  if (!c || !gram) return fail(PIKS_ERR_ARG, "null argument");
  if (n < 2) return fail(PIKS_ERR_ARG, "the Gram matrix of differences needs two slots or more");
  piks_status st = check_slots(c, n);
  if (st) return st;
  cudaSetDevice(c->device);
  StateRegion r[5];
  const int nr = state_regions(c, r);
  const bool f32 = c->prec == PIKS_PREC_FP32;
  const size_t sb = slot_bytes(c);
  const int nd = n - 1, npair = nd * (nd + 1) / 2;
  const int nblk = kGramBlocks;
  double *part = nullptr;
  if ((st = cuda_check(cudaMalloc(&part, (size_t)nr * nblk * npair * sizeof(double)), "gram partials"))) return st;
  size_t off = 0;
  for (int i = 0; i < nr; ++i) {
    const char *base = static_cast<const char *>(c->snap) + off;
    double *pi = part + (size_t)i * nblk * npair;
    if (i == 2 || !f32) launch_gram(reinterpret_cast<const double *>(base), sb, n, r[i].bytes / sizeof(double), pi, c->stream);
    else launch_gram(reinterpret_cast<const float *>(base), sb, n, r[i].bytes / sizeof(float), pi, c->stream);
    off += (r[i].bytes + 255) / 256 * 256;
  }
  std::vector<double> h((size_t)nr * nblk * npair);
  st = cuda_check(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "gram D2H");
  if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "gram");
  cudaFree(part);
  if (st) return st;
  // fixed summation order: regions, then blocks
  int q = 0;
  for (int a = 0; a < nd; ++a)
    for (int b = a; b < nd; ++b, ++q) {
      double sum = 0.0;
      for (int i = 0; i < nr; ++i)
        for (int k = 0; k < nblk; ++k) sum += h[((size_t)i * nblk + k) * npair + q];
      gram[a * nd + b] = gram[b * nd + a] = sum;
    }
  return PIKS_OK;
}

piks_status piks_snapshot_combine(piks_ctx *c, int32_t n, const double *coef) {
  if (!c || !coef) return fail(PIKS_ERR_ARG, "null argument");
  piks_status st = check_slots(c, n);
  if (st) return st;
  for (int j = 0; j < n; ++j)
    if (!std::isfinite(coef[j])) return fail(PIKS_ERR_ARG, "combination coefficient is not finite");
  cudaSetDevice(c->device);
  StateRegion r[5];
  const int nr = state_regions(c, r);
  const bool f32 = c->prec == PIKS_PREC_FP32;
  const size_t sb = slot_bytes(c);
  size_t off = 0;
  for (int i = 0; i < nr; ++i) {
    const char *base = static_cast<const char *>(c->snap) + off;
    if (i == 2 || !f32)
      launch_combine(static_cast<double *>(r[i].p), reinterpret_cast<const double *>(base), sb, n, coef,
                     r[i].bytes / sizeof(double), c->stream);
    else
      launch_combine(static_cast<float *>(r[i].p), reinterpret_cast<const float *>(base), sb, n, coef,
                     r[i].bytes / sizeof(float), c->stream);
    off += (r[i].bytes + 255) / 256 * 256;
  }
  for (auto &v : c->snap_steps) v = -1;  // used up: the state moved off the iteration's path
  st = cuda_check(cudaGetLastError(), "combine");
  if (!st) st = cuda_check(cudaStreamSynchronize(c->stream), "combine");
  return st;
}

piks_status piks_set_decomposition(piks_ctx *c, int32_t nranks, int32_t rank) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  if (c->have_host_geometry) return fail(PIKS_ERR_STATE, "piks_set_decomposition must come before piks_setup_physical_grid");
  std::string err;
  piks_status st = set_slab(c->setup, nranks, rank, err);
  if (st) return fail(st, err);
  return PIKS_OK;
}

piks_status piks_get_slab(piks_ctx *c, int32_t *out) {
  if (!c || !out) return fail(PIKS_ERR_ARG, "null argument");
  out[0] = c->setup.xl; out[1] = c->setup.xu; out[2] = c->setup.nranks; out[3] = c->setup.rank;
  return PIKS_OK;
}

piks_status piks_halo_buffers(piks_ctx *c, int32_t side, void **send, void **recv, int64_t *bytes) {
  if (!c || !send || !recv || !bytes) return fail(PIKS_ERR_ARG, "null argument");
  if (side != 0 && side != 1) return fail(PIKS_ERR_ARG, "side must be 0 (west) or 1 (east)");
  if (!c->have_geometry) return fail(PIKS_ERR_STATE, "piks_setup_physical_grid has not been called");
  *send = *recv = nullptr;
  bytes[0] = bytes[1] = 0;
  if (c->setup.nranks == 1) return PIKS_OK;  // one rank exchanges with itself inside the iteration
  const DevState &s = c->ds;
  const bool f32 = c->prec == PIKS_PREC_FP32;
  const size_t e = f32 ? sizeof(float) : sizeof(double);
  const int par = c->iStep & 1;  // the buffers the last iteration packed / the next one reads
  const StateSizes z = state_sizes(c);
  const bool edge = side == 0 ? c->geo.wglob : c->geo.eglob;
  if (edge) {
    // the periodic pair of the first and last slab: the plane x = 1 (sent west, read by
    // the outlet) and the plane x = Nx (sent east, read by the inlet), one iteration behind
    if (side == 0) {
      *send = f32 ? (void *)s.ghostE32[par] : (void *)s.ghostE[par];
      *recv = f32 ? (void *)s.ghostW32[par] : (void *)s.ghostW[par];
    } else {
      *send = f32 ? (void *)s.ghostW32[par] : (void *)s.ghostW[par];
      *recv = f32 ? (void *)s.ghostE32[par] : (void *)s.ghostE[par];
    }
    bytes[0] = bytes[1] = (int64_t)(z.plane * e);
    return PIKS_OK;
  }
  *send = f32 ? (void *)s.hsend32[side][par] : (void *)s.hsend[side][par];
  *recv = f32 ? (void *)s.hrecv32[side] : (void *)s.hrecv[side];
  bytes[0] = (int64_t)(z.hsend[side] * e);
  bytes[1] = (int64_t)(z.hrecv[side] * e);
  return PIKS_OK;
}

piks_status piks_set_stream(piks_ctx *c, void *stream) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
  return PIKS_OK;
}

piks_status piks_enable_timing(piks_ctx *c, int32_t on) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  drain_timing(c);
  c->timing = on != 0;
  return PIKS_OK;
}

piks_status piks_kernel_times(piks_ctx *c, double *out, int32_t n, int32_t reset) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  drain_timing(c);
  for (int k = 0; k < KT_N && 2 * k + 1 < n; ++k) { out[2 * k] = c->kt_ms[k]; out[2 * k + 1] = (double)c->kt_n[k]; }
  if (reset) for (int k = 0; k < KT_N; ++k) { c->kt_ms[k] = 0; c->kt_n[k] = 0; }
  return PIKS_OK;
}

piks_status piks_launches_per_iteration(piks_ctx *c, int64_t *n) {
  if (!c || !n || !c->have_geometry) return fail(PIKS_ERR_STATE, "no geometry");
  const DevState &s = c->ds;
  int64_t k = 0;
  if (c->use_tiles) {
    k += (c->schedule == PIKS_SCHED_TILE_DATAFLOW || c->tiles.split) ? 1 : (int64_t)(c->tiles.launches.size() / 4);
  } else {
    for (size_t h = 0; h + 1 < c->geo.hyper_start.size(); ++h) k += c->geo.hyper_start[h + 1] > c->geo.hyper_start[h];
  }
  k += (s.ncommit > 0) + 1 /*capture*/ + (int64_t)(c->geo.level_start.size() - 1) + 1 /*inlet*/ +
       (s.nsym > 0) + (s.NF > 0);
  *n = k;
  return PIKS_OK;
}

piks_status piks_selftest_wait_timeout(piks_ctx *c, double *seconds) {
  if (!c || !seconds) return fail(PIKS_ERR_ARG, "null argument");
  if (c->device < 0 || !c->have_geometry || !c->use_tiles || c->ds.tv.njobs < 1 || c->tiles.split)
    return fail(PIKS_ERR_STATE, "the wait self-test needs a device state with a dataflow or diagonal tile schedule");
  cudaSetDevice(c->device);
  DevState &s = c->ds;
  TileView &tv = s.tv;
  // job 0's first upstream entry -> the job index njobs, whose flags nothing sets
  int32_t *up = const_cast<int32_t *>(tv.up);
  int32_t old_up = 0;
  const int32_t never = tv.njobs;
  piks_status st = cuda_check(cudaMemcpy(&old_up, up, sizeof(int32_t), cudaMemcpyDeviceToHost), "selftest up");
  if (!st) st = cuda_check(cudaMemcpy(up, &never, sizeof(int32_t), cudaMemcpyHostToDevice), "selftest up");
  if (st) return st;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // a negative epoch: no flag of an earlier sweep holds it, and no later iteration uses it
  static std::atomic<int> calls{0};
  const int epoch = -(++calls);
  const bool f32 = c->prec == PIKS_PREC_FP32;
  cudaEventRecord(e0, c->stream);
  launch_tile_sweep_dataflow(s, f32, epoch, c->tiles.max_rows, c->tiles.max_tasks, c->stream);
  cudaEventRecord(e1, c->stream);
  st = cuda_check(cudaStreamSynchronize(c->stream), "selftest sweep");
  float ms = 0.f;
  if (!st) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int err = 0;
  if (!st) st = cuda_check(cudaMemcpy(&err, tv.err, sizeof(int), cudaMemcpyDeviceToHost), "selftest err");
  // restore the schedule and clear the error flag in any case
  cudaMemcpy(up, &old_up, sizeof(int32_t), cudaMemcpyHostToDevice);
  cudaMemset(tv.err, 0, sizeof(int));
  if (st) return st;
  *seconds = ms * 1e-3;
  if (!err) return fail(PIKS_ERR_STATE, "the dataflow wait did not give up");
  return PIKS_OK;
}

piks_status piks_synchronize(piks_ctx *c) {
  if (!c) return fail(PIKS_ERR_ARG, "null context");
  cudaSetDevice(c->device);
  piks_status st = cuda_check(cudaStreamSynchronize(c->stream), "synchronize");
  if (!st && c->have_geometry) st = check_sweep_error(c);
  return st;
}

piks_status piks_destroy(piks_ctx *c) {
  if (!c) return PIKS_OK;
  drop_tiles_next(c);
  if (c->device < 0) { delete c; return PIKS_OK; }
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
  free_device(c);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return PIKS_OK;
}

}  // extern "C"
