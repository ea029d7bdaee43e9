// Batches of solves (piks_batch_*, include/piks3d_gpu.h): several contexts on one device
// iterated together. One iteration of a batch is, per precision class of its members, one
// dataflow launch that sweeps every member's tile jobs, followed by each member's boundary
// kernels. The members' boundary chains are independent of one another, so they fork onto
// side streams after the sweep and join before the next iteration: in the captured graph they
// are parallel branches, and small members' launches overlap instead of running one after
// another. The sequence is captured once as a CUDA graph per iteration parity and replayed
// while the membership stays the same.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "context.h"

using namespace piks;

struct piks_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<piks_ctx *> members;
  std::vector<int> versions;     // members' state versions at the last rebuild
  bool dirty = true;
  struct Class {
    bool fp32 = false;
    int V = 0, slots = 0, tasks = 0, stride = 0;
    std::vector<int2> items;
    int2 *d_items = nullptr;
    size_t cap = 0;
  };
  std::vector<Class> classes;
  DevState *d_states = nullptr;
  size_t states_cap = 0;
  int *d_ctl = nullptr;          // [class counters ..., error flag], kMaxClasses + 1
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int warm = 0;                  // iterations run since the last rebuild
  double *h_mass = nullptr;      // pinned, one per member
  size_t h_cap = 0;
  // fork / join of the members' boundary chains: member m runs on side[m % side.size()]
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> joined;  // one per side stream
  cudaEvent_t swept = nullptr;      // recorded on the batch stream after the sweeps
};

namespace {

constexpr int kMaxClasses = 8;
// Side streams for the members' boundary chains (more gives the graph no further overlap:
// a boundary chain is a handful of dependent launches of a few microseconds each).
constexpr int kMaxSide = 16;

piks_status make_side_streams(piks_batch *b, size_t want) {
  want = std::min<size_t>(want, kMaxSide);
  if (!b->swept) {
    piks_status st = cuda_check(cudaEventCreateWithFlags(&b->swept, cudaEventDisableTiming), "batch event");
    if (st) return st;
  }
  while (b->side.size() < want) {
    cudaStream_t s = nullptr;
    cudaEvent_t e = nullptr;
    piks_status st = cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "batch side stream");
    if (!st) st = cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch event");
    if (st) {
      if (s) cudaStreamDestroy(s);
      return st;
    }
    b->side.push_back(s);
    b->joined.push_back(e);
  }
  return PIKS_OK;
}

void drop_graphs(piks_batch *b) {
  for (auto &g : b->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

// Device copies of the members' states and, per (precision, V) class, the work items of the
// merged sweep: ordered by tile diagonal, then member, then the member's launch order, then
// velocity chunk, so that every item's upstream items come before it.
piks_status rebuild(piks_batch *b) {
  drop_graphs(b);
  b->warm = 0;
  const size_t nm = b->members.size();
  if (nm > b->states_cap) {
    if (b->d_states) cudaFree(b->d_states);
    b->d_states = nullptr;
    piks_status st = cuda_check(cudaMalloc(&b->d_states, nm * sizeof(DevState)), "batch states");
    if (st) return st;
    b->states_cap = nm;
  }
  std::vector<DevState> hs(nm);
  for (size_t m = 0; m < nm; ++m) hs[m] = b->members[m]->ds;
  if (nm) {
    piks_status st = cuda_check(cudaMemcpyAsync(b->d_states, hs.data(), nm * sizeof(DevState), cudaMemcpyHostToDevice,
                                                b->stream), "batch states upload");
    if (st) return st;
  }
  std::vector<piks_batch::Class> cls;
  std::vector<int> cls_of(nm);
  for (size_t m = 0; m < nm; ++m) {
    const piks_ctx *c = b->members[m];
    const bool f32 = c->prec == PIKS_PREC_FP32;
    const int V = tile_sweep_velocities(c->vel.Nc8, f32);
    int k = 0;
    while (k < (int)cls.size() && !(cls[k].fp32 == f32 && cls[k].V == V)) ++k;
    if (k == (int)cls.size()) {
      if (k == kMaxClasses) return fail(PIKS_ERR_ARG, "batch: too many precision / velocity classes");
      piks_batch::Class nc;
      nc.fp32 = f32;
      nc.V = V;
      cls.push_back(nc);
    }
    cls_of[m] = k;
    cls[k].slots = std::max(cls[k].slots, c->tiles.max_rows);
    cls[k].tasks = std::max(cls[k].tasks, c->tiles.max_tasks);
    cls[k].stride = std::max(cls[k].stride, c->tiles.steps_stride);
  }
  int maxdiag = 0;
  for (auto *c : b->members) maxdiag = std::max(maxdiag, (int)c->tiles.launch_diag_end.size());
  for (int d = 0; d < maxdiag; ++d)
    for (size_t m = 0; m < nm; ++m) {
      const piks_ctx *c = b->members[m];
      const TileJobs &tj = c->tiles;
      if (d >= (int)tj.launch_diag_end.size()) continue;
      const int l0 = d ? tj.launch_diag_end[(size_t)d - 1] : 0, l1 = tj.launch_diag_end[(size_t)d];
      const int nchunk = c->vel.Nc8 / cls[(size_t)cls_of[m]].V;
      auto &items = cls[(size_t)cls_of[m]].items;
      for (int l = l0; l < l1; ++l)
        for (int q = tj.launches[(size_t)l * 4]; q < tj.launches[(size_t)l * 4] + tj.launches[(size_t)l * 4 + 1]; ++q)
          for (int ch = 0; ch < nchunk; ++ch) items.push_back(make_int2((int)m | (ch << 12), tj.job_list[(size_t)q]));
    }
  // keep the device buffers of the old classes where they fit
  for (size_t k = 0; k < cls.size(); ++k) {
    if (k < b->classes.size() && b->classes[k].cap >= cls[k].items.size()) {
      cls[k].d_items = b->classes[k].d_items;
      cls[k].cap = b->classes[k].cap;
      b->classes[k].d_items = nullptr;
    } else {
      piks_status st = cuda_check(cudaMalloc(&cls[k].d_items, std::max<size_t>(1, cls[k].items.size()) * sizeof(int2)),
                                  "batch items");
      if (st) return st;
      cls[k].cap = std::max<size_t>(1, cls[k].items.size());
    }
    if (!cls[k].items.empty()) {
      piks_status st = cuda_check(cudaMemcpyAsync(cls[k].d_items, cls[k].items.data(), cls[k].items.size() * sizeof(int2),
                                                  cudaMemcpyHostToDevice, b->stream), "batch items upload");
      if (st) return st;
    }
  }
  for (auto &oc : b->classes)
    if (oc.d_items) cudaFree(oc.d_items);
  b->classes.swap(cls);
  piks_status sst = make_side_streams(b, nm);
  if (sst) return sst;
  b->versions.resize(nm);
  for (size_t m = 0; m < nm; ++m) b->versions[m] = b->members[m]->version;
  b->dirty = false;
  return cuda_check(cudaStreamSynchronize(b->stream), "batch rebuild");
}

// One iteration of every member, on the batch stream; `parity` offsets the members'
// iteration numbers (0 = their next iteration, 1 = the one after).
void enqueue_batch_iteration(piks_batch *b, int parity) {
  for (piks_ctx *c : b->members) {
    const int nchunk_max = c->vel.Nc8 / 8 > 0 ? c->vel.Nc8 / 8 : 1;
    cudaMemsetAsync(c->ds.tv.flags, 0, (size_t)c->ds.tv.njobs * nchunk_max * sizeof(int), b->stream);
  }
  for (size_t k = 0; k < b->classes.size(); ++k) {
    const auto &cl = b->classes[k];
    launch_tile_sweep_batch(b->d_states, cl.d_items, (int)cl.items.size(), cl.fp32, cl.V, cl.slots, cl.tasks,
                            cl.stride, b->d_ctl + k, b->d_ctl + kMaxClasses, b->stream);
  }
  const size_t ns = std::min(b->side.size(), b->members.size());
  if (ns < 2) {
    for (piks_ctx *c : b->members) enqueue_boundaries(c, b->stream, c->iStep + 1 + parity);
    return;
  }
  cudaEventRecord(b->swept, b->stream);
  for (size_t k = 0; k < ns; ++k) cudaStreamWaitEvent(b->side[k], b->swept, 0);
  for (size_t m = 0; m < b->members.size(); ++m)
    enqueue_boundaries(b->members[m], b->side[m % ns], b->members[m]->iStep + 1 + parity);
  for (size_t k = 0; k < ns; ++k) {
    cudaEventRecord(b->joined[k], b->side[k]);
    cudaStreamWaitEvent(b->stream, b->joined[k], 0);
  }
}

}  // namespace

extern "C" {

piks_status piks_batch_create(int32_t device, piks_batch **out) {
  if (!out) return fail(PIKS_ERR_ARG, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PIKS_ERR_NOT_FOUND, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(PIKS_ERR_ARG, "device index out of range");
  auto *b = new piks_batch();
  b->device = device;
  piks_status st = cuda_check(cudaSetDevice(device), "cudaSetDevice");
  if (!st) st = cuda_check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  if (!st) st = cuda_check(cudaMalloc(&b->d_ctl, (kMaxClasses + 1) * sizeof(int)), "batch control");
  if (!st) st = cuda_check(cudaMemset(b->d_ctl, 0, (kMaxClasses + 1) * sizeof(int)), "batch control");
  if (st) {
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return st;
  }
  *out = b;
  return PIKS_OK;
}

piks_status piks_batch_add(piks_batch *b, piks_ctx *c) {
  if (!b || !c) return fail(PIKS_ERR_ARG, "null argument");
  if (!c->have_geometry) return fail(PIKS_ERR_STATE, "batch member has no device state");
  if (c->device != b->device) return fail(PIKS_ERR_ARG, "batch member lives on another device");
  if (!c->use_tiles) return fail(PIKS_ERR_ARG, "batch members need the tile schedule");
  if (c->setup.nranks > 1) return fail(PIKS_ERR_ARG, "a slab of a decomposed box cannot join a batch");
  if (b->members.size() >= 4096) return fail(PIKS_ERR_ARG, "batch holds at most 4096 members");
  if (std::find(b->members.begin(), b->members.end(), c) != b->members.end()) return PIKS_OK;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(c->stream);
  b->members.push_back(c);
  b->dirty = true;
  return PIKS_OK;
}

piks_status piks_batch_remove(piks_batch *b, piks_ctx *c) {
  if (!b || !c) return fail(PIKS_ERR_ARG, "null argument");
  auto it = std::find(b->members.begin(), b->members.end(), c);
  if (it == b->members.end()) return fail(PIKS_ERR_NOT_FOUND, "not a member of the batch");
  cudaSetDevice(b->device);
  piks_status st = cuda_check(cudaStreamSynchronize(b->stream), "batch sync");
  b->members.erase(it);
  b->dirty = true;
  return st;
}

piks_status piks_batch_size(piks_batch *b, int32_t *n) {
  if (!b || !n) return fail(PIKS_ERR_ARG, "null argument");
  *n = (int32_t)b->members.size();
  return PIKS_OK;
}

piks_status piks_batch_iterate(piks_batch *b, int32_t nsteps) {
  if (!b) return fail(PIKS_ERR_ARG, "null batch");
  if (nsteps < 0) return fail(PIKS_ERR_ARG, "nsteps < 0");
  cudaSetDevice(b->device);
  piks_status st;
  for (size_t m = 0; m < b->members.size() && !b->dirty; ++m)
    if (m >= b->versions.size() || b->versions[m] != b->members[m]->version) b->dirty = true;
  if (b->dirty && (st = rebuild(b))) return st;
  for (int n = 0; n < nsteps; ++n) {
    if (b->members.empty()) break;
    const int par = b->members[0]->iStep & 1;
    if (b->warm < 2) {
      // the first iterations after a change run as plain launches (they also configure the
      // kernels); the graph of each parity is captured on the next occasion
      enqueue_batch_iteration(b, 0);
      ++b->warm;
    } else {
      if (!b->graph[par]) {
        cudaGraph_t g = nullptr;
        st = cuda_check(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed), "batch capture");
        if (st) return st;
        enqueue_batch_iteration(b, 0);
        st = cuda_check(cudaStreamEndCapture(b->stream, &g), "batch capture end");
        if (st) return st;
        st = cuda_check(cudaGraphInstantiate(&b->graph[par], g, 0), "batch graph instantiate");
        cudaGraphDestroy(g);
        if (st) return st;
      }
      st = cuda_check(cudaGraphLaunch(b->graph[par], b->stream), "batch graph launch");
      if (st) return st;
    }
    for (piks_ctx *c : b->members) c->iStep += 1;
  }
  return cuda_check(cudaGetLastError(), "batch iterate");
}

piks_status piks_batch_chk_converge(piks_batch *b, double *mass, double *perm, double *err) {
  if (!b) return fail(PIKS_ERR_ARG, "null batch");
  cudaSetDevice(b->device);
  const size_t nm = b->members.size();
  if (nm > b->h_cap) {
    if (b->h_mass) cudaFreeHost(b->h_mass);
    b->h_mass = nullptr;
    piks_status st = cuda_check(cudaMallocHost(&b->h_mass, nm * sizeof(double)), "batch pinned");
    if (st) return st;
    b->h_cap = nm;
  }
  for (size_t m = 0; m < nm; ++m) {
    piks_ctx *c = b->members[m];
    launch_check(c, b->stream);
    cudaMemcpyAsync(b->h_mass + m, c->ds.flux_out, sizeof(double), cudaMemcpyDeviceToHost, b->stream);
  }
  int e = 0;
  cudaMemcpyAsync(&e, b->d_ctl + kMaxClasses, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
  piks_status st = cuda_check(cudaStreamSynchronize(b->stream), "batch check");
  if (st) return st;
  if (e) return fail(PIKS_ERR_CUDA, "batch sweep: a dependency wait timed out");
  for (size_t m = 0; m < nm; ++m) {
    piks_ctx *c = b->members[m];
    finish_check(c, b->h_mass[m]);
    if (mass) mass[m] = c->mass;
    if (perm) perm[m] = c->permeability;
    if (err) err[m] = c->error;
  }
  return PIKS_OK;
}

piks_status piks_batch_synchronize(piks_batch *b) {
  if (!b) return fail(PIKS_ERR_ARG, "null batch");
  cudaSetDevice(b->device);
  return cuda_check(cudaStreamSynchronize(b->stream), "batch sync");
}

piks_status piks_batch_destroy(piks_batch *b) {
  if (!b) return PIKS_OK;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  for (auto &cl : b->classes)
    if (cl.d_items) cudaFree(cl.d_items);
  if (b->d_states) cudaFree(b->d_states);
  if (b->d_ctl) cudaFree(b->d_ctl);
  if (b->h_mass) cudaFreeHost(b->h_mass);
  for (size_t k = 0; k < b->side.size(); ++k) {
    cudaStreamDestroy(b->side[k]);
    cudaEventDestroy(b->joined[k]);
  }
  if (b->swept) cudaEventDestroy(b->swept);
  cudaStreamDestroy(b->stream);
  delete b;
  return PIKS_OK;
}

}  // extern "C"
