// The solver context behind the C ABI's piks_ctx, shared by capi.cu and batch.cu.
#pragma once
#include <cuda_runtime.h>

#include <future>
#include <string>
#include <utility>
#include <vector>

#include "kernels.h"
#include "piks3d_gpu.h"
#include "piks_internal.h"

namespace piks {
enum { KT_SWEEP, KT_COMMIT, KT_CAPTURE, KT_WALLS, KT_INLET, KT_SYM, KT_MOM, KT_FLUX, KT_N };
piks_status fail(piks_status st, const std::string &msg);   // records the message for piks_last_error
piks_status cuda_check(cudaError_t e, const char *what);
}  // namespace piks

struct piks_ctx {
  piks::Setup setup;
  piks::Velocity vel;
  piks::Geometry geo;
  int device = 0;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  bool have_geometry = false;       // device state ready
  bool have_host_geometry = false;  // preprocessing done
  piks::DevState ds{};
  std::vector<std::pair<void *, size_t>> allocations;  // device buffers and their bytes
  size_t dev_bytes = 0;
  int prec = PIKS_PREC_FP64;        // storage / sweep precision of the state
  int tile_dims[3] = {8, 4, 4};     // tile shape of the sweep schedule (0: per-node hyperplanes)
  bool tiles_explicit = false;      // set by piks_set_tiles; otherwise chosen by precision at setup
  bool tiles_tuned = false;         // chosen by piks_autotune (kept across precision switches)
  // the schedule of the other precision's default tile shape, built on a host thread while
  // an FP32 state iterates (taken up by the switch to FP64)
  piks::TileJobs tiles_next;
  int tiles_next_dims[3] = {0, 0, 0};
  std::future<bool> tiles_next_ready;
  piks::TileJobs tiles;
  bool use_tiles = false;           // tile schedule built and uploaded
  int schedule = PIKS_SCHED_TILE_DIAGONALS;
  int prep = PIKS_PREP_DEVICE;      // where voxels are classified (device contexts)
  double setup_seconds[4] = {0, 0, 0, 0};  // last setup: box, classification, rest of the geometry, all
  int iStep = 0;
  int version = 0;                  // bumped whenever the device state is reallocated
  // copies of the iteration state (piks_snapshot_slot): per slot f, fw, moments and the
  // ghost planes the next iteration reads, slots back to back in one buffer
  void *snap = nullptr;
  size_t snap_bytes = 0;
  int snap_prec = -1, snap_version = -1;
  int snap_steps[8] = {-1, -1, -1, -1, -1, -1, -1, -1};  // iteration of each slot's copy
  double mass = 1.0, error = 1.0, permeability = 0.0;
  bool timing = false;
  double kt_ms[piks::KT_N] = {0};
  int64_t kt_n[piks::KT_N] = {0};
  // one iteration of each parity as a CUDA graph (tile diagonals, hyperplanes), valid for
  // graph_key = version * 8 + schedule; the first two iterations after a change run plain
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int graph_key = -1, graph_warm = 0;
  bool graph_failed = false;
  cudaStream_t cap_stream = nullptr;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  size_t ev_next = 0;
};

namespace piks {
// The boundary part of iteration n (commit ... moments) on stream st, untimed.
void enqueue_boundaries(piks_ctx *c, cudaStream_t st, int n);
// chkConverge's flux kernel on stream st, and the host update from its result m2.
void launch_check(piks_ctx *c, cudaStream_t st);
void finish_check(piks_ctx *c, double m2);
}  // namespace piks
