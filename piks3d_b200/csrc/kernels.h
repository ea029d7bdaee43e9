// Device-side data of one solve and the launch wrappers of the iteration kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace piks {

// Device copy of the tile-wavefront schedule (TileJobs in piks_internal.h).
struct TileView {
  const int32_t *rows;          // global row codes of every job's shared-memory slots 1..
  const int64_t *row_begin;     // [njobs + 1], multiples of 4
  const int32_t *row_count;     // [njobs]
  const int4 *tasks;            // node | fx<<27 | fy<<28 | fz<<29, slots x1|x2<<16, y1|y2<<16, z1|z2<<16
  const int64_t *task_begin;    // [njobs + 1]
  const uint16_t *steps;        // [njobs][steps_stride] task offsets of the local hyperplanes
  const int32_t *job_list;      // job indices in launch order
  const int32_t *up;            // [njobs][4] upstream jobs (tile neighbours upwind, same octant) or -1
  int *flags;                   // [njobs][chunks] epoch of the last sweep that finished the item
  int *counter;                 // work-item counter of the dataflow launch
  int *err;                     // set when a dependency wait gave up
  int njobs;
  int nsteps, steps_stride;
  int paired;                   // diagonal launches sweep job pairs (TileJobs::paired)
  // column form (TileJobs::columns): per-job headers, carry lists, columns in dependency order
  const int32_t *hdr;           // [njobs][8]
  const int32_t *carry;
  const int32_t *col_jobs, *col_begin, *col_list;
  int ncols, ncells, max_region, max_carry, max_tasks, max_nrows;
  float mean_region;
};

// Everything the kernels read, as device pointers (one struct passed by value).
struct DevState {
  int Nx, Ny, Nz, GX, GXY;      // interior extents; ghosted row / plane strides
  int NF, NB, Nc8, nchunk, lpt; // fluid nodes, read solid nodes, velocities per octant, sweep chunks, lanes per task
  const int32_t *nodemap;       // ghosted: >=0 node, -1 unread solid, -2 ghost
  const uint8_t *label;         // ghosted labels
  double *h;                    // [node][octant][Nc8] distribution function
  double *fw;                   // [corner][octant][Nc8] 3-fold corner storage
  const int32_t *bcorner;       // [NB] corner of a solid node or -1
  const uint16_t *roles;        // [NB][8] sources seen by y1/y2/z1/z2 readers
  double *mom;                  // [NF][4] moments Rho, Ux, Uy, Uz
  const double *cx, *cy, *cz, *w;  // [Nc8]
  double mu;                    // sqrt(pi/2)/Kn
  double c15, c20, c05, c10;    // 1.5/ds, 2/ds, -0.5/ds, 1/ds (physicalGrid.F90:1259-1297)
  double accom, pressDrop, DiffFlux;
  const double *vtab;           // [Nc8][kVtab] per-velocity sweep constants (see kernels.cu)
  const double2 *vtab2;         // [Nc8/2][kVtab] the same for velocity pairs (l, l+1), even Nc8
  const int32_t *tasks;         // sweep task records, 8 int32 each
  // walls
  int nWall;
  const int32_t *wall_node, *wall_label, *wall_corner, *wall_nb, *wall_order;
  const double *wall_e;
  // the same fields in level order, one 64-byte record (four int4) per wall position:
  // node, corner, label, 0 | e1, e2 (FP64) | nb[0..3] | nb[4], nb[5], 0, 0; the on-chip wall
  // kernels read a wall's fields in one round trip instead of two (wall_order, then the
  // rest). Per iteration on a 128^3 pack: FP32 0.476 -> 0.446 ms; FP64 0.845 -> 0.758 ms
  // together with up to 85 registers per thread instead of 64 (no spills; the records alone at 64
  // registers spilled and took 0.870 against 0.834)
  const int4 *wall_rec;
  // post-sweep switch commits
  int ncommit;
  const int32_t *commit;
  // x = 1 / x = Nx planes and the two lagged ghost planes
  const int32_t *plane_x1, *plane_xN;
  double *ghostW[2], *ghostE[2];  // [Ny*Nz][4][Nc8]
  // symmetry planes
  int nsym;
  const int32_t *sym_node;
  const uint8_t *sym_flag;
  // chkConverge
  const int32_t *flux_list;
  int flux_groups[10];
  double *flux_out;             // [1]
  // FP32 storage of the same state (used instead of h/fw/ghost* when the context runs the
  // FP32 sweep); moments, wall densities and the flux stay FP64
  float *h32, *fw32;
  float *ghostW32[2], *ghostE32[2];
  const float *vtab32;          // [Nc8][kVtab] sweep constants rounded to FP32
  TileView tv;                  // tile-wavefront sweep schedule (when built)
  // x halos of a slab (side 0 west, 1 east; solver.F90:535-560): the nodes whose rows are
  // sent and the ghost-plane nodes received into, and per precision the send buffers (by
  // iteration parity) and the receive buffer, [count][4][Nc8] of the four octants the
  // receiver reads (west ghosts: cx > 0, east ghosts: cx < 0)
  int nhalo_send[2], nhalo_recv[2];
  const int32_t *halo_send[2], *halo_recv[2];
  double *hsend[2][2], *hrecv[2];
  float *hsend32[2][2], *hrecv32[2];
};

// Runs configure() once per (key, current device) for the whole process, under a mutex:
// launchers set kernel attributes this way from any host thread.
void once_per_device(const void *key, void (*configure)(int device));
// Resident blocks of kernel `fn` on the whole current device (blocks per SM x SMs) for
// `threads` threads and `smem` dynamic shared memory; cached per (fn, device, smem).
long resident_blocks(const void *fn, int threads, size_t smem);

// Per-velocity sweep constants: cx cy cz w, then c*C products (x: 2/ds, 1/ds, -0.5/ds;
// y: same; z: same), the 8 denominators by first-order class and their reciprocals.
constexpr int kVtab = 29;
void launch_sweep_hyperplane(const DevState &s, long t0, long ntask, cudaStream_t st);
void launch_commit(const DevState &s, cudaStream_t st);
// Wall-slot commits as 16-byte row copies (FP64 rows need an even Nc8, FP32 rows Nc8 % 4 == 0).
void launch_commit_rows(const DevState &s, bool fp32, cudaStream_t st);
void launch_capture(const DevState &s, int buf, cudaStream_t st);
void launch_walls(const DevState &s, int begin, int end, int gbuf, cudaStream_t st);
void launch_inlet_outlet(const DevState &s, int buf, cudaStream_t st);
void launch_symmetry(const DevState &s, cudaStream_t st);
void launch_moments(const DevState &s, cudaStream_t st);
void launch_flux(const DevState &s, double ds, double sqrt_half, double inv_refl2, cudaStream_t st);
void upload_tables();
// FP32 path (kernels_fp32.cu)
void upload_tables_fp32();
void launch_sweep_hyperplane32(const DevState &s, long t0, long ntask, cudaStream_t st);
void launch_commit32(const DevState &s, cudaStream_t st);
void launch_capture32(const DevState &s, int buf, cudaStream_t st);
void launch_walls32(const DevState &s, int begin, int end, int gbuf, cudaStream_t st);
void launch_inlet_outlet32(const DevState &s, int buf, cudaStream_t st);
void launch_symmetry32(const DevState &s, cudaStream_t st);
void launch_moments32(const DevState &s, cudaStream_t st);
// Tile-wavefront sweep: the jobs job_list[first .. first + njobs) (all of one diagonal),
// `slots` shared-memory rows and room for `tasks` task records per CTA. tile_sweep_velocities() is the chunk width V used for the precision.
int tile_sweep_velocities(int Nc8, bool fp32);
int tile_sweep_max_slots(int Nc8, bool fp32, int tile_voxels, int nsteps);
// pdl: launch as a programmatic dependent of the previous kernel in the stream: the next tile
// diagonal's CTAs start their first loads (codes, records, moments) while the previous
// diagonal finishes, and wait for it before reading rows. Only for diagonals after the first.
void launch_tile_sweep(const DevState &s, bool fp32, int job0, int njobs, int slots, int tasks, bool pdl,
                       cudaStream_t st);
// Dataflow form: all jobs in one launch, ordered by the flags of `epoch` (> 0, one value per
// sweep); slots / tasks are the largest of any job.
void launch_tile_sweep_dataflow(const DevState &s, bool fp32, int epoch, int slots, int tasks, cudaStream_t st);
// Batched dataflow sweep over several solves of one precision / chunk width V: states is a
// device array of DevState, items (member | chunk << 12, job) in dependency order; the
// members' flags must be zero.
void launch_tile_sweep_batch(const DevState *states, const int2 *items, int nitems, bool fp32, int V, int slots,
                             int tasks, int stride, int *counter, int *err, cudaStream_t st);
// Column-march sweep over the column form: one persistent launch per sweep (flags cleared
// on the stream first, so the launch sequence can be captured in a graph).
void launch_tile_sweep_columns(const DevState &s, bool fp32, int epoch, cudaStream_t st);
// Pipelined dataflow sweep over the split form: the same persistent producer / consumer
// kernel, with single jobs in the diagonal launch order as its work items.
void launch_tile_sweep_pipelined(const DevState &s, bool fp32, int epoch, cudaStream_t st);
// Whether the column-march kernel's shared memory holds the schedule's largest job.
bool column_sweep_fits(const TileView &tv, int Nc8, bool fp32);
// Halo rows of iteration parity `cap`: pack the rows this slab sends into its send buffers,
// unpack the received buffers into its ghost-plane nodes (FP32 or FP64 state).
void launch_halo(const DevState &s, bool fp32, int cap, cudaStream_t st);
// State snapshots (piks_snapshot_slot): at most kMaxSnapSlots copies, `stride` bytes apart.
constexpr int kMaxSnapSlots = 8;
constexpr int kGramBlocks = 148 * 4;
// Per-block FP64 sums of u_a[i] u_b[i] (a <= b < n - 1, u_a = slot_{a+1} - slot_a) over the
// `count` elements of one region at `base` in every slot: partial[block][pair], pairs in
// row order of the upper triangle; a fixed-size grid and fixed summation order.
void launch_gram(const double *base, size_t stride, int n, size_t count, double *partial, cudaStream_t st);
void launch_gram(const float *base, size_t stride, int n, size_t count, double *partial, cudaStream_t st);
// dst[i] = sum_j coef[j] slot_j[i] over n slots, evaluated in FP64.
void launch_combine(double *dst, const double *base, size_t stride, int n, const double *coef, size_t count,
                    cudaStream_t st);
void launch_combine(float *dst, const float *base, size_t stride, int n, const double *coef, size_t count,
                    cudaStream_t st);
void launch_widen(const float *src, double *dst, size_t n, cudaStream_t st);
void launch_narrow(const double *src, float *dst, size_t n, cudaStream_t st);
void launch_division_selftest(int64_t samples, uint64_t seed, unsigned long long *mismatches);
int division_selftest_noalloc(int device, int64_t samples, uint64_t seed, int64_t *mismatches, const char **err);

}  // namespace piks
