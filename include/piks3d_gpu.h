/*
 * piks3d_gpu.h — C ABI of the B200 solver for PIKS3D's discrete-velocity source
 * iteration (linearised BGK on binary voxel images).
 *
 * PIKS3D (Fortran 90 + MPI + OpenMP) has no library API: main.F90 drives zero-argument
 * module routines over module globals. Each entry point below replaces one of those
 * routines for one GPU holding the box (the reference's mpi 1x1x1 layout; x slabs of a box
 * over several GPUs: piks_set_decomposition) and keeps its argument meaning, file formats
 * and error behaviour. Every function takes
 * plain pointers and sizes, is callable from C, C++, Fortran ISO_C_BINDING or ctypes,
 * and returns a piks_status (0 = success). piks_last_error() gives the message.
 *
 * Threading: one host thread per context at a time; each context owns one CUDA stream
 * (or uses the one given with piks_set_stream). Host arrays are borrowed for the call.
 */
#ifndef PIKS3D_GPU_H
#define PIKS3D_GPU_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum piks_status {
  PIKS_OK = 0,
  PIKS_ERR_ARG = 1,          /* bad argument or parameter value                           */
  PIKS_ERR_NC = 2,           /* Nc_fundamental not in {2,4,6,8,12,16} (velocityGrid.F90:122-126, :149-153) */
  PIKS_ERR_IMAGE = 3,        /* voxel byte other than 0/1 or short stream (physicalGrid.F90:268-275) */
  PIKS_ERR_CUDA = 4,         /* CUDA runtime error                                        */
  PIKS_ERR_OOM = 5,          /* device memory exhausted                                   */
  PIKS_ERR_STATE = 6,        /* call out of order (e.g. iterate before the image is set)  */
  PIKS_ERR_IO = 7,           /* cannot open / read / write a file (parameters.F90:101-105, output.F90:241-245) */
  PIKS_ERR_NOT_FOUND = 8     /* no GPU, or the extension was built without a device        */
} piks_status;

/* Namelist variables of para.in, as read (before initParams adds 2*fluidlayer to Nx and
 * multiplies by block_rep): parameters.F90:78-82. imageFileName is returned separately. */
typedef struct piks_params {
  int32_t Nx, Ny, Nz;            /* physicalNml */
  int32_t wallExtOrder;          /* 1, 2 (default) or 3                                  */
  int32_t fluidlayer;            /* fluid layers added at inlet and outlet (default 0)   */
  double Ref_L;                  /* 1 (default) or 2                                     */
  int32_t Nc_fundamental;        /* velocityNml: half the points per velocity axis       */
  int32_t halfRange;             /* 1 = half-range Gauss-Hermite                          */
  int32_t mpi_xdim, mpi_ydim, mpi_zdim;   /* mpiNml: read; slabs via piks_set_decomposition */
  int32_t block_repx, block_repy, block_repz;
  int32_t maxStep, chkConvergeStep, saveStep;   /* solverNml */
  double eps;
  int32_t saveLast, saveFormat;  /* saveFormat 1 = VTI, 2 = Tecplot, 3 = VTK               */
  double Kn, pressDrop, accom;   /* flowNml */
} piks_params;

typedef struct piks_ctx piks_ctx;

/* Fills the defaults of initParams (parameters.F90:91-98); other fields zero. */
piks_status piks_params_default(piks_params *p);

/* Reads the namelists physicalNml, velocityNml, mpiNml, solverNml, flowNml from a para.in
 * file (initParams, parameters.F90:100-118). image_file receives imageFileName. */
piks_status piks_read_params(const char *path, piks_params *p, char *image_file, int32_t image_file_len);

/* Creates a context on CUDA device `device`: applies initParams' adjustments and sets up
 * the velocity grid (setupVelocityGrid, velocityGrid.F90:90-192). device = -1 gives a
 * host-only context that preprocesses images and answers the getters but cannot iterate. */
piks_status piks_create(const piks_params *p, int32_t device, piks_ctx **out);

/* setupPhysicalGrid + setupFlow + allocateBuf (physicalGrid.F90:217-1625, flow.F90:76-163):
 * takes the raw image stream exactly as the reference reads it from imageFileName
 * (uint8, 0 = fluid, 1 = solid, x fastest, Nx*Ny*Nz bytes for the para.in extents),
 * drills / thins / labels it on the host, uploads the compact state and zeroes f. */
piks_status piks_setup_physical_grid(piks_ctx *ctx, const uint8_t *raw, int64_t nbytes);

/* `nsteps` calls of iterate (solver.F90:111-1940) on the device, asynchronously on the
 * context's stream. iStep advances by nsteps. */
piks_status piks_iterate(piks_ctx *ctx, int32_t nsteps);

/* chkConverge (output.F90:60-164) at the current iStep: mass flux through x = 2,
 * error = |1 - mass_new/mass_old| / chkConvergeStep, permeability = mass*Kn*sqrt(4/pi).
 * Blocks until the device result is on the host. Outputs may be NULL. */
piks_status piks_chk_converge(piks_ctx *ctx, double *mass, double *permeability, double *error);

/* main.F90:95-128: iterate / chkConverge until error <= eps or maxStep; appends each
 * check to results_path (Results.dat format, may be NULL) and prints the reference's
 * stdout lines when verbose. Saves fields every saveStep and at the end (saveLast) into
 * out_dir when out_dir is not NULL. */
piks_status piks_run(piks_ctx *ctx, const char *results_path, const char *out_dir, int32_t verbose,
                     int32_t *steps, double *permeability, double *seconds);

/* Rho, Ux, Uy, Uz over the Nx*Ny*Nz box (x fastest, 0 at non-fluid voxels); any may be NULL. */
piks_status piks_get_macro(piks_ctx *ctx, double *rho, double *ux, double *uy, double *uz);

/* Field writers saveFlowFieldVTI / saveFlowField / saveFlowFieldVTK (output.F90:166-360)
 * into directory dir; format as saveFormat. */
piks_status piks_save_fields(piks_ctx *ctx, const char *dir, int32_t format);

/* Interior voxel labels after preprocessing (image(1:Nx,1:Ny,1:Nz), x fastest): 0 fluid,
 * 1 solid, 20..73 wall labels of physicalGrid.F90:127-134. */
piks_status piks_get_labels(piks_ctx *ctx, int32_t *labels);

/* Sizes: [Nx, Ny, Nz, Nc8, Nfluid, nWall, nCorner, nNodes, iStep, nWallLevels,
 * device bytes held by the context]. */
piks_status piks_get_info(piks_ctx *ctx, int64_t *info, int32_t n);

/* Distribution function in the reference's layout f(Ntotal, Nc8, 8) over the ghosted box
 * (Nx+4)(Ny+4)(Nz+4), column-major; only voxels the solver reads (fluid voxels and solid
 * voxels within two cells of fluid along an axis) are filled, the rest are 0. And fw. */
piks_status piks_get_f(piks_ctx *ctx, double *f_ref, double *fw);

/* f of n nodes (compact node indices, see the "node_g" geometry array for their voxels) as
 * out[n][8][Nc8] (octant, then velocity), for sampled comparisons of large cases. */
piks_status piks_get_f_nodes(piks_ctx *ctx, const int32_t *nodes, int32_t n, double *out);

/* Host-side arrays of the preprocessed geometry by name ("label", "nodemap", "roles",
 * "commit", "wall_nb", ...), for inspection and tests; *count receives the element count,
 * out (capacity bytes) the data when not NULL. */
piks_status piks_geometry_array(piks_ctx *ctx, const char *name, void *out, int64_t capacity, int64_t *count);

/* Where piks_setup_physical_grid classifies the voxels (wall labels, the node map of the
 * voxels the solver reads, 3-fold corner numbers and the wall list; physicalGrid.F90:546-936):
 * PIKS_PREP_DEVICE (the default for a context with a device) runs it as CUDA kernels,
 * PIKS_PREP_HOST on the host; both give identical arrays. The image read and the drill /
 * thin passes (physicalGrid.F90:257-422, whose in-place raster order decides their result)
 * and the sweep schedule stay on the host. No counterpart in the reference. */
enum { PIKS_PREP_HOST = 0, PIKS_PREP_DEVICE = 1 };
piks_status piks_set_preprocessing(piks_ctx *ctx, int32_t where);
/* Wall-clock seconds of the last piks_setup_physical_grid (out[4]): image read, replication
 * and drill / thin; voxel classification; the rest of the geometry and the sweep tasks; the
 * whole call (tile schedule, uploads and allocation included). */
piks_status piks_setup_seconds(piks_ctx *ctx, double *out);

/* ---- Extrapolation of the iteration (refined solves) ----
 * The source iteration is affine, f_{n+1} = M f_n + b: its error e_n = M^n e_0 is soon
 * dominated by a few slow modes of M. From states x_0 .. x_{k+1} taken every m iterations
 * (m even), minimal polynomial extrapolation (MPE) finds the combination s = sum_j g_j x_j
 * (j <= k) that cancels k modes: with u_j = x_{j+1} - x_j, c minimises |U c + u_k| over the
 * first k differences, c_k = 1 and g = c / sum(c). k = 1 is Aitken's extrapolation of the
 * whole state.
 *   piks_snapshot_slot  copies the state the next iteration reads (f, fw, the moments, the
 *                       lagged ghost planes) into slot `slot` of `nslots` (at most 8, one
 *                       device buffer of nslots state sizes);
 *   piks_snapshot_gram  the (n-1) x (n-1) Gram matrix of the differences of slots 0 .. n-1,
 *                       summed in FP64 in a fixed order (the same states give the same matrix);
 *   piks_snapshot_combine  the state becomes sum_j coef[j] * slot_j over slots 0 .. n-1
 *                       (FP64 evaluation); slots must lie an even number of iterations from
 *                       the current state.
 * This takes the iteration off the reference's path: the refined solver (piks3d_b200.solve,
 * FP32 + FP64 refinement) uses it and is assessed by its permeability against the plain FP64
 * solve; the plain FP64 solve never calls it. Single-box contexts only. No counterpart in
 * the reference. */
piks_status piks_snapshot_slot(piks_ctx *ctx, int32_t slot, int32_t nslots);
piks_status piks_snapshot_gram(piks_ctx *ctx, int32_t n, double *gram);
piks_status piks_snapshot_combine(piks_ctx *ctx, int32_t n, const double *coef);

/* ---- One box over several GPUs: x slabs (setupVirtualProcessGrid, mpiParams.F90:120-240,
 * with mpi_xdim = nranks, mpi_ydim = mpi_zdim = 1; the halo exchange of solver.F90:146-170
 * and :535-612). Each rank's context owns the x planes [xl, xu] of the reference's
 * partition and reads two planes of each neighbour (periodic in x: the last rank's east
 * neighbour is rank 0), one iteration behind, as the reference's MPI ranks do.
 *
 * piks_set_decomposition: before piks_setup_physical_grid (every rank passes the whole
 * image); fails when a rank would own fewer than two planes. A slab context iterates one
 * step per piks_iterate call; before each call the host moves, for each side, `send` of
 * this rank to the neighbour's `recv` on the opposite side (NCCL send / recv, a peer copy,
 * or a device copy when the ranks share a GPU), on the context's stream or ordered before
 * it. piks_chk_converge computes the check on rank 0 (the plane x = 2, output.F90:89) and
 * returns the others' stored values: the host broadcasts rank 0's triple. piks_run and
 * batches refuse slab contexts. Replaces: the MPI calls of the reference; no counterpart
 * in its call sequence. */
piks_status piks_set_decomposition(piks_ctx *ctx, int32_t nranks, int32_t rank);
/* out[4] = xl, xu (global 1-based x), nranks, rank. */
piks_status piks_get_slab(piks_ctx *ctx, int32_t *out);
/* Device buffers of the exchange that precedes the next iteration on `side` (0 west, 1 east):
 * `send` (bytes[0] bytes) goes to the neighbour on that side, `recv` (bytes[1]) receives what
 * that neighbour sends; valid until that iteration runs. One rank: NULL / 0 (no exchange). */
piks_status piks_halo_buffers(piks_ctx *ctx, int32_t side, void **send, void **recv, int64_t *bytes);

/* Makes the context enqueue on `stream` (a cudaStream_t); NULL restores its own stream. */
piks_status piks_set_stream(piks_ctx *ctx, void *stream);

/* Per-kernel device time accumulated since the last reset (CUDA events on the context's
 * stream): out[2*k] = milliseconds, out[2*k+1] = launches, k over piks_kernel_names(). */
piks_status piks_kernel_times(piks_ctx *ctx, double *out, int32_t n, int32_t reset);
const char *piks_kernel_names(void);  /* comma-separated */
piks_status piks_enable_timing(piks_ctx *ctx, int32_t on);

/* Number of kernel launches one iterate issues on this context (for launch accounting). */
piks_status piks_launches_per_iteration(piks_ctx *ctx, int64_t *n);

/* Device self-test of the sweep's division (a correctly rounded reciprocal followed by one
 * fused correction step) against IEEE division: counts differing quotients over `samples`
 * random operand pairs. Expected 0. */
piks_status piks_selftest_division(int32_t device, int64_t samples, uint64_t seed, int64_t *mismatches);

/* The same self-test for hosts that cannot allocate device memory when they want to run
 * it: a program that runs under a fixed device-memory budget, or that hands every device
 * allocation to its own pool and does not allow other allocators, can still check the
 * division. This entry point calls no allocator: its scratch is a static device buffer
 * compiled into the library (8 KB of per-block counts, a total and a count of the samples
 * tested; held on every GPU that loads the library until the process exits). It accepts
 * at most 16,777,216 samples and returns PIKS_ERR_ARG with a message above that. Each call
 * looks up the buffer's device address on `device` (a lookup, not an allocation); the
 * first lookup on a device can load the library's device code, so make the first call
 * before any stream capture. All calls share the buffer: calls that overlap on the GPU
 * race, so do not run two at once. The call clears the total first and returns
 * PIKS_ERR_CUDA when a kernel failed to launch or did not test every sample, so a result
 * always comes from this call. Runs on the default stream, returns after the result is on
 * the host, and leaves the caller's current device as it found it.
 * Has no counterpart in the reference, which has no device code. */
piks_status piks_selftest_division_noalloc(int32_t device, int64_t samples, uint64_t seed, int64_t *mismatches);

/* Self-test of the bounded waits of the dataflow sweep: runs one tile-dataflow sweep of
 * the context in which one job waits on a flag that no job sets. Its wait gives up after
 * its iteration limit (about a second), sets the sweep's error flag, and every job finishes;
 * the call restores the schedule, clears the flag, and stores the sweep's duration in
 * *seconds. Returns PIKS_OK when the wait ran out as designed, PIKS_ERR_STATE when it did not
 * (or the context has no tile schedule). The sweep overwrites f with values that are not the
 * solver's: set the image up again before iterating. Has no counterpart in the reference. */
piks_status piks_selftest_wait_timeout(piks_ctx *ctx, double *seconds);

/* Storage and sweep precision of a context. PIKS_PREC_FP64 (the default) is the
 * reference's arithmetic, operation for operation. PIKS_PREC_FP32 stores f, the 3-fold
 * corner slots and the x ghost planes in FP32 and sweeps in FP32, while the moments
 * (Rho, U), the diffuse-wall densities, the mass flux and the convergence test stay FP64.
 * Switching a context that holds a state converts it on the device (FP32 -> FP64 widens
 * exactly), so an FP32 solve can be continued in FP64: the refinement phase of
 * piks_run_refined. Has no counterpart in the reference, which computes in FP64 only. */
enum { PIKS_PREC_FP64 = 0, PIKS_PREC_FP32 = 1 };
piks_status piks_set_precision(piks_ctx *ctx, int32_t precision);
piks_status piks_get_precision(piks_ctx *ctx, int32_t *precision);

/* Sweep schedule. The default cuts the box into 8x4x4 tiles (4x4x4 when the context is in
 * FP32 at setup) and sweeps, for each octant,
 * the tiles in diagonal order, each tile's local hyperplanes in shared memory (one launch
 * per tile diagonal). tx = 0 selects the per-node hyperplane schedule (one launch per
 * voxel hyperplane u+v+w). Both give identical results; the tile schedule also falls back
 * to the per-node one when a tile needs more rows than shared memory holds. Takes effect
 * at the next piks_setup_physical_grid. No counterpart in the reference (its sweep is a
 * serial raster loop per octant). */
piks_status piks_set_tiles(piks_ctx *ctx, int32_t tx, int32_t ty, int32_t tz);
/* How the tile jobs are launched: PIKS_SCHED_TILE_DIAGONALS (default) launches each tile
 * diagonal separately; PIKS_SCHED_TILE_DATAFLOW runs all jobs of an iteration in one
 * launch, each job waiting for its upwind neighbour tiles through device flags (waits give
 * up after about a second: piks_synchronize / piks_chk_converge then return
 * PIKS_ERR_CUDA); PIKS_SCHED_TILE_COLUMNS runs one persistent launch in which each CTA
 * marches down columns of tiles (one octant, one (x, y) tile position, the octant's z
 * order): a producer warp stages the next tile with bulk asynchronous copies while the
 * other warps sweep the current one, and the tile's last two z layers stay on chip for the
 * next (waits give up after about two seconds, reported as for the dataflow launch);
 * PIKS_SCHED_TILE_PIPELINED runs the same producer / consumer kernel over single jobs taken
 * in diagonal order, each job's upwind rows staged from HBM once their jobs are done, the
 * producer up to three jobs ahead. A change between launch schedules that read different
 * forms of the tile jobs rebuilds them. All give identical values. */
enum { PIKS_SCHED_TILE_DATAFLOW = 0, PIKS_SCHED_TILE_DIAGONALS = 1, PIKS_SCHED_TILE_COLUMNS = 2,
       PIKS_SCHED_TILE_PIPELINED = 3 };
piks_status piks_set_schedule(piks_ctx *ctx, int32_t schedule);
/* Autotuner of the sweep schedule: right after piks_setup_physical_grid (before the first
 * iteration) times `sweeps` sweeps of each candidate (4 int32 each: TX, TY, TZ, launch
 * schedule; NULL / ncand 0 = a built-in list) on this image, keeps the fastest, and resets
 * the state to setupFlow's zeros. chosen (4 int32) receives the winner, ms_out (ncand) the
 * milliseconds per sweep of each candidate (-1 where a candidate does not apply). */
piks_status piks_autotune(piks_ctx *ctx, const int32_t *candidates, int32_t ncand, int32_t sweeps,
                          int32_t *chosen, double *ms_out);
/* [tile schedule in use (0/1), TX, TY, TZ, largest shared-memory slot count of a job,
 *  launch schedule, number of jobs] */
piks_status piks_get_schedule(piks_ctx *ctx, int32_t *out, int32_t n);

/* FP32 solve with FP64 refinement: runs FP32 iterations with chkConverge every
 * chkConvergeStep until error <= switch_eps (or until the error has not reached a new
 * minimum for 5 checks in a row: the FP32 iterate has stopped improving), widens the state
 * to FP64 and continues main.F90's loop in FP64 until error <= eps or maxStep iterations
 * in total. Same files and stdout lines as piks_run; *steps32 receives the FP32
 * iterations, *steps all iterations. No counterpart in the reference (FP64 only). */
piks_status piks_run_refined(piks_ctx *ctx, const char *results_path, const char *out_dir, int32_t verbose,
                             double switch_eps, int32_t *steps32, int32_t *steps, double *permeability,
                             double *seconds);

/* Batches: several solves (contexts with the tile schedule, on one device, of any size,
 * velocity set, Knudsen number and precision) iterated together. One batch iteration runs,
 * per (precision, velocity-chunk) class, a single dataflow launch over the tile jobs of all
 * members, then every member's boundary kernels; after two plain iterations the sequence is
 * captured as a CUDA graph per iteration parity and replayed until the membership changes.
 * Each member's values are those of the same solve run alone. While a context is in a
 * batch, iterate and check it only through the batch. Members may be added and removed
 * between iterations (continuous batching); piks_set_precision on a member is picked up
 * at the next batch iteration. No counterpart in the reference (one image per run). */
typedef struct piks_batch piks_batch;
piks_status piks_batch_create(int32_t device, piks_batch **out);
piks_status piks_batch_add(piks_batch *b, piks_ctx *ctx);
piks_status piks_batch_remove(piks_batch *b, piks_ctx *ctx);
piks_status piks_batch_size(piks_batch *b, int32_t *n);
/* nsteps iterations of every member (asynchronous on the batch's stream). */
piks_status piks_batch_iterate(piks_batch *b, int32_t nsteps);
/* chkConverge of every member (arrays in membership order, any may be NULL). */
piks_status piks_batch_chk_converge(piks_batch *b, double *mass, double *permeability, double *error);
piks_status piks_batch_synchronize(piks_batch *b);
piks_status piks_batch_destroy(piks_batch *b);

piks_status piks_synchronize(piks_ctx *ctx);
piks_status piks_destroy(piks_ctx *ctx);
const char *piks_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
