// Internal host-side structures of libpiks3d_b200 (not part of the C ABI).
#pragma once
#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "piks3d_gpu.h"

namespace piks {

// std::allocator that leaves new elements uninitialised: for the large host arrays that
// are written in full right after they are sized (their pages are then first touched by
// the threads that fill them).
template <typename T>
struct NoInitAlloc : std::allocator<T> {
  template <typename U> struct rebind { using other = NoInitAlloc<U>; };
  NoInitAlloc() = default;
  template <typename U> NoInitAlloc(const NoInitAlloc<U> &) {}
  template <typename U> void construct(U *p) noexcept { ::new (static_cast<void *>(p)) U; }
  template <typename U, typename... A> void construct(U *p, A &&...a) {
    ::new (static_cast<void *>(p)) U(std::forward<A>(a)...);
  }
};
template <typename T> using BigVec = std::vector<T, NoInitAlloc<T>>;

// Voxel labels of PIKS3D (physicalGrid.F90:127-134).
enum : int {
  L_FLUID = 0, L_SOLID = 1, L_GHOST = 4,
  L_E = 20, L_W = 21, L_N = 22, L_S = 23, L_F = 24, L_B = 25,
  L_EN = 30, L_WN = 31, L_ES = 32, L_WS = 33,
  L_NF = 40, L_NB = 41, L_SF = 42, L_SB = 43,
  L_EF = 50, L_EB = 51, L_WF = 52, L_WB = 53,
  L_ENF = 60, L_WNF = 61, L_WSF = 62, L_ESF = 63,
  L_ENB = 70, L_WNB = 71, L_WSB = 72, L_ESB = 73
};

// Fluid-side bits of a wall label: which face neighbours are fluid.
enum : uint8_t { FACE_E = 1, FACE_W = 2, FACE_N = 4, FACE_S = 8, FACE_F = 16, FACE_B = 32 };
uint8_t face_mask(int label);  // 0 for non-wall labels
bool is_wall_label(int label);
bool is_corner3_label(int label);

// Octant o (0-based, the reference's group o+1) velocity signs.
inline int oct_sx(int o) { return (o == 0 || o == 3 || o == 4 || o == 7) ? 1 : -1; }
inline int oct_sy(int o) { return (o == 0 || o == 1 || o == 4 || o == 5) ? 1 : -1; }
inline int oct_sz(int o) { return o < 4 ? 1 : -1; }

// Source code of a resolved read: 0..7 = slot (octant) of the same node, 8 = fw(corner, o).
constexpr int SRC_FW = 8;

// Wall re-emission program (solver.F90:772-1823), shared with the device kernels.
enum { DIR_PX, DIR_MX, DIR_PY, DIR_MY, DIR_PZ, DIR_MZ };
enum { ST_F, ST_Z, ST_W };
struct WFace { int dir, store; };
struct WWrite { int dst_store, dst_o, face, src_store, src_o; };
struct WProg { int label, nface; WFace face[3]; int nwr; WWrite wr[12]; };
const WProg *wall_program(int label);
extern const int kIncoming[6][4];  // 1-based octants arriving from each fluid side

// A wall program resolved for kernels that keep a wall's extrapolated values on chip:
// every write's source is the extrapolation v(face, m) of one of the wall's faces, so a
// write reads it from there; a face value is stored only where no write later replaces
// it (the slot's final content is then the face value).
struct WPlan {
  int nface;
  int dir[3], store[3];
  int keep[3];        // per face: bit m set when v(face, m) is the final content of its slot
  int nwr;
  int dst_store[12], dst_o[12], face[12];  // 0-based destination octant
  int src[12];        // producing face * 4 + m
};
// Resolves `p`; false if some write reads a value that is not a face extrapolation, reads
// a slot that an earlier write replaced, or two writes share a destination.
bool make_wall_plan(const WProg &p, WPlan &out);

struct Velocity {
  int Nc_fundamental = 0, Nc = 0, Nc8 = 0;
  std::vector<double> cx, cy, cz, w;
  double DiffFlux = 0.0;
};

// initParams-adjusted sizes and constants.
struct Setup {
  piks_params p{};
  int Nx = 0, Ny = 0, Nz = 0;              // box after fluidlayer and block_rep
  int Nx_base = 0, Ny_base = 0, Nz_base = 0;
  double ds = 0.0, mu = 0.0;
  // x-only decomposition of the box into slabs, one per rank (mpiParams.F90:150-191 with
  // dims = (nranks, 1, 1)); this rank owns the x planes [xl, xu] (the whole box for one rank)
  int nranks = 1, rank = 0, xl = 1, xu = 0;
};
// Sets the slab of `rank` among `nranks` (the reference's partition of xmax - xmin planes);
// fails when a rank would own fewer than two planes (its neighbours read two of them).
piks_status set_slab(Setup &s, int nranks, int rank, std::string &err);

// Compact device-side geometry produced by preprocess().
struct Geometry {
  int Nx = 0, Ny = 0, Nz = 0, GX = 0, GY = 0, GZ = 0;  // ghosted extents = N + 4
  std::vector<uint8_t> label;      // ghosted labels
  std::vector<int32_t> nodemap;    // ghosted: >= 0 node index, -1 never read, -2 ghost
  int32_t NF = 0, NB = 0;          // nodes [0,NF) fluid (raster order), [NF,NF+NB) solid read by the solver
  std::vector<int32_t> node_g;     // ghosted linear index of each node
  int32_t nWall = 0, nCorner = 0;
  std::vector<int32_t> wall_node;  // vecWall order
  std::vector<int32_t> wall_label;
  std::vector<double> wall_e;      // [nWall][2] extrapolation coefficients
  std::vector<int32_t> wall_corner;
  std::vector<int32_t> wall_nb;    // [nWall][3][2]: node at +d and code at +2d (see kernels)
  std::vector<int32_t> wall_order; // wall indices grouped by dependency level
  std::vector<int32_t> level_start;  // nlevels + 1 offsets into wall_order
  std::vector<int32_t> bcorner;    // [NB] corner index or -1
  std::vector<uint16_t> roles;     // [NB][8] 4-bit sources for reads as y1,y2,z1,z2
  std::vector<int32_t> commit;     // triples (node, octant, src): post-sweep slot content
  std::vector<int32_t> plane_x1, plane_xN;  // [Nz*Ny] node at x=1 / x=Nx or -1
  std::vector<int32_t> sym_node;   // nodes on the y/z boundary planes
  std::vector<uint8_t> sym_flag;   // bit0 y=1, bit1 y=Ny, bit2 z=1, bit3 z=Nz
  std::vector<int32_t> flux_list;  // x=2 plane entries in chkConverge's summation order (west-most slab only)
  // Slab of an x-decomposed box: owned planes [xl, xu]; a side that is not the box's side
  // (wglob / eglob false) has two ghost planes owned by the neighbour rank, whose read
  // voxels are nodes here too (after the fluid nodes, in [NF, NF + NB)).
  int xl = 1, xu = 0;
  bool wglob = true, eglob = true;
  // x halos (side 0 west, 1 east): the nodes whose rows this rank sends (its two planes at
  // that side) and the ghost-plane nodes it receives into; both ranks of a pair list the
  // same voxels in the same order (z, then y, then x)
  std::vector<int32_t> halo_send[2], halo_recv[2];
  bool in_window(int i) const { return i >= (wglob ? 1 : xl - 2) && i <= (eglob ? Nx : xu + 2); }
  // Sweep tasks: one per (swept fluid node, octant), ordered by the hyperplane index
  // u+v+w of the octant's frame; tasks of one hyperplane are independent.
  // Record (8 x int32): node, flags (octant | fx<<3 | fy<<4 | fz<<5), then the value
  // source of the x1, x2, y1, y2, z1, z2 upwind neighbours (row node*8+slot of h, or with
  // bit 30 set row corner*8+octant of fw, or -2 for a ghost that is only multiplied by 0).
  BigVec<int32_t> tasks;
  std::vector<int64_t> hyper_start;   // task offset of each hyperplane (+1 end entry)
  int32_t flux_groups[10] = {0};   // offsets of the 9 partial sums
  int64_t ghost_index(int i, int j, int k) const {
    return (int64_t)(i + 1) + (int64_t)(j + 1) * GX + (int64_t)(k + 1) * GX * GY;
  }
};

// Tile-wavefront form of the sweep tasks. The box is cut into TX x TY x TZ tiles; a job is
// one (tile, octant): its swept fluid nodes, ordered by the local hyperplane index of the
// octant's frame inside the tile (the steps), and the unique rows they read or write.
// Jobs are grouped by the tile hyperplane index of the octant's frame (the diagonals): the
// jobs of one diagonal are independent, and every row a job reads from another tile was
// written by a job of an earlier diagonal.
struct TileJobs {
  int TX = 0, TY = 0, TZ = 0;
  int nsteps = 0;                    // TX + TY + TZ - 2 local hyperplanes per tile
  // rows of each job (global row codes as in Geometry::tasks): the job's own rows first,
  // in task order, then the other rows it reads; shared-memory slot = 1 + position
  // (slot 0 is a row of zeros)
  // (each job's list starts at a multiple of 4 entries, for 16-byte copies)
  BigVec<int32_t> rows;
  std::vector<int64_t> row_begin;    // njobs + 1
  std::vector<int32_t> row_count;    // njobs
  // per task: node | fx<<27 | fy<<28 | fz<<29, then the slots of x1 | x2<<16, y1 | y2<<16,
  // z1 | z2<<16; the task's own slot is 1 + its index within the job
  BigVec<int32_t> tasks;             // 4 int32 per task
  std::vector<int64_t> task_begin;   // njobs + 1
  std::vector<uint16_t> steps;       // [njobs][steps_stride] task offsets within the job
  int steps_stride = 0;              // nsteps + 1 rounded up to a multiple of 8
  std::vector<int32_t> diag_begin;   // job offset of each diagonal (+1 end entry)
  std::vector<int32_t> diag_rows;    // largest slot count (rows + zero row) per diagonal
  std::vector<int32_t> diag_tasks;   // largest task count of a job per diagonal
  // launch plan: the jobs of each diagonal sorted by slot count and cut into size classes,
  // one launch per class, each sized for its largest job
  std::vector<int32_t> job_list;     // job indices in launch order
  std::vector<int32_t> launches;     // per launch: first job_list entry, job count, slots, tasks
  std::vector<int32_t> launch_diag_end;  // launch offset after each diagonal
  std::vector<int32_t> up;           // [njobs][4]: jobs of the upwind x, y, z neighbour tiles (same octant) or -1
  bool paired = false;               // launches sweep job pairs (job_list holds the pairs adjacently)
  int slot_cap = 0;                  // the shared-memory slots one job may use (build_tile_jobs' max_slots)
  int plan_prec = -1;                // precision the launch plan was made for (plan_for_precision)
  int32_t max_rows = 0;              // largest slot count of a job
  int32_t max_tasks = 0;             // largest task count of a job
  // Column form (built with columns = true; only the column-march sweep reads it). A column
  // is one octant's tiles at one (x, y) tile position, in the octant's z sweep order; one CTA
  // runs a column's jobs one after another and keeps the last two z layers of each tile on
  // chip for the next. A job's rows are then its own rows, the static rows (solid, corner
  // and inflow-plane rows, which the sweep never writes) and the dependent rows (own rows of
  // the x- and y-upwind tiles, read once their jobs are done); the rows it reads from the
  // previous tile of its column come from the carried layers instead. Slots: 0 a zero row,
  // 1 .. ncin the carried rows, then the job's rows in that order.
  bool columns = false;
  // Split form (built with form TILE_FORM_SPLIT or TILE_FORM_COLUMNS): rows ordered own,
  // static, dependent, with the per-job headers; without the carried layers (columns false)
  // the rows of the z-upwind tile are dependent rows like the x and y ones. Read by the
  // pipelined dataflow sweep.
  bool split = false;
  std::vector<int32_t> hdr;          // [njobs][8]: row_begin, task_begin, carry_begin, nrows, ntask,
                                     // first dependent row, ncin, ncout
  BigVec<int32_t> carry;             // per job: ncin entries cell | slot << 16, then ncout entries
                                     // own index | cell << 16 (padded to a multiple of 4)
  std::vector<int64_t> carry_begin;  // njobs + 1
  std::vector<int32_t> col_jobs;     // jobs of every column in sweep order
  std::vector<int32_t> col_begin;    // ncols + 1
  std::vector<int32_t> col_list;     // columns in dependency order (x+y tile diagonal of the octant)
  int32_t ncells = 0;                // carried cells: 2 * TX * TY
  int32_t max_region = 0;            // largest 1 + ncin + nrows of a job
  int32_t max_carry = 0;             // largest ncin + ncout of a job, rounded up to 4
  int64_t sum_region = 0;            // sum of 1 + ncin + nrows over the jobs
};

// Builds the tile jobs from g.tasks; returns false when a job needs more than max_slots
// shared-memory rows (the caller then keeps the hyperplane schedule).
// Forms of the tile jobs: slots in first-read order (diagonal, dataflow and batch sweeps),
// split rows (pipelined dataflow sweep), split rows with carried z layers (column march).
enum { TILE_FORM_SLOTS = 0, TILE_FORM_SPLIT = 1, TILE_FORM_COLUMNS = 2 };
bool build_tile_jobs(const Geometry &g, int TX, int TY, int TZ, int max_slots, TileJobs &tj,
                     int form = TILE_FORM_SLOTS);
// (Re)builds the launch plan with at most max_classes size classes per diagonal; a class
// holds the jobs whose slot count is above `ratio` times its largest.
// Launch plan of the diagonals: the jobs of a diagonal by slot count, in up to max_classes
// size classes (one launch each); with `pairs` (one class) the jobs are interleaved largest
// with smallest and each launch record holds the largest slot and task sums of a pair (one
// CTA sweeps a pair, each job in its own part of the CTA's shared memory).
void plan_tile_launches(TileJobs &tj, int max_classes, double ratio, bool pairs);
// The launch plan of a precision: job pairs for the FP64 sweep (when a pair fits the shared
// memory one job may use), single jobs for FP32 (prec: PIKS_PREC_FP64 or PIKS_PREC_FP32).
void plan_for_precision(TileJobs &tj, int prec);

piks_status make_setup(const piks_params &p, Setup &s, std::string &err);
piks_status make_velocity(const piks_params &p, Velocity &v, std::string &err);
piks_status preprocess(const Setup &s, const uint8_t *raw, int64_t nbytes, Geometry &g, std::string &err);
// The stages of preprocess: the ghosted working box after the stream read, block replication
// and the two drill / thin rounds (raster-order passes, physicalGrid.F90:257-422); the
// classification of its voxels into labels, the node map (fluid nodes, then the solid
// nodes the solver reads, both in raster order), the 3-fold corner numbers and the wall
// list (physicalGrid.F90:546-936), on the host or on the device (classify_device,
// preprocess.cu); the rest of the geometry from those (wall levels, switch roles,
// commits, sweep tasks, planes, flux list).
piks_status preprocess_box(const Setup &s, const uint8_t *raw, int64_t nbytes, std::vector<uint8_t> &box,
                           std::string &err);
void classify_host(const Setup &s, const std::vector<uint8_t> &box, Geometry &g);
// classify_host on the current CUDA device (preprocess.cu), identical results; synchronous on
// `stream` (a cudaStream_t).
piks_status classify_device(const Setup &s, const std::vector<uint8_t> &box, Geometry &g, void *stream,
                            std::string &err);
piks_status finish_geometry(const Setup &s, Geometry &g, std::string &err);
void wall_extrapolation(const Setup &s, const Geometry &g, int i, int j, int k, double &e1, double &e2);
void wall_neighbours(const Geometry &g, const WProg *P, int i, int j, int k, int32_t *nb);
piks_status read_namelist(const char *path, piks_params &p, std::string &image_file, std::string &err);
std::string fortran_es15_6(double v);

}  // namespace piks
