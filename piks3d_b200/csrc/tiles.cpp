// Tile-wavefront schedule of the sweep tasks (TileJobs, declared in piks_internal.h).
#include <algorithm>
#include <atomic>
#include <numeric>
#include <thread>

#include "piks_internal.h"

namespace piks {

namespace {

// Number of contiguous chunks parallel_chunks splits [0, n) into (one per thread, up to 16).
int chunk_count(int64_t n) {
  unsigned hw = std::thread::hardware_concurrency();
  int nt = (int)std::min<unsigned>(hw ? hw : 1, 16u);
  return n < 4096 ? 1 : std::max(nt, 1);
}

// Runs fn(chunk, begin, end) over [0, n) split into chunk_count(n) contiguous chunks, one
// thread each.
template <typename F>
void parallel_chunks_indexed(int64_t n, F fn) {
  const int nt = chunk_count(n);
  if (nt <= 1) { fn(0, (int64_t)0, n); return; }
  std::vector<std::thread> th;
  th.reserve((size_t)nt);
  for (int i = 0; i < nt; ++i) {
    const int64_t b = n * i / nt, e = n * (i + 1) / nt;
    th.emplace_back([=, &fn] { fn(i, b, e); });
  }
  for (auto &t : th) t.join();
}

// Runs fn(begin, end) over [0, n) split into contiguous chunks on up to 16 threads.
template <typename F>
void parallel_chunks(int64_t n, F fn) {
  parallel_chunks_indexed(n, [&fn](int, int64_t b, int64_t e) { fn(b, e); });
}

// Row de-duplication inside one job: open addressing on the row index, cleared by a
// generation count.
struct RowSet {
  std::vector<int64_t> key;
  std::vector<int32_t> val, gen;
  int32_t cur = 0;
  unsigned mask = 0;
  explicit RowSet(unsigned cap) : key(cap), val(cap), gen(cap, -1), mask(cap - 1) {}
  void clear() { ++cur; }
  // slot of `k`, inserting `next` if absent (then *added = true)
  int32_t find_or_add(int64_t k, int32_t next, bool *added) {
    unsigned h = (unsigned)((uint64_t)k * 0x9E3779B97F4A7C15ull >> 40) & mask;
    for (;;) {
      if (gen[h] != cur) { gen[h] = cur; key[h] = k; val[h] = next; *added = true; return next; }
      if (key[h] == k) { *added = false; return val[h]; }
      h = (h + 1) & mask;
    }
  }
};

// Rows, task records, steps, carried layers and column lists of the column form (see
// TileJobs). Returns false when a job reads a row of a tile that is not its own or one of
// its three upwind neighbours, or needs more shared-memory rows than `max_slots`.
bool build_column_rows(const Geometry &g, TileJobs &tj, const BigVec<int64_t> &order, int32_t njobs,
                       const std::vector<int64_t> &job_pair, int64_t ntiles, int nTx, int nTy, int nTz, int max_slots,
                       unsigned cap, const BigVec<uint16_t> &step, bool carry_z) {
  const int TX = tj.TX, TY = tj.TY, TZ = tj.TZ;
  const int64_t GX = g.GX, GXY = (int64_t)g.GX * g.GY;
  const int64_t nrows_h = ((int64_t)g.NF + g.NB) * 8;
  tj.columns = carry_z;
  tj.split = true;
  tj.ncells = carry_z ? 2 * TX * TY : 0;
  // owner job and own index of every swept h row
  BigVec<int32_t> job_of_row((size_t)nrows_h);
  BigVec<uint16_t> own_of_row((size_t)nrows_h);
  parallel_chunks(nrows_h, [&](int64_t b, int64_t e) { std::fill(job_of_row.begin() + b, job_of_row.begin() + e, -1); });
  parallel_chunks(njobs, [&](int64_t jb, int64_t je) {
    for (int64_t j = jb; j < je; ++j)
      for (int64_t p = tj.task_begin[(size_t)j]; p < tj.task_begin[(size_t)j + 1]; ++p) {
        const int32_t *r = &g.tasks[(size_t)order[(size_t)p] * 8];
        const int64_t row = (int64_t)r[0] * 8 + (r[1] & 7);
        job_of_row[(size_t)row] = (int32_t)j;
        own_of_row[(size_t)row] = (uint16_t)(p - tj.task_begin[(size_t)j]);
      }
  });
  // carried cell of a node in the two z layers of tile-z index c nearest to the next tile in
  // the octant's sweep order (-1 when the node is not in them)
  auto cell_of = [&](int32_t node, int o, int c) -> int {
    if (!carry_z) return -1;
    const int64_t gi = g.node_g[(size_t)node];
    const int x = (int)(gi % GX) - 2, y = (int)((gi / GX) % g.GY) - 2, z = (int)(gi / GXY) - 2;
    if (z / TZ != c) return -1;
    const int layer = oct_sz(o) > 0 ? z - (c * TZ + TZ - 2) : (c * TZ + 1) - z;
    if (layer < 0 || layer > 1) return -1;
    return layer * TX * TY + (y % TY) * TX + (x % TX);
  };
  auto row_index = [&](int32_t code) -> int64_t {
    return (code & (1 << 30)) ? nrows_h + (code & ~(1 << 30)) : (int64_t)code;
  };
  std::vector<int32_t> ncin((size_t)njobs), ncout((size_t)njobs), nstat((size_t)njobs), ndep((size_t)njobs);
  std::vector<char> bad((size_t)njobs, 0);
  // pass 1: counts
  unsigned ccap = 64;
  while (ccap < (unsigned)(4 * TX * TY)) ccap <<= 1;
  parallel_chunks(njobs, [&](int64_t jb, int64_t je) {
    RowSet cin(ccap), stat(cap), dep(cap);
    for (int64_t j = jb; j < je; ++j) {
      cin.clear(); stat.clear(); dep.clear();
      const int64_t pr = job_pair[(size_t)j];
      const int o = (int)(pr / ntiles);
      const int c = (int)((pr % ntiles) / ((int64_t)nTx * nTy));
      const int32_t ux = tj.up[(size_t)j * 4], uy = tj.up[(size_t)j * 4 + 1], uz = tj.up[(size_t)j * 4 + 2];
      int32_t ni = 0, ns = 0, nd = 0, no = 0;
      bool added;
      for (int64_t p = tj.task_begin[(size_t)j]; p < tj.task_begin[(size_t)j + 1]; ++p) {
        const int32_t *r = &g.tasks[(size_t)order[(size_t)p] * 8];
        if (cell_of(r[0], o, c) >= 0) ++no;
        for (int k = 0; k < 6; ++k) {
          const int32_t code = r[2 + k];
          if (code < 0) continue;
          const int32_t jq = (code & (1 << 30)) ? -1 : job_of_row[(size_t)code];
          if (jq < 0) { stat.find_or_add(row_index(code), ns, &added); ns += added; continue; }
          if (jq == (int32_t)j) continue;
          if (carry_z && jq == uz && k >= 4) {
            const int cell = cell_of(code >> 3, o, c - oct_sz(o));
            if (cell < 0) { bad[(size_t)j] = 1; break; }
            cin.find_or_add(cell, ni, &added); ni += added;
          } else if (jq == ux || jq == uy || (!carry_z && jq == uz && k >= 4)) {
            dep.find_or_add(row_index(code), nd, &added); nd += added;
          } else {
            bad[(size_t)j] = 1;
            break;
          }
        }
      }
      const int32_t nt = (int32_t)(tj.task_begin[(size_t)j + 1] - tj.task_begin[(size_t)j]);
      ncin[(size_t)j] = ni; ncout[(size_t)j] = no; nstat[(size_t)j] = ns; ndep[(size_t)j] = nd;
      if (1 + ni + nt + ns + nd > max_slots) bad[(size_t)j] = 1;
    }
  });
  for (int32_t j = 0; j < njobs; ++j)
    if (bad[(size_t)j]) return false;
  tj.row_count.assign((size_t)njobs, 0);
  tj.row_begin.assign((size_t)njobs + 1, 0);
  tj.carry_begin.assign((size_t)njobs + 1, 0);
  for (int32_t j = 0; j < njobs; ++j) {
    const int32_t nt = (int32_t)(tj.task_begin[(size_t)j + 1] - tj.task_begin[(size_t)j]);
    tj.row_count[(size_t)j] = nt + nstat[(size_t)j] + ndep[(size_t)j];
    tj.row_begin[(size_t)j + 1] = tj.row_begin[(size_t)j] + (tj.row_count[(size_t)j] + 3) / 4 * 4;
    tj.carry_begin[(size_t)j + 1] = tj.carry_begin[(size_t)j] + (ncin[(size_t)j] + ncout[(size_t)j] + 3) / 4 * 4;
  }
  // the device addresses these arrays with 32-bit offsets
  if (tj.row_begin.back() + 4 > INT32_MAX || tj.task_begin.back() > INT32_MAX || tj.carry_begin.back() + 4 > INT32_MAX)
    return false;
  // (+4: bulk copies move whole 16-byte pieces past a job's last entry)
  tj.rows.assign((size_t)tj.row_begin.back() + 4, 0);
  tj.carry.assign((size_t)tj.carry_begin.back() + 4, 0);
  tj.tasks.resize((size_t)tj.task_begin.back() * 4);
  tj.steps.assign((size_t)njobs * tj.steps_stride, 0);
  tj.hdr.assign((size_t)njobs * 8, 0);
  // pass 2: slots and records
  parallel_chunks(njobs, [&](int64_t jb, int64_t je) {
    RowSet cin(ccap), stat(cap), dep(cap);
    for (int64_t j = jb; j < je; ++j) {
      cin.clear(); stat.clear(); dep.clear();
      const int64_t pr = job_pair[(size_t)j];
      const int o = (int)(pr / ntiles);
      const int c = (int)((pr % ntiles) / ((int64_t)nTx * nTy));
      const int32_t uz = tj.up[(size_t)j * 4 + 2];
      const int64_t q = tj.task_begin[(size_t)j], e = tj.task_begin[(size_t)j + 1];
      const int32_t nt = (int32_t)(e - q), ni = ncin[(size_t)j], ns = nstat[(size_t)j];
      int32_t *rows = &tj.rows[(size_t)tj.row_begin[(size_t)j]];
      int32_t *cl = &tj.carry[(size_t)tj.carry_begin[(size_t)j]];
      const int32_t own0 = 1 + ni;
      int32_t ci = 0, si = 0, di = 0, co = 0;
      bool added;
      for (int64_t p = q; p < e; ++p) {
        const int32_t *r = &g.tasks[(size_t)order[(size_t)p] * 8];
        rows[p - q] = r[0] * 8 + (r[1] & 7);
        const int cell = cell_of(r[0], o, c);
        if (cell >= 0) cl[ni + co++] = (int32_t)(p - q) | (cell << 16);
      }
      for (int64_t p = q; p < e; ++p) {
        const int32_t *r = &g.tasks[(size_t)order[(size_t)p] * 8];
        int32_t sl[6];
        for (int k = 0; k < 6; ++k) {
          const int32_t code = r[2 + k];
          if (code < 0) { sl[k] = 0; continue; }
          const int32_t jq = (code & (1 << 30)) ? -1 : job_of_row[(size_t)code];
          if (jq < 0) {
            const int32_t idx = stat.find_or_add(row_index(code), si, &added);
            if (added) rows[nt + si++] = code;
            sl[k] = own0 + nt + idx;
          } else if (jq == (int32_t)j) {
            sl[k] = own0 + own_of_row[(size_t)code];
          } else if (carry_z && jq == uz && k >= 4) {
            const int cell = cell_of(code >> 3, o, c - oct_sz(o));
            const int32_t idx = cin.find_or_add(cell, ci, &added);
            if (added) { cl[ci] = cell | ((1 + ci) << 16); ++ci; }
            sl[k] = 1 + idx;
          } else {
            const int32_t idx = dep.find_or_add(row_index(code), di, &added);
            if (added) rows[nt + ns + di++] = code;
            sl[k] = own0 + nt + ns + idx;
          }
        }
        const int fl = r[1];
        int32_t *tr = &tj.tasks[(size_t)p * 4];
        tr[0] = r[0] | ((fl & 8) ? 1 << 27 : 0) | ((fl & 16) ? 1 << 28 : 0) | ((fl & 32) ? 1 << 29 : 0);
        tr[1] = sl[0] | (sl[1] << 16);
        tr[2] = sl[2] | (sl[3] << 16);
        tr[3] = sl[4] | (sl[5] << 16);
      }
      uint16_t *st = &tj.steps[(size_t)j * tj.steps_stride];
      for (int64_t p = q; p < e; ++p) st[step[(size_t)order[(size_t)p]] + 1]++;
      for (int s2 = 0; s2 < tj.nsteps; ++s2) st[s2 + 1] = (uint16_t)(st[s2 + 1] + st[s2]);
      int32_t *h = &tj.hdr[(size_t)j * 8];
      h[0] = (int32_t)tj.row_begin[(size_t)j];
      h[1] = (int32_t)q;
      h[2] = (int32_t)tj.carry_begin[(size_t)j];
      h[3] = tj.row_count[(size_t)j];
      h[4] = nt;
      h[5] = nt + ns;
      h[6] = ni;
      h[7] = co;
    }
  });
  tj.max_region = 0;
  tj.max_carry = 0;
  tj.sum_region = 0;
  for (int32_t j = 0; j < njobs; ++j) {
    const int32_t reg = 1 + ncin[(size_t)j] + tj.row_count[(size_t)j];
    tj.max_region = std::max(tj.max_region, reg);
    tj.sum_region += reg;
    tj.max_carry = std::max(tj.max_carry, (ncin[(size_t)j] + ncout[(size_t)j] + 3) / 4 * 4);
  }
  // columns: (octant, x tile, y tile), their jobs in the octant's z order, listed by the
  // x+y tile diagonal of the octant's frame (every upwind column comes first)
  const int64_t ncol_all = (int64_t)8 * nTx * nTy;
  std::vector<int32_t> job_at((size_t)ntiles * 8, -1);
  for (int32_t j = 0; j < njobs; ++j) job_at[(size_t)job_pair[(size_t)j]] = j;
  tj.col_begin.assign(1, 0);
  tj.col_jobs.clear();
  std::vector<std::pair<int, int32_t>> keyed;
  for (int64_t col = 0; col < ncol_all; ++col) {
    const int o = (int)(col / ((int64_t)nTx * nTy));
    const int a = (int)(col % nTx), b = (int)((col / nTx) % nTy);
    const size_t before = tj.col_jobs.size();
    for (int k = 0; k < nTz; ++k) {
      const int cz = oct_sz(o) > 0 ? k : nTz - 1 - k;
      const int32_t j = job_at[(size_t)((int64_t)o * ntiles + a + (int64_t)nTx * (b + (int64_t)nTy * cz))];
      if (j >= 0) tj.col_jobs.push_back(j);
    }
    if (tj.col_jobs.size() == before) continue;
    const int d = (oct_sx(o) > 0 ? a : nTx - 1 - a) + (oct_sy(o) > 0 ? b : nTy - 1 - b);
    keyed.push_back({d, (int32_t)(tj.col_begin.size() - 1)});
    tj.col_begin.push_back((int32_t)tj.col_jobs.size());
  }
  std::stable_sort(keyed.begin(), keyed.end(),
                   [](const std::pair<int, int32_t> &x, const std::pair<int, int32_t> &y) { return x.first < y.first; });
  tj.col_list.resize(keyed.size());
  for (size_t i = 0; i < keyed.size(); ++i) tj.col_list[i] = keyed[i].second;
  return true;
}

}  // namespace

bool build_tile_jobs(const Geometry &g, int TX, int TY, int TZ, int max_slots, TileJobs &tj, int form) {
  tj = TileJobs{};
  tj.TX = TX; tj.TY = TY; tj.TZ = TZ;
  tj.nsteps = TX + TY + TZ - 2;
  tj.steps_stride = (tj.nsteps + 1 + 7) / 8 * 8;
  if (max_slots > 65535) max_slots = 65535;  // slots are stored in 16 bits
  const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
  const int nTx = (Nx + TX - 1) / TX, nTy = (Ny + TY - 1) / TY, nTz = (Nz + TZ - 1) / TZ;
  const int ndiag = nTx + nTy + nTz - 2;
  const int64_t ntiles = (int64_t)nTx * nTy * nTz;
  const int64_t GX = g.GX, GXY = (int64_t)g.GX * g.GY;
  const int64_t ntask = (int64_t)(g.tasks.size() / 8);
  const int nsteps = tj.nsteps;
  // (octant, tile) pair and local step of every task. A node's ghosted coordinates are
  // found once (its octants are up to eight tasks); the tile of a coordinate and its local
  // position from either side come from per-axis tables over the ghosted extent.
  struct AxisTable { std::vector<int32_t> tile, pos, neg; };
  auto axis_table = [](int G, int N, int T) {
    AxisTable t{std::vector<int32_t>((size_t)G), std::vector<int32_t>((size_t)G), std::vector<int32_t>((size_t)G)};
    for (int X = 0; X < G; ++X) {
      const int x = X - 2, a = x / T, hi = std::min((a + 1) * T, N) - 1;
      t.tile[(size_t)X] = a;
      t.pos[(size_t)X] = x - a * T;
      t.neg[(size_t)X] = hi - x;
    }
    return t;
  };
  const AxisTable ax = axis_table(g.GX, Nx, TX), ay = axis_table(g.GY, Ny, TY), az = axis_table(g.GZ, Nz, TZ);
  const int64_t nnode = (int64_t)g.node_g.size();
  BigVec<uint64_t> xyz((size_t)nnode);  // X | Y << 21 | Z << 42 (ghosted coordinates)
  parallel_chunks(nnode, [&](int64_t b, int64_t e) {
    for (int64_t n = b; n < e; ++n) {
      const int64_t gi = g.node_g[(size_t)n];
      xyz[(size_t)n] = (uint64_t)(gi % GX) | ((uint64_t)((gi / GX) % g.GY) << 21) | ((uint64_t)(gi / GXY) << 42);
    }
  });
  BigVec<int32_t> pair_of((size_t)ntask);
  BigVec<uint16_t> step((size_t)ntask);
  parallel_chunks(ntask, [&](int64_t b, int64_t e) {
    for (int64_t t = b; t < e; ++t) {
      const int32_t *r = &g.tasks[(size_t)t * 8];
      const int node = r[0], o = r[1] & 7;
      const uint64_t q = xyz[(size_t)node];
      const size_t X = (size_t)(q & 0x1FFFFF), Y = (size_t)((q >> 21) & 0x1FFFFF), Z = (size_t)(q >> 42);
      const int a = ax.tile[X], bb = ay.tile[Y], c = az.tile[Z];
      const int u = oct_sx(o) > 0 ? ax.pos[X] : ax.neg[X];
      const int v = oct_sy(o) > 0 ? ay.pos[Y] : ay.neg[Y];
      const int w = oct_sz(o) > 0 ? az.pos[Z] : az.neg[Z];
      step[(size_t)t] = (uint16_t)(u + v + w);
      pair_of[(size_t)t] = (int32_t)((int64_t)o * ntiles + a + (int64_t)nTx * (bb + (int64_t)nTy * c));
    }
  });
  // The passes over all tasks below run one thread per octant: the pairs, jobs and output
  // positions of different octants are disjoint, and each thread visits its tasks in order.
  // The tasks lie in hyperplane order with a hyperplane's octants one after another, so an
  // octant's tasks form one segment per hyperplane (found by binary search) and a thread
  // visits only its octant's segments; should the tasks not be grouped that way, the count
  // pass misses tasks and every pass falls back to scanning all tasks.
  std::vector<std::vector<std::pair<int64_t, int64_t>>> oct_seg(8);
  {
    const auto &hs = g.hyper_start;
    auto oct = [&](int64_t t) { return g.tasks[(size_t)t * 8 + 1] & 7; };
    for (size_t h = 0; h + 1 < hs.size(); ++h) {
      int64_t b = hs[h];
      const int64_t e = hs[h + 1];
      for (int o = 0; o < 8; ++o) {
        int64_t lo = b, hi = e;  // first task in [b, e) whose octant is above o
        while (lo < hi) {
          const int64_t m = lo + (hi - lo) / 2;
          if (oct(m) <= o) lo = m + 1; else hi = m;
        }
        if (lo > b) oct_seg[(size_t)o].push_back({b, lo});
        b = lo;
      }
    }
  }
  bool segmented = true;
  // fn(lo, hi, begin, end): the octant's pairs are [lo, hi), its tasks lie among [begin, end)
  auto by_octant = [&](auto fn) {
    auto run = [&](int o) {
      const int64_t lo = (int64_t)o * ntiles, hi = lo + ntiles;
      if (segmented) {
        for (const auto &sg : oct_seg[(size_t)o]) fn(lo, hi, sg.first, sg.second);
      } else {
        fn(lo, hi, (int64_t)0, ntask);
      }
    };
    if (ntask < 4096) { for (int o = 0; o < 8; ++o) run(o); return; }
    std::vector<std::thread> th;
    for (int o = 0; o < 8; ++o) th.emplace_back([&run, o] { run(o); });
    for (auto &x : th) x.join();
  };
  // jobs = non-empty pairs, ordered by (diagonal * 8 + octant), then tile (counting sort)
  const int64_t npairs = ntiles * 8;
  std::vector<int32_t> pair_tasks((size_t)npairs, 0);
  std::atomic<int64_t> counted{0};
  auto count_pairs = [&](int64_t lo, int64_t hi, int64_t tb, int64_t te) {
    int64_t k = 0;
    for (int64_t t = tb; t < te; ++t) {
      const int64_t pr = pair_of[(size_t)t];
      if (pr >= lo && pr < hi) { pair_tasks[(size_t)pr]++; ++k; }
    }
    counted += k;
  };
  by_octant(count_pairs);
  if (counted.load() != ntask) {
    segmented = false;
    counted = 0;
    std::fill(pair_tasks.begin(), pair_tasks.end(), 0);
    by_octant(count_pairs);
  }
  auto dio_of = [&](int64_t pr) {
    const int o = (int)(pr / ntiles);
    const int64_t tl = pr % ntiles;
    const int a = (int)(tl % nTx), bb = (int)((tl / nTx) % nTy), c = (int)(tl / ((int64_t)nTx * nTy));
    const int diag = (oct_sx(o) > 0 ? a : nTx - 1 - a) + (oct_sy(o) > 0 ? bb : nTy - 1 - bb) +
                     (oct_sz(o) > 0 ? c : nTz - 1 - c);
    return diag * 8 + o;
  };
  std::vector<int64_t> dcnt((size_t)ndiag * 8 + 1, 0);
  for (int64_t pr = 0; pr < npairs; ++pr)
    if (pair_tasks[(size_t)pr]) dcnt[(size_t)dio_of(pr) + 1]++;
  for (size_t k = 1; k < dcnt.size(); ++k) dcnt[k] += dcnt[k - 1];
  const int32_t njobs = (int32_t)dcnt.back();
  std::vector<int64_t> job_pair((size_t)njobs);
  std::vector<int32_t> job_of_pair((size_t)npairs, -1);
  {
    // within one (diagonal, octant) the pairs of one octant come in tile order
    std::vector<int64_t> pos(dcnt.begin(), dcnt.end() - 1);
    for (int o = 0; o < 8; ++o)
      for (int64_t tl = 0; tl < ntiles; ++tl) {
        const int64_t pr = (int64_t)o * ntiles + tl;
        if (!pair_tasks[(size_t)pr]) continue;
        const int64_t j = pos[(size_t)dio_of(pr)]++;
        job_pair[(size_t)j] = pr;
        job_of_pair[(size_t)pr] = (int32_t)j;
      }
  }
  // tasks in job order, then local step, then their original order (stable placement)
  tj.task_begin.assign((size_t)njobs + 1, 0);
  for (int32_t j = 0; j < njobs; ++j)
    tj.task_begin[(size_t)j + 1] = tj.task_begin[(size_t)j] + pair_tasks[(size_t)job_pair[(size_t)j]];
  std::vector<int32_t> jstep((size_t)njobs * nsteps + 1, 0);  // tasks per (job, step), then positions
  by_octant([&](int64_t lo, int64_t hi, int64_t tb, int64_t te) {
    for (int64_t t = tb; t < te; ++t) {
      const int64_t pr = pair_of[(size_t)t];
      if (pr >= lo && pr < hi) jstep[(size_t)job_of_pair[(size_t)pr] * nsteps + step[(size_t)t]]++;
    }
  });
  {
    int64_t acc = 0;
    for (size_t k = 0; k + 1 < jstep.size(); ++k) { const int32_t c = jstep[k]; jstep[k] = (int32_t)acc; acc += c; }
  }
  BigVec<int64_t> order((size_t)ntask);
  by_octant([&](int64_t lo, int64_t hi, int64_t tb, int64_t te) {
    for (int64_t t = tb; t < te; ++t) {
      const int64_t pr = pair_of[(size_t)t];
      if (pr >= lo && pr < hi) order[(size_t)jstep[(size_t)job_of_pair[(size_t)pr] * nsteps + step[(size_t)t]]++] = t;
    }
  });
  jstep.clear(); jstep.shrink_to_fit();
  pair_of.clear(); pair_of.shrink_to_fit();

  // upstream jobs: the neighbour tiles on the upwind side of each axis, same octant
  tj.up.assign((size_t)njobs * 4, -1);
  for (int32_t j = 0; j < njobs; ++j) {
    const int64_t pr = job_pair[(size_t)j];
    const int o = (int)(pr / ntiles);
    const int64_t t = pr % ntiles;
    const int a = (int)(t % nTx), b = (int)((t / nTx) % nTy), c = (int)(t / ((int64_t)nTx * nTy));
    const int na = a - oct_sx(o), nb = b - oct_sy(o), nc = c - oct_sz(o);
    const int64_t base = (int64_t)o * ntiles;
    if (na >= 0 && na < nTx) tj.up[(size_t)j * 4 + 0] = job_of_pair[(size_t)(base + na + (int64_t)nTx * (b + (int64_t)nTy * c))];
    if (nb >= 0 && nb < nTy) tj.up[(size_t)j * 4 + 1] = job_of_pair[(size_t)(base + a + (int64_t)nTx * (nb + (int64_t)nTy * c))];
    if (nc >= 0 && nc < nTz) tj.up[(size_t)j * 4 + 2] = job_of_pair[(size_t)(base + a + (int64_t)nTx * (b + (int64_t)nTy * nc))];
  }
  const int64_t nrows_h = ((int64_t)g.NF + g.NB) * 8;
  auto row_index = [&](int32_t code) -> int64_t {
    return (code & (1 << 30)) ? nrows_h + (code & ~(1 << 30)) : (int64_t)code;
  };
  unsigned cap = 64;
  while (cap < (unsigned)std::max(2 * max_slots, 64)) cap <<= 1;
  if (form != TILE_FORM_SLOTS) {
    if (!build_column_rows(g, tj, order, njobs, job_pair, ntiles, nTx, nTy, nTz, max_slots, cap, step,
                           form == TILE_FORM_COLUMNS))
      return false;
  } else {
  // pass 1: rows (slots - 1) of every job
  tj.row_count.assign((size_t)njobs, 0);
  parallel_chunks(njobs, [&](int64_t jb, int64_t je) {
    RowSet set(cap);
    for (int64_t j = jb; j < je; ++j) {
      set.clear();
      const int64_t q = tj.task_begin[(size_t)j], e = tj.task_begin[(size_t)j + 1];
      int32_t n = 0;
      bool added;
      // both loops stop at max_slots rows (the job is then too large for the tile shape), so
      // the set never holds more than max_slots + 6 rows, within its capacity
      for (int64_t p = q; p < e && n < max_slots; ++p) {
        const int32_t *r = &g.tasks[(size_t)order[(size_t)p] * 8];
        set.find_or_add(r[0] * 8 + (r[1] & 7), n + 1, &added);
        n += added;
      }
      for (int64_t p = q; p < e && n < max_slots; ++p) {
        const int32_t *r = &g.tasks[(size_t)order[(size_t)p] * 8];
        for (int k = 0; k < 6; ++k) {
          const int32_t code = r[2 + k];
          if (code < 0) continue;
          set.find_or_add(row_index(code), n + 1, &added);
          n += added;
        }
      }
      tj.row_count[(size_t)j] = n;
    }
  });
  for (int32_t j = 0; j < njobs; ++j)
    if (tj.row_count[(size_t)j] + 1 > max_slots) return false;
  tj.row_begin.assign((size_t)njobs + 1, 0);
  for (int32_t j = 0; j < njobs; ++j)
    tj.row_begin[(size_t)j + 1] = tj.row_begin[(size_t)j] + (tj.row_count[(size_t)j] + 3) / 4 * 4;
  tj.rows.resize((size_t)tj.row_begin.back());  // written below, padding included
  tj.tasks.resize((size_t)ntask * 4);
  tj.steps.assign((size_t)njobs * tj.steps_stride, 0);
  // pass 2: rows (own rows first, in task order, then the others as first read), task
  // records with slots, local step offsets
  parallel_chunks(njobs, [&](int64_t jb, int64_t je) {
    RowSet set(cap);
    for (int64_t j = jb; j < je; ++j) {
      set.clear();
      const int64_t q = tj.task_begin[(size_t)j], e = tj.task_begin[(size_t)j + 1];
      int32_t *rows = &tj.rows[(size_t)tj.row_begin[(size_t)j]];
      int32_t n = 0;
      bool added;
      for (int64_t p = q; p < e; ++p) {
        const int32_t *r = &g.tasks[(size_t)order[(size_t)p] * 8];
        const int32_t own = r[0] * 8 + (r[1] & 7);
        set.find_or_add(own, n + 1, &added);
        if (added) rows[n++] = own;
      }
      for (int64_t p = q; p < e; ++p) {
        const int32_t *r = &g.tasks[(size_t)order[(size_t)p] * 8];
        int32_t sl[6];
        for (int k = 0; k < 6; ++k) {
          const int32_t code = r[2 + k];
          if (code < 0) { sl[k] = 0; continue; }
          sl[k] = set.find_or_add(row_index(code), n + 1, &added);
          if (added) rows[n++] = code;
        }
        const int fl = r[1];
        int32_t *tr = &tj.tasks[(size_t)p * 4];
        tr[0] = r[0] | ((fl & 8) ? 1 << 27 : 0) | ((fl & 16) ? 1 << 28 : 0) | ((fl & 32) ? 1 << 29 : 0);
        tr[1] = sl[0] | (sl[1] << 16);
        tr[2] = sl[2] | (sl[3] << 16);
        tr[3] = sl[4] | (sl[5] << 16);
      }
      for (int32_t k = n; k < (int32_t)(tj.row_begin[(size_t)j + 1] - tj.row_begin[(size_t)j]); ++k) rows[k] = 0;
      uint16_t *st = &tj.steps[(size_t)j * tj.steps_stride];
      for (int64_t p = q; p < e; ++p) st[step[(size_t)order[(size_t)p]] + 1]++;
      for (int s2 = 0; s2 < nsteps; ++s2) st[s2 + 1] = (uint16_t)(st[s2 + 1] + st[s2]);
    }
  });
  }
  // per-diagonal bounds
  tj.diag_begin.assign((size_t)ndiag + 1, 0);
  tj.diag_rows.assign((size_t)ndiag, 0);
  tj.diag_tasks.assign((size_t)ndiag, 0);
  for (int32_t j = 0; j < njobs; ++j) {
    const int diag = dio_of(job_pair[(size_t)j]) / 8;
    const int32_t nslots = tj.row_count[(size_t)j] + 1;
    const int32_t nt = (int32_t)(tj.task_begin[(size_t)j + 1] - tj.task_begin[(size_t)j]);
    tj.diag_rows[(size_t)diag] = std::max(tj.diag_rows[(size_t)diag], nslots);
    tj.diag_tasks[(size_t)diag] = std::max(tj.diag_tasks[(size_t)diag], nt);
    tj.max_rows = std::max(tj.max_rows, nslots);
    tj.max_tasks = std::max(tj.max_tasks, nt);
    tj.diag_begin[(size_t)diag + 1] = j + 1;
  }
  for (int d = 0; d < ndiag; ++d) tj.diag_begin[(size_t)d + 1] = std::max(tj.diag_begin[(size_t)d + 1], tj.diag_begin[(size_t)d]);
  tj.slot_cap = max_slots;
  plan_tile_launches(tj, 1, 0.0, false);
  return true;
}

// Pairs for FP64 (measured on B200, 128^3 pack, 512 velocities, sweep per iteration: FP64
// 5.27 ms with pairs against 5.42 without; FP32 3.06 against 2.66, so FP32 keeps single jobs).
void plan_for_precision(TileJobs &tj, int prec) {
  const bool pairs = prec == PIKS_PREC_FP64;
  plan_tile_launches(tj, 1, 0.0, pairs);
  // a pair must fit the shared memory one job may use; its task records take up to one
  // tile's worth more than a single job's (48 bytes each, at most one slot's worth apiece)
  if (pairs)
    for (size_t k = 0; k + 3 < tj.launches.size(); k += 4)
      if (tj.launches[k + 2] + tj.TX * tj.TY * tj.TZ + 4 > tj.slot_cap) {
        plan_tile_launches(tj, 1, 0.0, false);
        break;
      }
  tj.plan_prec = prec;
}

void plan_tile_launches(TileJobs &tj, int max_classes, double ratio, bool pairs) {
  tj.job_list.clear();
  tj.launches.clear();
  tj.launch_diag_end.clear();
  tj.paired = pairs && max_classes == 1;
  const size_t ndiag = tj.diag_begin.empty() ? 0 : tj.diag_begin.size() - 1;
  std::vector<int32_t> jobs;
  for (size_t d = 0; d < ndiag; ++d) {
    jobs.clear();
    for (int32_t j = tj.diag_begin[d]; j < tj.diag_begin[d + 1]; ++j) jobs.push_back(j);
    std::stable_sort(jobs.begin(), jobs.end(),
                     [&](int32_t a, int32_t b) { return tj.row_count[(size_t)a] > tj.row_count[(size_t)b]; });
    if (tj.paired) {
      // largest with smallest: pair k = (jobs[k], jobs[n - 1 - k]), a lone middle job last
      const size_t n = jobs.size();
      if (!n) { tj.launch_diag_end.push_back((int32_t)(tj.launches.size() / 4)); continue; }
      const int32_t first = (int32_t)tj.job_list.size();
      int32_t smax = 0, tmax = 0;
      auto ntask = [&](int32_t j) { return (int32_t)(tj.task_begin[(size_t)j + 1] - tj.task_begin[(size_t)j]); };
      for (size_t k = 0; k < n / 2; ++k) {
        const int32_t ja = jobs[k], jb = jobs[n - 1 - k];
        tj.job_list.push_back(ja);
        tj.job_list.push_back(jb);
        smax = std::max(smax, tj.row_count[(size_t)ja] + tj.row_count[(size_t)jb] + 2);
        tmax = std::max(tmax, ntask(ja) + ntask(jb));
      }
      if (n & 1) {
        const int32_t jm = jobs[n / 2];
        tj.job_list.push_back(jm);
        smax = std::max(smax, tj.row_count[(size_t)jm] + 1);
        tmax = std::max(tmax, ntask(jm));
      }
      tj.launches.push_back(first);
      tj.launches.push_back((int32_t)n);
      tj.launches.push_back(smax);
      tj.launches.push_back(tmax);
      tj.launch_diag_end.push_back((int32_t)(tj.launches.size() / 4));
      continue;
    }
    size_t q = 0;
    int classes = 0;
    while (q < jobs.size()) {
      const int32_t top = tj.row_count[(size_t)jobs[q]];
      size_t e = q;
      int32_t tmax = 0;
      while (e < jobs.size() && (classes + 1 == max_classes || tj.row_count[(size_t)jobs[e]] > ratio * top)) {
        tmax = std::max(tmax, (int32_t)(tj.task_begin[(size_t)jobs[e] + 1] - tj.task_begin[(size_t)jobs[e]]));
        ++e;
      }
      tj.launches.push_back((int32_t)tj.job_list.size());
      tj.launches.push_back((int32_t)(e - q));
      tj.launches.push_back(top + 1);
      tj.launches.push_back(tmax);
      for (size_t k = q; k < e; ++k) tj.job_list.push_back(jobs[k]);
      ++classes;
      q = e;
    }
    tj.launch_diag_end.push_back((int32_t)(tj.launches.size() / 4));
  }
}

}  // namespace piks
