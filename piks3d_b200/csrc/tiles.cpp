// Tile-wavefront schedule of the sweep tasks (TileJobs, declared in piks_internal.h).
#include <algorithm>
#include <numeric>

#include "piks_internal.h"

namespace piks {

bool build_tile_jobs(const Geometry &g, int TX, int TY, int TZ, int max_slots, TileJobs &tj) {
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
  const size_t ntask = g.tasks.size() / 8;
  // job of every task: (diagonal, octant) and tile; local step inside the tile
  std::vector<int32_t> dio(ntask);   // diagonal * 8 + octant
  std::vector<int64_t> tile(ntask);
  std::vector<uint16_t> step(ntask);
  for (size_t t = 0; t < ntask; ++t) {
    const int32_t *r = &g.tasks[t * 8];
    const int node = r[0], o = r[1] & 7;
    const int64_t gi = g.node_g[node];
    const int x = (int)(gi % GX) - 2, y = (int)((gi / GX) % g.GY) - 2, z = (int)(gi / GXY) - 2;
    const int a = x / TX, b = y / TY, c = z / TZ;
    const int sx = oct_sx(o), sy = oct_sy(o), sz = oct_sz(o);
    const int diag = (sx > 0 ? a : nTx - 1 - a) + (sy > 0 ? b : nTy - 1 - b) + (sz > 0 ? c : nTz - 1 - c);
    const int xhi = std::min((a + 1) * TX, Nx) - 1, yhi = std::min((b + 1) * TY, Ny) - 1,
              zhi = std::min((c + 1) * TZ, Nz) - 1;
    const int u = sx > 0 ? x - a * TX : xhi - x;
    const int v = sy > 0 ? y - b * TY : yhi - y;
    const int w = sz > 0 ? z - c * TZ : zhi - z;
    step[t] = (uint16_t)(u + v + w);
    dio[t] = diag * 8 + o;
    tile[t] = a + (int64_t)nTx * (b + (int64_t)nTy * c);
  }
  // stable counting sorts by step, then tile, then (diagonal, octant)
  std::vector<int64_t> order(ntask), tmp(ntask);
  std::iota(order.begin(), order.end(), (int64_t)0);
  auto counting_sort = [&](int64_t nb, auto keyf) {
    std::vector<int64_t> cnt((size_t)nb + 1, 0);
    for (size_t q = 0; q < ntask; ++q) cnt[(size_t)keyf(order[q]) + 1]++;
    for (int64_t k = 0; k < nb; ++k) cnt[(size_t)k + 1] += cnt[(size_t)k];
    for (size_t q = 0; q < ntask; ++q) tmp[(size_t)cnt[(size_t)keyf(order[q])]++] = order[q];
    order.swap(tmp);
  };
  counting_sort(tj.nsteps, [&](int64_t t) { return (int64_t)step[(size_t)t]; });
  counting_sort(ntiles, [&](int64_t t) { return tile[(size_t)t]; });
  counting_sort((int64_t)ndiag * 8, [&](int64_t t) { return (int64_t)dio[(size_t)t]; });
  tmp.clear(); tmp.shrink_to_fit();
  auto same_job = [&](int64_t a, int64_t b) { return dio[(size_t)a] == dio[(size_t)b] && tile[(size_t)a] == tile[(size_t)b]; };

  const int64_t nrows_h = ((int64_t)g.NF + g.NB) * 8;
  const int64_t nrows_all = nrows_h + (int64_t)g.nCorner * 8;
  std::vector<int32_t> stamp((size_t)nrows_all, -1), slot_of((size_t)nrows_all, 0);
  auto row_index = [&](int32_t code) -> int64_t {
    return (code & (1 << 30)) ? nrows_h + (code & ~(1 << 30)) : (int64_t)code;
  };
  tj.tasks.reserve(ntask * 4);
  tj.rows.reserve(ntask * 2);
  tj.diag_begin.assign((size_t)ndiag + 1, 0);
  tj.diag_rows.assign((size_t)ndiag, 0);
  tj.diag_tasks.assign((size_t)ndiag, 0);
  int32_t njobs = 0;
  std::vector<int64_t> job_tile;
  std::vector<int8_t> job_oct;
  size_t q = 0;
  while (q < ntask) {
    size_t e = q;
    while (e < ntask && same_job(order[e], order[q])) ++e;
    const int diag = dio[(size_t)order[q]] / 8;
    job_tile.push_back(tile[(size_t)order[q]]);
    job_oct.push_back((int8_t)(dio[(size_t)order[q]] % 8));
    const int64_t rb = (int64_t)tj.rows.size();
    tj.row_begin.push_back(rb);
    tj.task_begin.push_back((int64_t)(tj.tasks.size() / 4));
    for (size_t p = q; p < e; ++p) {  // own rows, in task order
      const int32_t *r = &g.tasks[(size_t)order[p] * 8];
      const int32_t own = r[0] * 8 + (r[1] & 7);
      stamp[(size_t)own] = njobs;
      slot_of[(size_t)own] = (int32_t)(1 + (p - q));
      tj.rows.push_back(own);
    }
    for (size_t p = q; p < e; ++p) {
      const int32_t *r = &g.tasks[(size_t)order[p] * 8];
      int32_t sl[6];
      for (int n = 0; n < 6; ++n) {
        const int32_t code = r[2 + n];
        if (code < 0) { sl[n] = 0; continue; }
        const int64_t idx = row_index(code);
        if (stamp[(size_t)idx] != njobs) {
          stamp[(size_t)idx] = njobs;
          slot_of[(size_t)idx] = (int32_t)(1 + ((int64_t)tj.rows.size() - rb));
          tj.rows.push_back(code);
        }
        sl[n] = slot_of[(size_t)idx];
      }
      const int fl = r[1];
      tj.tasks.push_back(r[0] | ((fl & 8) ? 1 << 27 : 0) | ((fl & 16) ? 1 << 28 : 0) | ((fl & 32) ? 1 << 29 : 0));
      tj.tasks.push_back(sl[0] | (sl[1] << 16));
      tj.tasks.push_back(sl[2] | (sl[3] << 16));
      tj.tasks.push_back(sl[4] | (sl[5] << 16));
    }
    const int32_t nslots = (int32_t)(1 + ((int64_t)tj.rows.size() - rb));
    if (nslots > max_slots) return false;
    tj.row_count.push_back(nslots - 1);
    while (tj.rows.size() % 4) tj.rows.push_back(0);
    tj.diag_rows[(size_t)diag] = std::max(tj.diag_rows[(size_t)diag], nslots);
    tj.diag_tasks[(size_t)diag] = std::max(tj.diag_tasks[(size_t)diag], (int32_t)(e - q));
    tj.max_rows = std::max(tj.max_rows, nslots);
    tj.max_tasks = std::max(tj.max_tasks, (int32_t)(e - q));
    // step offsets
    const size_t sb = tj.steps.size();
    tj.steps.resize(sb + (size_t)tj.steps_stride, 0);
    for (size_t p = q; p < e; ++p) tj.steps[sb + step[order[p]] + 1]++;
    for (int s = 0; s < tj.nsteps; ++s) tj.steps[sb + s + 1] = (uint16_t)(tj.steps[sb + s + 1] + tj.steps[sb + s]);
    tj.diag_begin[(size_t)diag + 1] = njobs + 1;
    ++njobs;
    q = e;
  }
  tj.row_begin.push_back((int64_t)tj.rows.size());
  tj.task_begin.push_back((int64_t)(tj.tasks.size() / 4));
  for (int d = 0; d < ndiag; ++d) tj.diag_begin[(size_t)d + 1] = std::max(tj.diag_begin[(size_t)d + 1], tj.diag_begin[(size_t)d]);
  // upstream jobs: the neighbour tiles on the upwind side of each axis, same octant
  std::vector<int32_t> job_of((size_t)ntiles * 8, -1);
  for (int32_t j = 0; j < njobs; ++j) job_of[(size_t)job_tile[(size_t)j] * 8 + job_oct[(size_t)j]] = j;
  tj.up.assign((size_t)njobs * 4, -1);
  for (int32_t j = 0; j < njobs; ++j) {
    const int64_t t = job_tile[(size_t)j];
    const int o = job_oct[(size_t)j];
    const int a = (int)(t % nTx), b = (int)((t / nTx) % nTy), c = (int)(t / ((int64_t)nTx * nTy));
    const int na = a - oct_sx(o), nb = b - oct_sy(o), nc = c - oct_sz(o);
    if (na >= 0 && na < nTx) tj.up[(size_t)j * 4 + 0] = job_of[(size_t)(na + (int64_t)nTx * (b + (int64_t)nTy * c)) * 8 + o];
    if (nb >= 0 && nb < nTy) tj.up[(size_t)j * 4 + 1] = job_of[(size_t)(a + (int64_t)nTx * (nb + (int64_t)nTy * c)) * 8 + o];
    if (nc >= 0 && nc < nTz) tj.up[(size_t)j * 4 + 2] = job_of[(size_t)(a + (int64_t)nTx * (b + (int64_t)nTy * nc)) * 8 + o];
  }
  plan_tile_launches(tj, 1, 0.0);
  return true;
}

void plan_tile_launches(TileJobs &tj, int max_classes, double ratio) {
  tj.job_list.clear();
  tj.launches.clear();
  tj.launch_diag_end.clear();
  const size_t ndiag = tj.diag_begin.empty() ? 0 : tj.diag_begin.size() - 1;
  std::vector<int32_t> jobs;
  for (size_t d = 0; d < ndiag; ++d) {
    jobs.clear();
    for (int32_t j = tj.diag_begin[d]; j < tj.diag_begin[d + 1]; ++j) jobs.push_back(j);
    std::stable_sort(jobs.begin(), jobs.end(),
                     [&](int32_t a, int32_t b) { return tj.row_count[(size_t)a] > tj.row_count[(size_t)b]; });
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
