// clusters.cpp -- liquid / gas cluster statistics of the reference's
// calc_cluster (src/multiphase_lbm.cu:225-562), computed without recursion.
//
// The reference labels clusters with a recursive depth-first search
// (:163-223), which needs an unlimited stack for large clusters.  Here each
// cluster is flooded with an explicit queue; cluster membership does not
// depend on the traversal order, and clusters are numbered in the order of
// their first node in the reference's x-major scan, so the labels, the
// removal of clusters smaller than 7 nodes, the cluster-to-solid sets, the
// cluster order, the wet coordination number and the single-cluster radius
// all come out as the reference computes them.  Quantities the reference
// keeps in float (`real`) are computed in float.
#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <vector>

#include "../../../include/mlbm_driver.h"
#include "../errors.h"

namespace {

// D3Q19 velocities, include/lbm_model.cuh:49-54
const int EX[19] = {0, -1, 0, 0, -1, -1, -1, -1, 0, 0, 1, 0, 0, 1, 1, 1, 1, 0, 0};
const int EY[19] = {0, 0, -1, 0, -1, 1, 0, 0, -1, -1, 0, 1, 0, 1, -1, 0, 0, 1, 1};
const int EZ[19] = {0, 0, 0, -1, 0, 0, -1, 1, -1, 1, 0, 0, 1, 0, 0, 1, -1, 1, -1};

struct Grid {
  int lx, ly, lz;
  long long idx(int x, int y, int z) const {
    return ((long long)x * ly + y) * lz + z;
  }
};

// Flood one cluster from (x,y,z): nodes with member[k] set join, get label
// `id` and are cleared from member; returns the cluster size.  When solids
// is given, the solid numbers (!= 0) of non-member 6-neighbours are added.
long long flood(const Grid& g, std::vector<uint8_t>& member, int64_t* labels,
                int64_t id, int x, int y, int z, const int64_t* solid_number,
                std::set<long long>* solids, std::vector<long long>& queue) {
  queue.clear();
  const long long k0 = g.idx(x, y, z);
  member[k0] = 0;
  labels[k0] = id;
  queue.push_back(k0);
  size_t head = 0;
  while (head < queue.size()) {
    const long long k = queue[head++];
    const int cx = (int)(k / ((long long)g.ly * g.lz));
    const int cy = (int)((k / g.lz) % g.ly);
    const int cz = (int)(k % g.lz);
    const int xp = cx > 0 ? cx - 1 : g.lx - 1, xn = cx < g.lx - 1 ? cx + 1 : 0;
    const int yp = cy > 0 ? cy - 1 : g.ly - 1, yn = cy < g.ly - 1 ? cy + 1 : 0;
    const int zp = cz > 0 ? cz - 1 : g.lz - 1, zn = cz < g.lz - 1 ? cz + 1 : 0;
    const long long nb[6] = {g.idx(xp, cy, cz), g.idx(cx, yp, cz),
                             g.idx(cx, cy, zp), g.idx(xn, cy, cz),
                             g.idx(cx, yn, cz), g.idx(cx, cy, zn)};
    for (long long q : nb) {
      if (member[q]) {
        member[q] = 0;
        labels[q] = id;
        queue.push_back(q);
      } else if (solids && solid_number && solid_number[q] != 0) {
        solids->insert(solid_number[q]);
      }
    }
  }
  return (long long)queue.size();
}

void unlabel(const std::vector<long long>& nodes, int64_t* labels) {
  for (long long k : nodes) labels[k] = 0;
}

}  // namespace

extern "C" mlbm_status mlbm_cluster_stats(
    const float* rho, const uint8_t* is_fluid, const int64_t* solid_number,
    int32_t lx, int32_t ly, int32_t lz, float rhol, float rhog,
    int64_t solid_count, int64_t* liq_labels_out, int64_t* gas_labels_out,
    mlbm_stats_row* out) {
  if (!rho || !is_fluid || !out || lx < 1 || ly < 1 || lz < 1)
    return mlbm::set_error(MLBM_ERR_ARG, "cluster_stats: bad arguments");
  const Grid g{lx, ly, lz};
  const long long n = (long long)lx * ly * lz;
  std::vector<uint8_t> liq(n, 0), gas(n, 0);
  long long liquid_count = 0;
  for (long long k = 0; k < n; ++k) {
    if (!is_fluid[k]) continue;
    if (rho[k] > rhol) {
      liq[k] = 1;
      ++liquid_count;
    } else if (rho[k] < rhog) {
      gas[k] = 1;
    }
  }

  // liquid-solid / liquid-vapour boundary nodes (:278-316)
  long long n_ls = 0, n_lv = 0;
  for (int x = 0; x < lx; ++x)
    for (int y = 0; y < ly; ++y)
      for (int z = 0; z < lz; ++z) {
        if (!liq[g.idx(x, y, z)]) continue;
        for (int i = 1; i < 19; ++i) {
          const int nx = (x - EX[i] + lx) % lx, ny = (y - EY[i] + ly) % ly,
                    nz = (z - EZ[i] + lz) % lz;
          const long long q = g.idx(nx, ny, nz);
          if (!is_fluid[q]) { ++n_ls; break; }
          if (rho[q] < rhol) { ++n_lv; break; }
        }
      }
  if (liquid_count > 0) {
    out->liquid_solid_boundary = (float)((double)n_ls / liquid_count);
    out->liquid_vapor_boundary = (float)((double)n_lv / liquid_count);
  }

  std::vector<int64_t> liq_lab_local, gas_lab_local;
  int64_t* liq_lab = liq_labels_out;
  int64_t* gas_lab = gas_labels_out;
  if (!liq_lab) { liq_lab_local.assign(n, 0); liq_lab = liq_lab_local.data(); }
  else std::memset(liq_lab, 0, n * sizeof(int64_t));
  if (!gas_lab) { gas_lab_local.assign(n, 0); gas_lab = gas_lab_local.data(); }
  else std::memset(gas_lab, 0, n * sizeof(int64_t));

  const long long kMinCluster = 7;  // :321
  std::vector<long long> queue;
  queue.reserve(1024);
  std::map<long long, std::set<long long>> cluster_to_solids;
  long long liq_count = 0;
  for (int x = 0; x < lx; ++x)
    for (int y = 0; y < ly; ++y)
      for (int z = 0; z < lz; ++z) {
        if (!liq[g.idx(x, y, z)]) continue;
        ++liq_count;
        std::set<long long> solids;
        const long long size = flood(g, liq, liq_lab, liq_count, x, y, z,
                                     solid_number, &solids, queue);
        if (size < kMinCluster) {
          unlabel(queue, liq_lab);
          --liq_count;
        } else if (!solids.empty()) {
          cluster_to_solids[liq_count] = std::move(solids);
        }
      }
  long long gas_count = 0;
  for (int x = 0; x < lx; ++x)
    for (int y = 0; y < ly; ++y)
      for (int z = 0; z < lz; ++z) {
        if (!gas[g.idx(x, y, z)]) continue;
        ++gas_count;
        const long long size =
            flood(g, gas, gas_lab, gas_count, x, y, z, nullptr, nullptr, queue);
        if (size < kMinCluster) {
          unlabel(queue, gas_lab);
          --gas_count;
        }
      }
  out->liq_cluster_count = liq_count;
  out->gas_cluster_count = gas_count;

  // single liquid cluster: centre and radius with periodic unwrapping
  // (:362-533)
  float max_r = 0.f;
  if (liq_count == 1) {
    auto lab = [&](int x, int y, int z) { return liq_lab[g.idx(x, y, z)]; };
    bool xb = false, yb = false, zb = false;
    for (int y = 0; y < ly && !xb; ++y)
      for (int z = 0; z < lz; ++z)
        if (lab(0, y, z) == 1 && lab(lx - 1, y, z) == 1) { xb = true; break; }
    for (int x = 0; x < lx && !yb; ++x)
      for (int z = 0; z < lz; ++z)
        if (lab(x, 0, z) == 1 && lab(x, ly - 1, z) == 1) { yb = true; break; }
    for (int x = 0; x < lx && !zb; ++x)
      for (int y = 0; y < ly; ++y)
        if (lab(x, y, 0) == 1 && lab(x, y, lz - 1) == 1) { zb = true; break; }
    long long xv = 0, yv = 0, zv = 0;  // first plane free of the cluster
    if (xb)
      for (int x = 0; x < lx; ++x) {
        bool free = true;
        for (int y = 0; y < ly && free; ++y)
          for (int z = 0; z < lz; ++z)
            if (lab(x, y, z) == 1) { free = false; break; }
        if (free) { xv = x; break; }
      }
    if (yb)
      for (int y = 0; y < ly; ++y) {
        bool free = true;
        for (int z = 0; z < lz && free; ++z)
          for (int x = 0; x < lx; ++x)
            if (lab(x, y, z) == 1) { free = false; break; }
        if (free) { yv = y; break; }
      }
    if (zb)
      for (int z = 0; z < lz; ++z) {
        bool free = true;
        for (int x = 0; x < lx && free; ++x)
          for (int y = 0; y < ly; ++y)
            if (lab(x, y, z) == 1) { free = false; break; }
        if (free) { zv = z; break; }
      }
    unsigned long long sx = 0, sy = 0, sz = 0, size = 0;
    for (int x = 0; x < lx; ++x)
      for (int y = 0; y < ly; ++y)
        for (int z = 0; z < lz; ++z)
          if (lab(x, y, z) == 1) {
            sx += (xb && x < xv) ? x + lx : x;
            sy += (yb && y < yv) ? y + ly : y;
            sz += (zb && z < zv) ? z + lz : z;
            ++size;
          }
    // integer division, as the reference (:496-498)
    const float xc = (float)(sx / size), yc = (float)(sy / size),
                zc = (float)(sz / size);
    for (int x = 0; x < lx; ++x)
      for (int y = 0; y < ly; ++y)
        for (int z = 0; z < lz; ++z)
          if (lab(x, y, z) == 1) {
            const float ax = (float)((xb && x < xv) ? x + lx : x);
            const float ay = (float)((yb && y < yv) ? y + ly : y);
            const float az = (float)((zb && z < zv) ? z + lz : z);
            const float dxx = (xc - ax) * (xc - ax);
            const float dyy = (yc - ay) * (yc - ay);
            const float dzz = (zc - az) * (zc - az);
            const float r2 = (dxx + dyy) + dzz;
            const float r = (float)std::sqrt((double)r2);
            if (r > max_r) max_r = r;
          }
  }
  out->cluster_radius = max_r;

  // cluster order and wet coordination number (:535-561)
  float order = 0.f;
  for (const auto& kv : cluster_to_solids) order += (float)kv.second.size();
  if (liq_count != 0) order /= (float)cluster_to_solids.size();
  out->cluster_order = order;
  std::map<long long, std::set<long long>> solid_to_clusters;
  for (const auto& kv : cluster_to_solids)
    for (long long s : kv.second) solid_to_clusters[s].insert(kv.first);
  float wet = 0.f;
  for (const auto& kv : solid_to_clusters) wet += (float)kv.second.size();
  if (solid_count != 0) wet /= (float)solid_count;
  out->wet_coord_num = wet;
  return MLBM_OK;
}
