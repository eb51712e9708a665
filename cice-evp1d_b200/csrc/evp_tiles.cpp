// evp_tiles.cpp -- tile plan of the fused solver.
//
// Step 1: grid coordinates.  Either given (2D entry points) or rebuilt from
//   the neighbour vectors by a breadth-first walk: ee = (i-1,j),
//   ne = (i-1,j-1), se = (i,j-1), nw = (i+1,j), sw = (i+1,j+1),
//   sse = (i,j+1) (integration/ice_dyn_evp1d.F90:766-772).  Each connected
//   piece of the list gets its own origin.  A graph that contradicts itself
//   (two coordinates for one point, or two points on one coordinate) has no
//   grid layout, and the plan then tiles consecutive list points instead.
// Step 2: tiles.  Points are grouped by (piece, j / kTileH, i / kTileW), tiles
//   ordered row by row, points row by row inside a tile.
// Step 3: forward halo.  A tile whose halo would exceed kTileHalo points is
//   split in halves until it fits (possible only for irregular graphs).
#include "evp_tiles.h"

#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

namespace evp {

namespace {

const int kDI[6] = {-1, -1, 0, +1, +1, 0};  // ee ne se nw sw sse
const int kDJ[6] = {0, -1, -1, 0, +1, +1};

inline int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// Position of (x, y) along the Hilbert curve filling the n x n square (n a
// power of two), by the standard rotate-and-reflect walk over the quadrant
// bits (the published xy-to-d conversion).
uint64_t hilbert_index(uint32_t n, uint32_t x, uint32_t y) {
  uint64_t d = 0;
  for (uint32_t s = n / 2; s > 0; s /= 2) {
    const uint32_t rx = (x & s) ? 1u : 0u, ry = (y & s) ? 1u : 0u;
    d += (uint64_t)s * (uint64_t)s * ((3u * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = s - 1 - x;
        y = s - 1 - y;
      }
      const uint32_t t = x;
      x = y;
      y = t;
    }
  }
  return d;
}

bool reconstruct_coords(int na, const int32_t *const nb0[6],
                        std::vector<int32_t> &ci, std::vector<int32_t> &cj,
                        std::vector<int32_t> &comp) {
  ci.assign((size_t)na, 0);
  cj.assign((size_t)na, 0);
  comp.assign((size_t)na, -1);
  std::vector<int32_t> queue;
  queue.reserve((size_t)na);
  int ncomp = 0;
  for (int p0 = 0; p0 < na; p0++) {
    if (comp[p0] >= 0) continue;
    comp[p0] = ncomp;
    queue.clear();
    queue.push_back(p0);
    for (size_t h = 0; h < queue.size(); h++) {
      const int q = queue[h];
      for (int r = 0; r < 6; r++) {
        const int n = nb0[r][q];
        if (n < 0 || n >= na) continue;  // a halo slot, not a list point
        const long long ei = (long long)ci[q] + kDI[r], ej = (long long)cj[q] + kDJ[r];
        if (ei < INT_MIN / 2 || ei > INT_MAX / 2 || ej < INT_MIN / 2 || ej > INT_MAX / 2)
          return false;
        if (comp[n] < 0) {
          comp[n] = ncomp;
          ci[n] = (int32_t)ei;
          cj[n] = (int32_t)ej;
          queue.push_back(n);
        } else if (comp[n] != ncomp || ci[n] != ei || cj[n] != ej) {
          return false;
        }
      }
    }
    ncomp++;
  }
  // two points on one coordinate of one piece: no grid layout
  std::vector<int32_t> order((size_t)na);
  for (int p = 0; p < na; p++) order[p] = p;
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    if (comp[a] != comp[b]) return comp[a] < comp[b];
    if (cj[a] != cj[b]) return cj[a] < cj[b];
    return ci[a] < ci[b];
  });
  for (int k = 1; k < na; k++) {
    const int a = order[k - 1], b = order[k];
    if (comp[a] == comp[b] && ci[a] == ci[b] && cj[a] == cj[b]) return false;
  }
  return true;
}

}  // namespace

void build_tile_plan(int na, int navel, const int32_t *const nb0[6],
                     const int32_t *coords_i, const int32_t *coords_j,
                     TilePlan *plan, int max_tile) {
  const int tmax = max_tile < 1 ? 1 : (max_tile > kTileOwned ? kTileOwned : max_tile);
  TilePlan &P = *plan;
  P = TilePlan();
  P.na = na;
  P.navel = navel;
  P.nhalo_slots = navel - na;
  if (na == 0) return;

  // ---- step 1 + 2: candidate groups --------------------------------------
  std::vector<std::vector<int32_t>> groups;
  std::vector<int32_t> ci, cj, comp;
  bool have = false;
  if (coords_i && coords_j) {
    ci.assign(coords_i, coords_i + na);
    cj.assign(coords_j, coords_j + na);
    comp.assign((size_t)na, 0);
    have = true;
  } else {
    have = reconstruct_coords(na, nb0, ci, cj, comp);
  }
  P.from_coords = have;
  if (have) {
    // origin of each piece at its bounding-box corner, so that the tiles do
    // not depend on where the walk started (i.e. on the list order)
    int nc = 0;
    for (int p = 0; p < na; p++) nc = comp[p] + 1 > nc ? comp[p] + 1 : nc;
    std::vector<int32_t> mi((size_t)nc, INT_MAX), mj((size_t)nc, INT_MAX);
    for (int p = 0; p < na; p++) {
      mi[comp[p]] = ci[p] < mi[comp[p]] ? ci[p] : mi[comp[p]];
      mj[comp[p]] = cj[p] < mj[comp[p]] ? cj[p] : mj[comp[p]];
    }
    for (int p = 0; p < na; p++) {
      ci[p] -= mi[comp[p]];
      cj[p] -= mj[comp[p]];
    }
    // pieces in a canonical order (by their position in the grid walk's
    // coordinates is not canonical, so by size and extent), points of a piece
    // along a Hilbert curve over its coordinates, then consecutive runs of
    // tmax points: compact, full tiles.  A run may span two pieces;
    // pieces never share neighbours, so that only merges small floes.
    std::vector<int32_t> pn((size_t)nc, 0), pw((size_t)nc, 0), ph((size_t)nc, 0);
    for (int p = 0; p < na; p++) {
      pn[comp[p]]++;
      pw[comp[p]] = ci[p] + 1 > pw[comp[p]] ? ci[p] + 1 : pw[comp[p]];
      ph[comp[p]] = cj[p] + 1 > ph[comp[p]] ? cj[p] + 1 : ph[comp[p]];
    }
    std::vector<uint64_t> hkey((size_t)na);
    for (int p = 0; p < na; p++) {
      uint32_t n = 1;
      const int32_t ext = pw[comp[p]] > ph[comp[p]] ? pw[comp[p]] : ph[comp[p]];
      while ((int64_t)n < ext) n *= 2;
      hkey[p] = hilbert_index(n, (uint32_t)ci[p], (uint32_t)cj[p]);
    }
    // canonical piece order: larger first, then by extent and the first
    // point's Hilbert position -- none of which depends on the list order
    std::vector<uint64_t> pfirst((size_t)nc, UINT64_MAX);
    for (int p = 0; p < na; p++) pfirst[comp[p]] = hkey[p] < pfirst[comp[p]] ? hkey[p] : pfirst[comp[p]];
    std::vector<int32_t> order((size_t)na);
    for (int p = 0; p < na; p++) order[p] = p;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
      const int A = comp[a], B = comp[b];
      if (A != B) {
        if (pn[A] != pn[B]) return pn[A] > pn[B];
        if (pw[A] != pw[B]) return pw[A] < pw[B];
        if (ph[A] != ph[B]) return ph[A] < ph[B];
        if (pfirst[A] != pfirst[B]) return pfirst[A] < pfirst[B];
        return A < B;
      }
      return hkey[a] < hkey[b];
    });
    // each tile takes the longest run (up to tmax points) whose halo
    // and velocity extras fit, found by bisection on the run length
    std::vector<int32_t> m1((size_t)navel, -1), m2((size_t)navel, -1), m3((size_t)navel, -1);
    int st = 0;
    auto fits = [&](int k, int len) {
      st++;
      for (int q = k; q < k + len; q++) m1[order[q]] = st;
      int nh = 0, nx = 0;
      std::vector<int32_t> hl;
      for (int q = k; q < k + len; q++)
        for (int r = 3; r < 6; r++) {
          const int n = nb0[r][order[q]];
          if (n < na && m1[n] != st && m2[n] != st) {
            m2[n] = st;
            hl.push_back(n);
            if (++nh > kTileHalo) return false;
          }
        }
      auto add_x = [&](int n) {
        if (m1[n] != st && m3[n] != st) {
          m3[n] = st;
          nx++;
        }
      };
      for (int n : hl) add_x(n);
      for (int q = k; q < k + len; q++)
        for (int r = 0; r < 3; r++) add_x(nb0[r][order[q]]);
      for (int n : hl)
        for (int r = 0; r < 3; r++) add_x(nb0[r][n]);
      return nx <= kTileUvx;
    };
    for (int k = 0; k < na;) {
      int len = tmax < na - k ? tmax : na - k;
      if (!fits(k, len)) {
        int lo = 1, hi = len - 1;  // fits(k, 1) holds: a point reaches 3 + 6 + 9 others
        while (lo < hi) {
          const int mid = (lo + hi + 1) / 2;
          if (fits(k, mid)) lo = mid; else hi = mid - 1;
        }
        len = lo;
      }
      groups.emplace_back(order.begin() + k, order.begin() + k + len);
      k += len;
    }
  } else {
    for (int k = 0; k < na; k += tmax) {
      std::vector<int32_t> g;
      for (int p = k; p < na && p < k + tmax; p++) g.push_back(p);
      groups.push_back(std::move(g));
    }
  }

  // ---- step 3: split groups whose halo or velocity set is too large ------
  // halo H = list points outside the group reached through nw/sw/sse;
  // extras X = ({H} + ee/ne/se of group and H) minus the group, where the
  // reference's halo slots (>= na) count as points too.
  std::vector<int32_t> mark((size_t)navel, -1), hmark((size_t)navel, -1),
      xmark((size_t)navel, -1);
  int stamp = 0;
  std::vector<std::vector<int32_t>> tiles;
  std::vector<std::vector<int32_t>> stack;
  std::vector<int32_t> hl;
  for (auto &g0 : groups) {
    stack.push_back(std::move(g0));
    while (!stack.empty()) {
      std::vector<int32_t> g = std::move(stack.back());
      stack.pop_back();
      stamp++;
      for (int p : g) mark[p] = stamp;
      int nh = 0, nx = 0;
      hl.clear();
      for (int p : g)
        for (int r = 3; r < 6; r++) {
          const int n = nb0[r][p];
          if (n < na && mark[n] != stamp && hmark[n] != stamp) {
            hmark[n] = stamp;
            hl.push_back(n);
            nh++;
          }
        }
      auto add_x = [&](int n) {
        if (mark[n] != stamp && xmark[n] != stamp) {
          xmark[n] = stamp;
          nx++;
        }
      };
      for (int q : hl) add_x(q);
      for (int p : g)
        for (int r = 0; r < 3; r++) add_x(nb0[r][p]);
      for (int q : hl)
        for (int r = 0; r < 3; r++) add_x(nb0[r][q]);
      if ((int)g.size() <= tmax && nh <= kTileHalo && nx <= kTileUvx) {
        tiles.push_back(std::move(g));
      } else {
        const size_t half = g.size() / 2;
        std::vector<int32_t> a(g.begin(), g.begin() + half), b(g.begin() + half, g.end());
        stack.push_back(std::move(b));
        stack.push_back(std::move(a));
      }
    }
  }

  // ---- slots ---------------------------------------------------------------
  P.ntiles = (int)tiles.size();
  P.tile_off.resize(P.ntiles);
  P.tile_cnt.resize(P.ntiles);
  P.slot_of_point.assign((size_t)na, -1);
  std::vector<int32_t> tile_of((size_t)na, -1);
  int off = 0;
  for (int t = 0; t < P.ntiles; t++) {
    P.tile_off[t] = off;
    P.tile_cnt[t] = (int)tiles[t].size();
    for (size_t k = 0; k < tiles[t].size(); k++) {
      P.slot_of_point[tiles[t][k]] = off + (int)k;
      tile_of[tiles[t][k]] = t;
    }
    off += ((int)tiles[t].size() + kSlotAlign - 1) / kSlotAlign * kSlotAlign;
  }
  P.nslots = off;
  P.point_of_slot.assign((size_t)P.nslots, -1);
  for (int p = 0; p < na; p++) P.point_of_slot[P.slot_of_point[p]] = p;

  // ---- neighbour slots -------------------------------------------------------
  auto to_slot = [&](int n) { return n < na ? P.slot_of_point[n] : P.nslots + (n - na); };
  std::vector<int32_t> *arr[6] = {&P.ee, &P.ne, &P.se, &P.nw, &P.sw, &P.sse};
  for (int r = 0; r < 6; r++) {
    arr[r]->resize((size_t)P.nslots);
    for (int s = 0; s < P.nslots; s++) {
      const int p = P.point_of_slot[s];
      (*arr[r])[s] = p < 0 ? s : to_slot(nb0[r][p]);
    }
  }

  // ---- halo lists, velocity extras and packed local indices -----------------
  const uint32_t zero3 = (uint32_t)kZeroSlot | ((uint32_t)kZeroSlot << kLnbBits) |
                         ((uint32_t)kZeroSlot << (2 * kLnbBits));
  P.lnb.assign((size_t)P.nslots, zero3);
  P.lcor.assign((size_t)P.nslots, 0);
  P.halo_off.resize(P.ntiles);
  P.halo_cnt.resize(P.ntiles);
  P.uvx_off.resize(P.ntiles);
  P.uvx_cnt.resize(P.ntiles);
  // hpos/htile: forward-halo position of a list point in the current tile;
  // xpos/xtile: velocity-extra position of any u/v point (list or halo slot)
  std::vector<int32_t> hpos((size_t)na, -1), htile((size_t)na, -1);
  std::vector<int32_t> xpos((size_t)navel, -1), xtile((size_t)navel, -1);
  for (int t = 0; t < P.ntiles; t++) {
    P.halo_off[t] = (int)P.halo_idx.size();
    P.uvx_off[t] = (int)P.uvx_idx.size();
    int nh = 0, nx = 0;
    const int own = P.tile_cnt[t];
    std::vector<int32_t> &members = tiles[t];
    // stepu's str neighbours and the forward halo
    for (int k = 0; k < own; k++) {
      const int p = members[k];
      uint32_t packed = 0;
      for (int r = 3; r < 6; r++) {
        const int n = nb0[r][p];
        uint32_t loc;
        if (n >= na) {
          loc = kZeroSlot;
        } else if (tile_of[n] == t) {
          loc = (uint32_t)(P.slot_of_point[n] - P.tile_off[t]);
        } else {
          if (htile[n] != t) {  // first time this tile reaches n
            htile[n] = t;
            hpos[n] = nh++;
            P.halo_idx.push_back(P.slot_of_point[n]);
          }
          loc = (uint32_t)(kTileOwned + hpos[n]);
        }
        packed |= loc << ((r - 3) * kLnbBits);
      }
      P.lnb[P.slot_of_point[p]] = packed;
    }
    // velocity index of any u/v point n (list point or reference halo slot)
    auto uv_local = [&](int n) -> uint32_t {
      if (n < na && tile_of[n] == t) return (uint32_t)(P.slot_of_point[n] - P.tile_off[t]);
      if (xtile[n] != t) {
        xtile[n] = t;
        xpos[n] = nx++;
        P.uvx_idx.push_back(to_slot(n));
      }
      return (uint32_t)(kTileOwned + xpos[n]);
    };
    for (int k = 0; k < own; k++) {
      const int p = members[k];
      uint32_t packed = 0;
      for (int r = 0; r < 3; r++) packed |= uv_local(nb0[r][p]) << (r * kLnbBits);
      P.lcor[P.slot_of_point[p]] = packed;
    }
    for (int h = 0; h < nh; h++) {
      const int q = P.point_of_slot[P.halo_idx[P.halo_off[t] + h]];
      P.halo_lcc.push_back(uv_local(q));
      uint32_t packed = 0;
      for (int r = 0; r < 3; r++) packed |= uv_local(nb0[r][q]) << (r * kLnbBits);
      P.halo_lcor.push_back(packed);
    }
    P.halo_cnt[t] = nh;
    P.uvx_cnt[t] = nx;
  }
}

}  // namespace evp
