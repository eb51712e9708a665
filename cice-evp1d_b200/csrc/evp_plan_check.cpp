// evp_plan_check.cpp -- host-side verification of a tile plan.
//
// The kernels gather through indices that the planner derives from the
// neighbour vectors: slot positions, runs of tiles, forward-halo lists,
// velocity extras and 10-bit local indices packed three to a word (a str
// index may point into the previous tile of the same run).  A wrong one would read the
// wrong point (or outside a shared-memory array) without any fault to show
// it.  This check decodes every such index and compares it with what the
// neighbour vectors say it must be, so a plan is known good before any
// device code uses it: the host-side counterpart of a bounds checker (no
// sanitizer runs on the GPU here).
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "evp_tiles.h"

namespace evp {

namespace {

void note(long long &bad, std::string *first, const char *fmt, ...) {
  if (bad++ == 0 && first) {
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    *first = buf;
  }
}

uint32_t field(uint32_t w, int r) { return (w >> (r * kLnbBits)) & kLnbMask; }

}  // namespace

long long verify_tile_plan(const TilePlan &P, const int32_t *const nb0[6], int max_tile,
                           std::string *first) {
  long long bad = 0;
  const int na = P.na, navel = P.navel, S = P.nslots, T = P.ntiles;
  const int nuv = S + P.nhalo_slots;
  const size_t nh_all = P.halo_idx.size(), nx_all = P.uvx_idx.size();
  const std::vector<int32_t> *nbs[6] = {&P.ee, &P.ne, &P.se, &P.nw, &P.sw, &P.sse};

  // sizes first: the checks below index by them
  if (na < 0 || navel < na || S < na || T < 0 || P.nhalo_slots != navel - na)
    note(bad, first, "sizes: na %d navel %d nslots %d ntiles %d halo slots %d", na, navel, S, T,
         P.nhalo_slots);
  if (P.slot_of_point.size() != (size_t)na || P.point_of_slot.size() != (size_t)S)
    note(bad, first, "slot maps have %zu and %zu entries", P.slot_of_point.size(),
         P.point_of_slot.size());
  for (const auto *v : {&P.tile_off, &P.tile_cnt, &P.halo_off, &P.halo_cnt, &P.uvx_off, &P.uvx_cnt})
    if (v->size() != (size_t)T) note(bad, first, "a per-tile array has %zu entries", v->size());
  if (P.nruns < 0 || P.run_off.size() != (size_t)P.nruns + 1)
    note(bad, first, "%d runs with %zu run offsets", P.nruns, P.run_off.size());
  for (int r = 0; r < 6; r++)
    if (nbs[r]->size() != (size_t)S) note(bad, first, "neighbour slots %d: %zu entries", r, nbs[r]->size());
  if (P.lnb.size() != (size_t)S || P.lcor.size() != (size_t)S)
    note(bad, first, "packed index arrays have %zu and %zu entries", P.lnb.size(), P.lcor.size());
  if (P.halo_lcc.size() != nh_all || P.halo_lcor.size() != nh_all)
    note(bad, first, "halo index arrays do not match the halo list");
  for (int r = 0; r < 6 && bad == 0; r++)
    for (int p = 0; p < na; p++)
      if (nb0[r][p] < 0 || nb0[r][p] >= navel) {
        note(bad, first, "input neighbour %d of point %d is %d", r, p, nb0[r][p]);
        break;
      }
  if (bad) return bad;

  // slot <-> point
  int listed = 0;
  for (int s = 0; s < S; s++) {
    const int p = P.point_of_slot[s];
    if (p < -1 || p >= na) note(bad, first, "slot %d holds point %d", s, p);
    if (p >= 0) listed++;
  }
  if (listed != na) note(bad, first, "%d slots hold points, %d points listed", listed, na);
  for (int p = 0; p < na; p++) {
    const int s = P.slot_of_point[p];
    if (s < 0 || s >= S || P.point_of_slot[s] != p)
      note(bad, first, "point %d: slot %d does not hold it", p, s);
  }
  if (bad) return bad;

  // tiles: aligned, disjoint, increasing, full of points; every point in one
  std::vector<int32_t> tile_of((size_t)S, -1);
  std::vector<char> tile_ok((size_t)T, 0);
  int end = 0;
  for (int t = 0; t < T; t++) {
    const int off = P.tile_off[t], cnt = P.tile_cnt[t];
    if (off % kSlotAlign) note(bad, first, "tile %d starts at slot %d (not aligned)", t, off);
    if (cnt < 1 || cnt > max_tile || cnt > kTileOwned)
      note(bad, first, "tile %d holds %d points (limit %d)", t, cnt, max_tile);
    if (off < end || cnt < 1 || off + cnt > S) {
      note(bad, first, "tile %d range [%d, %d) overlaps or leaves the slots", t, off, off + cnt);
      continue;
    }
    for (int s = off; s < off + cnt; s++) {
      if (P.point_of_slot[s] < 0) note(bad, first, "tile %d slot %d is padding", t, s);
      tile_of[s] = t;
    }
    end = off + cnt;
    tile_ok[t] = 1;
  }
  for (int s = 0; s < S; s++)
    if (tile_of[s] < 0 && P.point_of_slot[s] >= 0)
      note(bad, first, "point %d (slot %d) is in no tile", P.point_of_slot[s], s);
  // runs: consecutive non-empty tile ranges that cover every tile once
  std::vector<char> first_of_run((size_t)T, 0);
  if (P.run_off.front() != 0 || P.run_off.back() != T)
    note(bad, first, "runs cover tiles [%d, %d), not [0, %d)", P.run_off.front(), P.run_off.back(),
         T);
  for (int r = 0; r < P.nruns; r++) {
    if (P.run_off[r + 1] <= P.run_off[r]) {
      note(bad, first, "run %d is [%d, %d)", r, P.run_off[r], P.run_off[r + 1]);
      continue;
    }
    if (P.run_off[r] >= 0 && P.run_off[r] < T) first_of_run[P.run_off[r]] = 1;
  }
  if (bad) return bad;

  auto to_slot = [&](int n) { return n < na ? P.slot_of_point[n] : S + (n - na); };

  // neighbour slots (padding slots point at themselves)
  for (int s = 0; s < S; s++) {
    const int p = P.point_of_slot[s];
    for (int r = 0; r < 6; r++) {
      const int want = p < 0 ? s : to_slot(nb0[r][p]);
      if ((*nbs[r])[s] != want)
        note(bad, first, "slot %d neighbour %d is %d, not %d", s, r, (*nbs[r])[s], want);
    }
  }

  // per tile: forward halo, velocity extras and every packed local index.
  // ppos: str-table position of a slot in the previous tile's compute set
  // (owned: slot offset; halo h: that tile's count + h), -1 elsewhere.
  std::vector<int32_t> hpos((size_t)S, -1), xpos((size_t)nuv, -1);
  std::vector<int32_t> ppos((size_t)S, -1), pslots;
  std::vector<char> hused((size_t)kTileHalo), xused((size_t)kTileUvx);
  for (int t = 0; t < T; t++) {
    if (!tile_ok[t]) continue;
    const int off = P.tile_off[t], cnt = P.tile_cnt[t];
    const int ho = P.halo_off[t], hc = P.halo_cnt[t], xo = P.uvx_off[t], xc = P.uvx_cnt[t];
    // the previous tile's table is alive only inside a run
    if (first_of_run[t]) {
      for (int sl : pslots) ppos[sl] = -1;
      pslots.clear();
    }
    if (hc < 0 || hc > kTileHalo || ho < 0 || (size_t)ho + hc > nh_all) {
      note(bad, first, "tile %d halo list [%d, +%d) is out of bounds", t, ho, hc);
      continue;
    }
    if (cnt + hc > max_tile || cnt + hc > kTileCompute)
      note(bad, first, "tile %d computes %d + %d points (limit %d)", t, cnt, hc, max_tile);
    if (xc < 0 || xc > kTileUvx || xo < 0 || (size_t)xo + xc > nx_all) {
      note(bad, first, "tile %d extra list [%d, +%d) is out of bounds", t, xo, xc);
      continue;
    }
    for (int h = 0; h < hc; h++) {
      const int s = P.halo_idx[ho + h];
      if (s < 0 || s >= S || P.point_of_slot[s] < 0)
        note(bad, first, "tile %d halo %d: slot %d is no list point", t, h, s);
      else if (tile_of[s] == t)
        note(bad, first, "tile %d halo %d: slot %d is the tile's own", t, h, s);
      else if (ppos[s] >= 0)
        note(bad, first, "tile %d halo %d: slot %d is in the previous tile's table", t, h, s);
      else if (hpos[s] >= 0)
        note(bad, first, "tile %d halo repeats slot %d", t, s);
      else
        hpos[s] = h;
    }
    for (int x = 0; x < xc; x++) {
      const int s = P.uvx_idx[xo + x];
      if (s < 0 || s >= nuv)
        note(bad, first, "tile %d extra %d: slot %d is outside u/v", t, x, s);
      else if (s < S && tile_of[s] == t)
        note(bad, first, "tile %d extra %d: slot %d is the tile's own", t, x, s);
      else if (xpos[s] >= 0)
        note(bad, first, "tile %d extras repeat slot %d", t, s);
      else
        xpos[s] = x;
    }
    std::fill(hused.begin(), hused.end(), 0);
    std::fill(xused.begin(), xused.end(), 0);
    // velocity index of point n (list point or halo slot) in this tile
    auto uv_want = [&](int n) -> int {
      const int sl = to_slot(n);
      if (n < na && tile_of[sl] == t) return sl - off;
      if (xpos[sl] < 0) return -1;
      xused[xpos[sl]] = 1;
      return kTileOwned + xpos[sl];
    };
    for (int s = off; s < off + cnt; s++) {
      const int p = P.point_of_slot[s];
      for (int r = 0; r < 3; r++) {  // stepu's str: nw, sw, sse
        const int n = nb0[3 + r][p];
        int want;
        if (n >= na) {
          want = kZeroSlot;
        } else {
          const int sl = P.slot_of_point[n];
          if (tile_of[sl] == t) {
            want = sl - off;
          } else if (ppos[sl] >= 0) {
            want = (int)kStrPrev | ppos[sl];
          } else if (hpos[sl] >= 0) {
            want = cnt + hpos[sl];
            hused[hpos[sl]] = 1;
          } else {
            want = -1;
          }
        }
        const int got = (int)field(P.lnb[s], r);
        if (want < 0 || got != want)
          note(bad, first, "tile %d point %d: str neighbour %d at %d, want %d", t, p, 3 + r, got,
               want);
      }
      for (int r = 0; r < 3; r++) {  // stress's corner velocities: ee, ne, se
        const int want = uv_want(nb0[r][p]);
        const int got = (int)field(P.lcor[s], r);
        if (want < 0 || got != want)
          note(bad, first, "tile %d point %d: velocity neighbour %d at %d, want %d", t, p, r, got,
               want);
      }
    }
    for (int h = 0; h < hc; h++) {
      const int s = P.halo_idx[ho + h];
      if (s < 0 || s >= S || P.point_of_slot[s] < 0) continue;
      const int q = P.point_of_slot[s];
      const int want_c = uv_want(q);
      if (want_c < 0 || (int)P.halo_lcc[ho + h] != want_c)
        note(bad, first, "tile %d halo point %d: own velocity at %u, want %d", t, q,
             P.halo_lcc[ho + h], want_c);
      for (int r = 0; r < 3; r++) {
        const int want = uv_want(nb0[r][q]);
        const int got = (int)field(P.halo_lcor[ho + h], r);
        if (want < 0 || got != want)
          note(bad, first, "tile %d halo point %d: velocity neighbour %d at %d, want %d", t, q, r,
               got, want);
      }
      if (!hused[h]) note(bad, first, "tile %d halo point %d is reached by no owned point", t, q);
    }
    for (int x = 0; x < xc; x++)
      if (!xused[x]) note(bad, first, "tile %d extra %d is read by no point", t, x);
    // this tile's compute set becomes the previous table
    for (int sl : pslots) ppos[sl] = -1;
    pslots.clear();
    for (int s = off; s < off + cnt; s++) {
      ppos[s] = s - off;
      pslots.push_back(s);
    }
    for (int h = 0; h < hc; h++) {
      const int s = P.halo_idx[ho + h];
      if (s >= 0 && s < S) {
        hpos[s] = -1;
        ppos[s] = cnt + h;
        pslots.push_back(s);
      }
    }
    for (int x = 0; x < xc; x++) {
      const int s = P.uvx_idx[xo + x];
      if (s >= 0 && s < nuv) xpos[s] = -1;
    }
  }
  if (bad) return bad;

  // subcycle dependencies: exactly the owners of what each tile reads (its
  // own points, extras and halo) and the tiles that read its points
  if (P.dep_off.size() != (size_t)T + 1 || P.dep_off.front() != 0 ||
      (size_t)P.dep_off.back() != P.dep_idx.size()) {
    note(bad, first, "dependency lists: %zu offsets for %d tiles", P.dep_off.size(), T);
    return bad;
  }
  std::vector<std::vector<int32_t>> want((size_t)T);
  for (int t = 0; t < T; t++) {
    want[t].push_back(t);
    for (int x = P.uvx_off[t]; x < P.uvx_off[t] + P.uvx_cnt[t]; x++)
      if (P.uvx_idx[x] < S) want[t].push_back(tile_of[P.uvx_idx[x]]);
    for (int h = P.halo_off[t]; h < P.halo_off[t] + P.halo_cnt[t]; h++)
      want[t].push_back(tile_of[P.halo_idx[h]]);
  }
  for (int t = 0; t < T; t++)
    for (size_t k = 0, n = want[t].size(); k < n; k++) want[want[t][k]].push_back(t);
  for (int t = 0; t < T; t++) {
    std::sort(want[t].begin(), want[t].end());
    want[t].erase(std::unique(want[t].begin(), want[t].end()), want[t].end());
    const int d0 = P.dep_off[t], d1 = P.dep_off[t + 1];
    if (d1 < d0 || (size_t)(d1 - d0) != want[t].size() ||
        !std::equal(want[t].begin(), want[t].end(), P.dep_idx.begin() + d0))
      note(bad, first, "tile %d: %d dependencies, want %zu", t, d1 - d0, want[t].size());
  }
  return bad;
}

}  // namespace evp
