// plan_check_shim.cpp -- test helper (host only): builds a tile plan with the
// library's planner (csrc/evp_tiles.cpp), plants one mistake of a chosen kind
// in it, and runs the plan verifier (csrc/evp_plan_check.cpp), so that a test
// can check that every kind of wrong index is caught.  Nothing here runs on a
// GPU.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "evp_tiles.h"

namespace {

// A tile with both a forward halo and extra velocity points.
int pick_tile(const evp::TilePlan &P) {
  for (int t = 0; t < P.ntiles; t++)
    if (P.halo_cnt[t] > 0 && P.uvx_cnt[t] > 0 && P.tile_cnt[t] > 1) return t;
  return -1;
}

// Plant mistake `kind` (1..kShimKinds); false if the plan has no place for it.
bool plant(evp::TilePlan &P, int kind) {
  const int t = pick_tile(P);
  if (t < 0) return false;
  const int off = P.tile_off[t], ho = P.halo_off[t], xo = P.uvx_off[t];
  const int far = P.tile_off[(t + P.ntiles / 2) % P.ntiles];
  switch (kind) {
    case 1: {  // two points swap slots in one map only
      const int p = P.point_of_slot[off], q = P.point_of_slot[far];
      std::swap(P.slot_of_point[p], P.slot_of_point[q]);
      return true;
    }
    case 2: P.tile_off[t] += 1; return true;                        // misaligned tile
    case 3: P.lnb[off] ^= 1u; return true;                          // str index of nw
    case 4: P.lcor[off] ^= 1u << evp::kLnbBits; return true;        // velocity index of ne
    case 5: P.halo_idx[ho] = off; return true;                      // own point in the halo
    case 6: P.uvx_idx[xo] = far; return true;                       // wrong extra point
    case 7: P.halo_lcor[ho] ^= 1u; return true;                     // halo point's ee
    case 8: P.halo_lcc[ho] ^= 1u; return true;                      // halo point's own u, v
    case 9: P.tile_cnt[t] = evp::kTileOwned + 1; return true;       // tile over its limit
    case 10: P.nw[off] += 1; return true;                           // neighbour slot
    case 11: P.point_of_slot[off] = -1; return true;                // point lost
    case 12: P.halo_cnt[t] -= 1; return true;                       // halo entry missing
    case 13: P.uvx_cnt[t] -= 1; return true;                        // extra missing
    case 14: {  // a previous-table str index in the first tile of a run
      if (P.nruns < 2) return false;
      const int f = P.run_off[1];
      P.lnb[P.tile_off[f]] = (P.lnb[P.tile_off[f]] & ~evp::kLnbMask) | evp::kStrPrev;
      return true;
    }
    case 15: {  // an empty run
      if (P.nruns < 2) return false;
      P.run_off[1] = P.run_off[0];
      return true;
    }
    case 16: {  // a previous-table index to a point the previous tile lacks
      for (int u = 1; u < P.ntiles; u++) {
        bool first_of_run = false;
        for (int r = 0; r <= P.nruns; r++) first_of_run |= P.run_off[r] == u;
        if (first_of_run) continue;
        for (int s = P.tile_off[u]; s < P.tile_off[u] + P.tile_cnt[u]; s++)
          for (int r = 0; r < 3; r++) {
            const uint32_t v = (P.lnb[s] >> (r * evp::kLnbBits)) & evp::kLnbMask;
            if (v & evp::kStrPrev) {
              const uint32_t w = evp::kStrPrev | ((v + 1) & 255u);
              P.lnb[s] = (P.lnb[s] & ~(evp::kLnbMask << (r * evp::kLnbBits))) |
                         (w << (r * evp::kLnbBits));
              return true;
            }
          }
      }
      return false;
    }
    case 17: {  // a dependency dropped
      for (int u = 0; u < P.ntiles; u++)
        if (P.dep_off[u + 1] - P.dep_off[u] > 1) {
          P.dep_idx.erase(P.dep_idx.begin() + P.dep_off[u]);
          for (int v = u + 1; v <= P.ntiles; v++) P.dep_off[v]--;
          return true;
        }
      return false;
    }
    default: return false;
  }
}

}  // namespace

extern "C" {

int shim_kinds(void) { return 17; }

// 1-based neighbour vectors as evp1d_init takes them.  Returns the number of
// violations found (0 for kind 0 on a good plan), or -1 if the mistake could
// not be planted; msg gets the first violation.
long long shim_plan_check(int na, int navel, const int32_t *const idx[6], int max_tile,
                          int kind, char *msg, int len) {
  std::vector<int32_t> nb0((size_t)na * 6);
  const int32_t *nbp[6];
  for (int k = 0; k < 6; k++) {
    for (int w = 0; w < na; w++) nb0[(size_t)k * na + w] = idx[k][w] - 1;
    nbp[k] = nb0.data() + (size_t)k * na;
  }
  evp::TilePlan plan;
  evp::build_tile_plan(na, navel, nbp, nullptr, nullptr, &plan, max_tile, 4);
  if (kind != 0 && !plant(plan, kind)) return -1;
  std::string first;
  const long long bad = evp::verify_tile_plan(plan, nbp, max_tile, &first);
  if (msg && len > 0) {
    strncpy(msg, first.c_str(), (size_t)len - 1);
    msg[len - 1] = 0;
  }
  return bad;
}

}  // extern "C"
