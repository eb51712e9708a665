// evp_tiles.h -- host-side tile plan of the fused solver (internal).
//
// The 1D list is regrouped into tiles of at most kTileOwned points.  A tile
// owns its points (their stresses and velocities are written by the tile's
// CTA only) and also recomputes `stress` on its forward halo: the points that
// its owned points reach through nw/sw/sse and that another tile owns.  With
// the halo recomputed locally, every str1..str8 value stepu needs is produced
// in the CTA's shared memory and str never travels through HBM.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace evp {

constexpr int kTileOwned = 256;   // owned slots per tile (one thread each)
constexpr int kTileHalo = 64;     // maximum forward-halo points per tile
constexpr int kTileUvx = 128;     // maximum extra velocity points per tile
constexpr int kTileW = 16;        // tile width in i (grid cells)
constexpr int kTileH = 16;        // tile height in j
// Shared-memory index spaces of one tile:
//  compute set (str):  owned c -> c, forward halo h -> kTileOwned + h,
//                      kZeroSlot -> a slot holding str = 0;
//  velocities (u, v):  owned c -> c, extra x -> kTileOwned + x.
constexpr int kTileCompute = kTileOwned + kTileHalo;
constexpr int kZeroSlot = kTileCompute;
// Per-tile producer record (int32): [0] slot offset, [1] owned count,
// [2] extra velocity count, [3] halo count, [4..7] unused, then the extra
// velocity slots, the halo slots, the halo points' packed corner indices and
// their own velocity indices.
constexpr int kRecUvx = 8;
constexpr int kRecHalo = kRecUvx + kTileUvx;
constexpr int kRecHLcor = kRecHalo + kTileHalo;
constexpr int kRecHLcc = kRecHLcor + kTileHalo;
constexpr int kRecInts = kRecHLcc + kTileHalo;
constexpr int kSlotAlign = 4;     // tile starts are multiples of 4 slots (32 B)
constexpr int kLnbBits = 10;      // bits per packed local index
constexpr uint32_t kLnbMask = (1u << kLnbBits) - 1;

struct TilePlan {
  int na = 0, navel = 0;
  int ntiles = 0;
  int nslots = 0;        // owned slots incl. alignment padding
  int nhalo_slots = 0;   // navel - na: the reference's halo slots, appended
  bool from_coords = false;  // tiles from reconstructed (i,j); else 1D chunks
  std::vector<int32_t> slot_of_point;  // [na]
  std::vector<int32_t> point_of_slot;  // [nslots], -1 for padding
  std::vector<int32_t> tile_off, tile_cnt, halo_off, halo_cnt;  // [ntiles]
  std::vector<int32_t> halo_idx;       // slots of the forward-halo points
  // neighbour slots in the u/v/str index space [0, nslots + nhalo_slots)
  std::vector<int32_t> ee, ne, se, nw, sw, sse;  // [nslots]
  // packed compute-set indices of nw, sw, sse (stepu's str gathers)
  std::vector<uint32_t> lnb;  // [nslots]
  // packed velocity indices of ee, ne, se (stress's u/v gathers)
  std::vector<uint32_t> lcor;  // [nslots]
  // per forward-halo entry: velocity index of the point itself and packed
  // velocity indices of its ee, ne, se, in the recomputing tile's space
  std::vector<uint32_t> halo_lcc, halo_lcor;  // [halo_idx.size()]
  // extra velocity points of each tile (u/v slots outside its owned range)
  std::vector<int32_t> uvx_off, uvx_cnt;  // [ntiles]
  std::vector<int32_t> uvx_idx;
};

// Build the plan from 0-based neighbour vectors (values in [0, navel)).
// coords_i/coords_j may be null; then (i,j) are reconstructed from the
// neighbour graph, and if that is inconsistent the plan falls back to tiles
// of consecutive list points.  Tiles hold at most max_tile points
// (1..kTileOwned; the kernels' shared-memory layout stays kTileOwned wide).
void build_tile_plan(int na, int navel, const int32_t *const nb0[6],
                     const int32_t *coords_i, const int32_t *coords_j,
                     TilePlan *plan, int max_tile = kTileOwned);

// Decode every index of `plan` that the kernels gather through (slot maps,
// tile ranges, neighbour slots, forward halos, velocity extras, the packed
// local indices) and compare it with what the 0-based neighbour vectors say
// it must be.  Returns the number of violations; *first (if not null) then
// describes the first one.  Host only (evp_plan_check.cpp).
long long verify_tile_plan(const TilePlan &plan, const int32_t *const nb0[6], int max_tile,
                           std::string *first);

}  // namespace evp
