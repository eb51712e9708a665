// evp_tiles.h -- host-side tile plan of the fused solver (internal).
//
// The 1D list is regrouped into tiles, and the tiles into runs: run r is the
// contiguous range of tiles [run_off[r], run_off[r+1]) that CTA r of the
// subcycle kernel works through, in order.  A tile owns its points (their
// stresses and velocities are written by the tile's CTA only).  stepu of an
// owned point reads str1..str8 at the point and at its nw/sw/sse neighbours.
// A neighbour's str is found in one of three places, all in the CTA's shared
// memory:
//   - the tile's own str table, when the tile owns the neighbour;
//   - the str table of the previous tile of the same run, when that tile
//     owns the neighbour or recomputed it (the tables of two consecutive
//     tiles are alive at once);
//   - otherwise the tile recomputes `stress` at the neighbour itself: the
//     neighbour joins the tile's forward halo.
// So str never travels through HBM.  Points are ordered so that the first
// two places serve almost every neighbour (evp_tiles.cpp).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace evp {

constexpr int kTileOwned = 256;    // owned slots per tile (constant block width)
constexpr int kTileCompute = 256;  // owned + forward-halo points per tile (one thread each)
constexpr int kTileHalo = 64;      // maximum forward-halo points per tile
constexpr int kTileUvx = 128;      // maximum extra velocity points per tile
// Shared-memory index spaces of one tile (10-bit fields, three to a word):
//  str (stepu's nw/sw/sse):  own table position c < kTileCompute (owned point
//                            c, or forward-halo point h at tile_cnt + h);
//                            kZeroSlot, a position holding str = 0 (the
//                            reference's halo slots, whose str stays 0);
//                            kStrPrev | c, position c of the previous tile's
//                            table (never in the first tile of a run);
//  velocities (u, v):        owned c -> c, extra x -> kTileOwned + x.
constexpr int kZeroSlot = kTileCompute;
constexpr uint32_t kStrPrev = 512;
constexpr int kStrRow = kTileCompute + 2;  // doubles per str field row (zero slot, 16-B rows)
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
// Widths (grid columns) of the strips the grid points are ordered in, chosen
// by the points per run: wide strips recompute less of the strip's right
// edge, narrow ones less of the row above a run's first tile, which matters
// when runs are short (grid1600x1200, 8,000 points per run: 97.9 us per
// subcycle at 64 columns against 100.1 at 48 and 100.3 at 80; the halo cap
// of 64 points bounds the width).
constexpr int kStripWide = 64, kStripNarrow = 48;
constexpr int kStripWideRun = 4096;  // points per run from which strips are wide

struct TilePlan {
  int na = 0, navel = 0;
  int ntiles = 0;
  int nruns = 0;         // CTAs of the subcycle kernel (<= the requested count)
  int nslots = 0;        // owned slots incl. alignment padding
  int nhalo_slots = 0;   // navel - na: the reference's halo slots, appended
  bool from_coords = false;  // points ordered by reconstructed (i,j); else list order
  std::vector<int32_t> slot_of_point;  // [na]
  std::vector<int32_t> point_of_slot;  // [nslots], -1 for padding
  std::vector<int32_t> run_off;        // [nruns + 1] tile ranges of the runs
  std::vector<int32_t> tile_off, tile_cnt, halo_off, halo_cnt;  // [ntiles]
  std::vector<int32_t> halo_idx;       // slots of the forward-halo points
  // neighbour slots in the u/v/str index space [0, nslots + nhalo_slots)
  std::vector<int32_t> ee, ne, se, nw, sw, sse;  // [nslots]
  // packed str indices of nw, sw, sse (stepu's str gathers)
  std::vector<uint32_t> lnb;  // [nslots]
  // packed velocity indices of ee, ne, se (stress's u/v gathers)
  std::vector<uint32_t> lcor;  // [nslots]
  // per forward-halo entry: velocity index of the point itself and packed
  // velocity indices of its ee, ne, se, in the recomputing tile's space
  std::vector<uint32_t> halo_lcc, halo_lcor;  // [halo_idx.size()]
  // extra velocity points of each tile (u/v slots outside its owned range)
  std::vector<int32_t> uvx_off, uvx_cnt;  // [ntiles]
  std::vector<int32_t> uvx_idx;
  // tiles a tile depends on from one subcycle to the next: the owners of
  // every point it reads (itself, its extras, its forward halo) and the
  // tiles that read any of its points; sorted, CSR [dep_off[t], dep_off[t+1])
  std::vector<int32_t> dep_off;  // [ntiles + 1]
  std::vector<int32_t> dep_idx;
};

// Build the plan from 0-based neighbour vectors (values in [0, navel)) for a
// kernel of at most `nruns` CTAs.  coords_i/coords_j may be null; then (i,j)
// are reconstructed from the neighbour graph, and if that is inconsistent
// the points keep their list order.  A tile's compute set (owned points plus
// forward halo) holds at most max_tile points (1..kTileCompute); strip_w is
// the width of the strips grid points are ordered in (0: by points per run).
void build_tile_plan(int na, int navel, const int32_t *const nb0[6],
                     const int32_t *coords_i, const int32_t *coords_j,
                     TilePlan *plan, int max_tile = kTileCompute, int nruns = 148,
                     int strip_w = 0);

// Decode every index of `plan` that the kernels gather through (slot maps,
// runs and tile ranges, neighbour slots, forward halos, velocity extras, the
// packed local indices) and compare it with what the 0-based neighbour
// vectors say it must be.  Returns the number of violations; *first (if not
// null) then describes the first one.  Host only (evp_plan_check.cpp).
long long verify_tile_plan(const TilePlan &plan, const int32_t *const nb0[6], int max_tile,
                           std::string *first);

}  // namespace evp
