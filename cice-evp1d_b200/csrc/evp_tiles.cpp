// evp_tiles.cpp -- tile plan of the fused solver.
//
// Step 1: grid coordinates.  Either given (2D entry points) or rebuilt from
//   the neighbour vectors by a breadth-first walk: ee = (i-1,j),
//   ne = (i-1,j-1), se = (i,j-1), nw = (i+1,j), sw = (i+1,j+1),
//   sse = (i,j+1) (integration/ice_dyn_evp1d.F90:766-772).  Each connected
//   piece of the list gets its own origin.  A graph that contradicts itself
//   (two coordinates for one point, or two points on one coordinate) has no
//   grid layout, and the points then keep their list order.
// Step 2: order.  Each piece is cut into strips of strip_w columns; a strip's
//   points are taken row by row from the top row down, each row right to
//   left.  stepu's neighbours nw, sw, sse lie at +i or +j, so every one of
//   them inside the strip comes at most strip_w + 1 places EARLIER in this
//   order: in the same tile, or in the tile before it.  Only the strip's
//   right edge (about one point per row) and the top of a run need their
//   stress recomputed as a forward halo.
// Step 3: runs and tiles.  The order is cut into runs of at most K tiles, one
//   run per CTA, K as small as the CTA count allows.  Within a run each tile
//   takes the longest prefix of the remaining points whose compute set
//   (owned points plus the forward-halo points that neither this tile nor
//   the run's previous tile holds) fits max_tile threads, kTileHalo halo
//   points and kTileUvx extra velocities.
#include "evp_tiles.h"

#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

namespace evp {

namespace {

const int kDI[6] = {-1, -1, 0, +1, +1, 0};  // ee ne se nw sw sse
const int kDJ[6] = {0, -1, -1, 0, +1, +1};

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

// The points of every piece in strips (step 2), pieces in a canonical order
// that does not depend on the list order: larger first, then by extent, then
// by the position of the piece's first point in its own strip order.
std::vector<int32_t> strip_order(int na, std::vector<int32_t> &ci, std::vector<int32_t> &cj,
                                 const std::vector<int32_t> &comp, int strip_w) {
  int nc = 0;
  for (int p = 0; p < na; p++) nc = comp[p] + 1 > nc ? comp[p] + 1 : nc;
  std::vector<int32_t> mi((size_t)nc, INT_MAX), mj((size_t)nc, INT_MAX);
  for (int p = 0; p < na; p++) {
    mi[comp[p]] = std::min(mi[comp[p]], ci[p]);
    mj[comp[p]] = std::min(mj[comp[p]], cj[p]);
  }
  for (int p = 0; p < na; p++) {
    ci[p] -= mi[comp[p]];
    cj[p] -= mj[comp[p]];
  }
  std::vector<int32_t> pn((size_t)nc, 0), pw((size_t)nc, 0), ph((size_t)nc, 0);
  for (int p = 0; p < na; p++) {
    pn[comp[p]]++;
    pw[comp[p]] = std::max(pw[comp[p]], ci[p] + 1);
    ph[comp[p]] = std::max(ph[comp[p]], cj[p] + 1);
  }
  // position in the strip order of a piece: strip, then rows top down, then
  // columns right to left
  auto key = [&](int p) -> long long {
    const long long strip = ci[p] / strip_w;
    return (strip * (long long)(ph[comp[p]] + 1) + (ph[comp[p]] - 1 - cj[p])) * (long long)(strip_w + 1) +
           (strip_w - 1 - ci[p] % strip_w);
  };
  std::vector<long long> pfirst((size_t)nc, LLONG_MAX);
  for (int p = 0; p < na; p++) pfirst[comp[p]] = std::min(pfirst[comp[p]], key(p));
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
    return key(a) < key(b);
  });
  return order;
}

// Incremental bookkeeping of one tile under construction (step 3): points
// join in order, and the forward halo and the extra velocities are kept
// counted with reference counts, so that the longest fitting prefix is found
// in one pass.
class TileBuilder {
 public:
  TileBuilder(int na, int navel, const int32_t *const nb0[6])
      : na_(na), nb_(nb0), owned_(navel, 0), prev_(navel, 0), href_(navel, 0),
        xref_(navel, 0) {}

  // Start a tile; `prev` = the compute set of the run's previous tile
  // (empty for the first tile of a run).
  void begin(const std::vector<int32_t> &prev) {
    clear();
    for (int q : prev) prev_[q] = 1;
    prev_list_ = prev;
  }

  void add(int p) {
    if (in_halo(p)) {  // p was a halo point: drop what it asked for
      nh_--;
      xdec(p);
      for (int r = 0; r < 3; r++) xdec(nb_[r][p]);
    }
    if (xref_[p] > 0) nx_--;  // p no longer an extra velocity
    owned_[p] = 1;
    touch(p);
    members_.push_back(p);
    for (int r = 0; r < 3; r++) xinc(nb_[r][p]);
    for (int r = 3; r < 6; r++) {
      const int q = nb_[r][p];
      if (q >= na_) continue;
      touch(q);
      if (++href_[q] == 1 && !owned_[q] && !prev_[q]) {
        nh_++;
        xinc(q);
        for (int r2 = 0; r2 < 3; r2++) xinc(nb_[r2][q]);
      }
    }
  }

  int owned() const { return (int)members_.size(); }
  int halo() const { return nh_; }
  int extras() const { return nx_; }

  // The forward-halo points, in the order the owned points first reach them.
  std::vector<int32_t> halo_list() const {
    std::vector<int32_t> h;
    std::vector<int32_t> seen;
    for (int p : members_)
      for (int r = 3; r < 6; r++) {
        const int q = nb_[r][p];
        if (q < na_ && in_halo(q) && std::find(seen.begin(), seen.end(), q) == seen.end()) {
          seen.push_back(q);
          h.push_back(q);
        }
      }
    return h;
  }

  void clear() {
    for (int q : touched_) owned_[q] = href_[q] = xref_[q] = 0;
    for (int q : prev_list_) prev_[q] = 0;
    touched_.clear();
    prev_list_.clear();
    members_.clear();
    nh_ = nx_ = 0;
  }

 private:
  bool in_halo(int q) const { return q < na_ && href_[q] > 0 && !owned_[q] && !prev_[q]; }
  void touch(int q) { touched_.push_back(q); }
  void xinc(int q) {
    touch(q);
    if (++xref_[q] == 1 && !owned_[q]) nx_++;
  }
  void xdec(int q) {
    if (--xref_[q] == 0 && !owned_[q]) nx_--;
  }

  int na_;
  const int32_t *const *nb_;
  std::vector<int32_t> owned_, prev_, href_, xref_;
  std::vector<int32_t> touched_, prev_list_, members_;
  int nh_ = 0, nx_ = 0;
};

struct Tiling {
  std::vector<std::vector<int32_t>> tiles;  // owned points of each tile
  std::vector<int32_t> run_off;
};

// Tiles of order[k0, k1) in runs of at most `per_run` tiles; a run never
// holds a previous-tile reference in its first tile.  per_run <= 0: one run.
Tiling make_tiles(TileBuilder &tb, const std::vector<int32_t> &order, int max_tile, int per_run) {
  Tiling T;
  T.run_off.push_back(0);
  const int n = (int)order.size();
  std::vector<int32_t> prev;
  int in_run = 0;
  for (int k = 0; k < n;) {
    if (per_run > 0 && in_run == per_run) {
      T.run_off.push_back((int)T.tiles.size());
      in_run = 0;
      prev.clear();
    }
    tb.begin(prev);
    int best = 1;
    // the counts are not monotone in the prefix length (a later point can
    // absorb a halo point), so every length up to the cap is tried
    for (int len = 1; len <= max_tile && k + len <= n; len++) {
      tb.add(order[k + len - 1]);
      if (len + tb.halo() <= max_tile && tb.halo() <= kTileHalo && tb.extras() <= kTileUvx)
        best = len;
    }
    // the chosen prefix again, for its halo list
    tb.begin(prev);
    for (int q = 0; q < best; q++) tb.add(order[k + q]);
    std::vector<int32_t> members(order.begin() + k, order.begin() + k + best);
    prev = members;
    for (int q : tb.halo_list()) prev.push_back(q);
    tb.clear();
    T.tiles.push_back(std::move(members));
    in_run++;
    k += best;
  }
  T.run_off.push_back((int)T.tiles.size());
  return T;
}

}  // namespace

void build_tile_plan(int na, int navel, const int32_t *const nb0[6],
                     const int32_t *coords_i, const int32_t *coords_j,
                     TilePlan *plan, int max_tile, int nruns, int strip_w) {
  const int tmax = max_tile < 1 ? 1 : (max_tile > kTileCompute ? kTileCompute : max_tile);
  const int want_runs = nruns < 1 ? 1 : nruns;
  const int w = strip_w >= 1 ? strip_w
                             : ((long long)na >= (long long)kStripWideRun * want_runs ? kStripWide
                                                                                     : kStripNarrow);
  TilePlan &P = *plan;
  P = TilePlan();
  P.na = na;
  P.navel = navel;
  P.nhalo_slots = navel - na;
  P.run_off.assign(1, 0);
  P.dep_off.assign(1, 0);
  if (na == 0) return;

  // ---- steps 1 + 2: the order ----------------------------------------------
  std::vector<int32_t> ci, cj, comp, order;
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
    order = strip_order(na, ci, cj, comp, w);
  } else {
    order.resize((size_t)na);
    for (int p = 0; p < na; p++) order[p] = p;
  }

  // ---- step 3: runs of at most K tiles, K as small as the CTAs allow -------
  TileBuilder tb(na, navel, nb0);
  const Tiling whole = make_tiles(tb, order, tmax, 0);
  int K = ((int)whole.tiles.size() + want_runs - 1) / want_runs;
  Tiling T;
  for (;; K++) {
    T = make_tiles(tb, order, tmax, K);
    if ((int)T.run_off.size() - 1 <= want_runs) break;
  }
  std::vector<std::vector<int32_t>> &tiles = T.tiles;
  P.nruns = (int)T.run_off.size() - 1;
  P.run_off = T.run_off;

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
  std::vector<char> first_of_run((size_t)P.ntiles, 0);
  for (int r = 0; r < P.nruns; r++)
    if (P.run_off[r] < P.ntiles) first_of_run[P.run_off[r]] = 1;
  // cpos/ctile: str-table position of a list point in tile ctile's compute
  // set (owned: its slot offset; halo h: tile_cnt + h), for the current and
  // the previous tile; xpos/xtile: velocity-extra position of any u/v point
  std::vector<int32_t> cpos((size_t)na, -1), ctile((size_t)na, -1);
  std::vector<int32_t> ppos((size_t)na, -1), ptile((size_t)na, -1);
  std::vector<int32_t> xpos((size_t)navel, -1), xtile((size_t)navel, -1);
  for (int t = 0; t < P.ntiles; t++) {
    P.halo_off[t] = (int)P.halo_idx.size();
    P.uvx_off[t] = (int)P.uvx_idx.size();
    int nh = 0, nx = 0;
    const int own = P.tile_cnt[t];
    const bool has_prev = !first_of_run[t];
    std::vector<int32_t> &members = tiles[t];
    for (int k = 0; k < own; k++) {
      ctile[members[k]] = t;
      cpos[members[k]] = k;
    }
    // stepu's str neighbours and the forward halo
    for (int k = 0; k < own; k++) {
      const int p = members[k];
      uint32_t packed = 0;
      for (int r = 3; r < 6; r++) {
        const int n = nb0[r][p];
        uint32_t loc;
        if (n >= na) {
          loc = kZeroSlot;
        } else if (ctile[n] == t) {
          loc = (uint32_t)cpos[n];
        } else if (has_prev && ptile[n] == t - 1) {
          loc = kStrPrev | (uint32_t)ppos[n];
        } else {
          ctile[n] = t;  // first time this tile reaches n: a halo point
          cpos[n] = own + nh++;
          P.halo_idx.push_back(P.slot_of_point[n]);
          loc = (uint32_t)cpos[n];
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
    // this tile's compute set is the next tile's previous table
    for (int k = 0; k < own; k++) {
      ptile[members[k]] = t;
      ppos[members[k]] = k;
    }
    for (int h = 0; h < nh; h++) {
      const int q = P.point_of_slot[P.halo_idx[P.halo_off[t] + h]];
      ptile[q] = t;
      ppos[q] = own + h;
    }
  }

  // ---- subcycle-to-subcycle dependencies ------------------------------------
  // reads[t]: owners of the list points tile t reads; deps = reads + reverse
  std::vector<std::vector<int32_t>> deps((size_t)P.ntiles);
  for (int t = 0; t < P.ntiles; t++) {
    std::vector<int32_t> &r = deps[t];
    r.push_back(t);
    for (int x = P.uvx_off[t]; x < P.uvx_off[t] + P.uvx_cnt[t]; x++)
      if (P.uvx_idx[x] < P.nslots) r.push_back(tile_of[P.point_of_slot[P.uvx_idx[x]]]);
    for (int h = P.halo_off[t]; h < P.halo_off[t] + P.halo_cnt[t]; h++)
      r.push_back(tile_of[P.point_of_slot[P.halo_idx[h]]]);
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
  }
  for (int t = 0; t < P.ntiles; t++)
    for (size_t k = 0; k < deps[t].size(); k++) {
      const int u = deps[t][k];
      if (u != t && u >= 0 && !std::binary_search(deps[u].begin(), deps[u].end(), t))
        deps[u].push_back(t);  // sorted again below
    }
  P.dep_off.assign((size_t)P.ntiles + 1, 0);
  for (int t = 0; t < P.ntiles; t++) {
    std::sort(deps[t].begin(), deps[t].end());
    deps[t].erase(std::unique(deps[t].begin(), deps[t].end()), deps[t].end());
    P.dep_off[t + 1] = P.dep_off[t] + (int)deps[t].size();
  }
  P.dep_idx.reserve((size_t)P.dep_off[P.ntiles]);
  for (int t = 0; t < P.ntiles; t++)
    P.dep_idx.insert(P.dep_idx.end(), deps[t].begin(), deps[t].end());
}

}  // namespace evp
