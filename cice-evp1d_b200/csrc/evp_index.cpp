// evp_index.cpp -- host-side 2D -> 1D index space of the evp1d adapter.
//
// Produces the same 1D list, halo slots and neighbour vectors as
// calc_2d_indices_init + calc_navel + convert_2d_1d_init
// (integration/ice_dyn_evp1d.F90:559-589, 743-797, 1047-1087):
//   - list points: mask(i,j) true, j outer from 1+nghost to ny, i inner from
//     1+nghost to nx (northern/eastern ghost rows included as in the
//     reference);
//   - linear index i + (j-1)*nx;
//   - halo slots: the linear indices reached by the six stencil offsets that
//     are not list points, sorted, after the na list points;
//   - neighbour vectors: 1-based slot of (i-1,j) ee, (i-1,j-1) ne, (i,j-1) se,
//     (i+1,j) nw, (i+1,j+1) sw, (i,j+1) sse.
// The reference merges seven sorted vectors and walks them with two cursors;
// here the union is one sort + unique and each neighbour is located by binary
// search, which gives the same slots in O(na log na).
#include <algorithm>
#include <cstdint>
#include <vector>

#include "evp1d.h"

namespace evp {
int error(int code, const char *fmt, ...);  // evp1d_api.cu
}

extern "C" int evp1d_build_index(int nx, int ny, int nghost,
                                 const int32_t *mask, int cap_na,
                                 int cap_navel, int *na_out, int *navel_out,
                                 int32_t *indxti, int32_t *indxtj,
                                 int32_t *indxtij, int32_t *ee, int32_t *ne,
                                 int32_t *se, int32_t *nw, int32_t *sw,
                                 int32_t *sse) {
  if (nx <= 0 || ny <= 0 || nghost < 0 || !mask || !na_out || !navel_out)
    return evp::error(EVP1D_ERR_INVALID_ARG, "bad grid arguments");
  if ((long long)nx * (long long)(ny + 1) + 2 > 0x7fffffffLL)
    return evp::error(EVP1D_ERR_INVALID_ARG, "grid too large for int32 indices");
  std::vector<int32_t> lin;
  std::vector<int32_t> ti, tj;
  for (int j = 1 + nghost; j <= ny; j++)
    for (int i = 1 + nghost; i <= nx; i++)
      if (mask[(size_t)(i - 1) + (size_t)(j - 1) * (size_t)nx]) {
        ti.push_back(i);
        tj.push_back(j);
        lin.push_back(i + (j - 1) * nx);
      }
  const int na = (int)lin.size();
  // stencil offsets in the order ee, ne, se, nw, sw, sse
  const int32_t off[6] = {-1, -1 - nx, -nx, +1, +1 + nx, +nx};
  std::vector<int32_t> all;
  all.reserve((size_t)na * 7);
  all.insert(all.end(), lin.begin(), lin.end());
  for (int k = 0; k < 6; k++)
    for (int w = 0; w < na; w++) all.push_back(lin[w] + off[k]);
  std::sort(all.begin(), all.end());
  all.erase(std::unique(all.begin(), all.end()), all.end());
  const int navel = (int)all.size();
  *na_out = na;
  *navel_out = navel;
  if (na > cap_na || navel > cap_navel)
    return evp::error(EVP1D_ERR_INVALID_ARG,
                      "capacity too small: need na=%d navel=%d", na, navel);
  if (!indxti || !indxtj || !indxtij || !ee || !ne || !se || !nw || !sw || !sse) {
    if (na == 0) return EVP1D_OK;
    return evp::error(EVP1D_ERR_INVALID_ARG, "output array is NULL");
  }
  // slot of each linear index: list points 1..na in list order, halo points
  // na+1..navel in increasing linear index.  `lin` is sorted (j outer,
  // i inner), so both parts are sorted and a merge walk assigns slots.
  std::vector<int32_t> slot((size_t)navel);
  {
    int a = 0, h = na;
    for (int q = 0; q < navel; q++) {
      if (a < na && all[q] == lin[a]) {
        slot[q] = ++a;
      } else {
        indxtij[h] = all[q];
        slot[q] = ++h;
      }
    }
  }
  for (int w = 0; w < na; w++) {
    indxti[w] = ti[w];
    indxtj[w] = tj[w];
    indxtij[w] = lin[w];
  }
  int32_t *outs[6] = {ee, ne, se, nw, sw, sse};
  for (int k = 0; k < 6; k++)
    for (int w = 0; w < na; w++) {
      const int32_t x = lin[w] + off[k];
      const size_t q = (size_t)(std::lower_bound(all.begin(), all.end(), x) - all.begin());
      outs[k][w] = slot[q];
    }
  return EVP1D_OK;
}
