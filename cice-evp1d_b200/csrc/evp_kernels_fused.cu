// evp_kernels_fused.cu -- one EVP subcycle per launch with plain loads: CTA r
// works through the tiles of run r in order.
//
// Phase 1 (stress, src/bench_v2b.F90:126-311): every thread takes a point of
//   the tile's compute set -- its owned points followed by its forward halo
//   (points reached through nw/sw/sse that neither this tile nor the run's
//   previous tile holds).  Velocities come from the previous subcycle's
//   buffer; new stresses of owned points go to the other buffer; str1..str8
//   of every compute-set point go to the tile's shared str table (0 for skipT
//   points, and a fixed zero slot stands for the reference's halo slots,
//   whose str stays 0).
// Phase 2 (stepu, src/bench_v2b.F90:506-547): one thread per owned point reads
//   str of itself and of nw/sw/sse from the tile's table or from the previous
//   tile's, and writes the new velocity to the other buffer.
//
// Recomputing the halo points' stress (owners compute the same values from
// the same inputs with the same operations) keeps str on chip: per point and
// subcycle the kernel moves the stress inputs and state, the stepu inputs and
// the velocity, and never str1..str8.  This is the plain-load counterpart of
// the TMA kernel (evp_kernels_tma.cu), kept as a second implementation of
// the same plan.
#include "evp_kernels.cuh"
#include "evp_tiles.h"

namespace evp {

namespace {

template <bool kLast>
__global__ void __launch_bounds__(kTileCompute, 1)
k_fused(FusedArgs a, Params p) {
  __shared__ double s_str[2][8][kStrRow];
  const int tid = threadIdx.x;
  if (tid < 16) s_str[tid >> 3][tid & 7][kZeroSlot] = 0.0;
  const int T0 = a.run_off[blockIdx.x], T1 = a.run_off[blockIdx.x + 1];
  for (int t = T0; t < T1; t++) {
    const int b = (t - T0) & 1;  // this tile's table; the previous tile's is b ^ 1
    const int own = a.tile_cnt[t], base = a.tile_off[t];
    const int nh = a.halo_cnt[t], hb = a.halo_off[t];
    // the previous tile's stepu has read table b (its b ^ 1) before it is refilled
    __syncthreads();

    // ---------------- phase 1: stress on owned points + forward halo ------
    for (int c = tid; c < own + nh; c += kTileCompute) {
      const bool owned = c < own;
      const int g = owned ? base + c : a.halo_idx[hb + (c - own)];
      double out[8];
      if (a.flags[g] & kSkipT) {
#pragma unroll
        for (int k = 0; k < 8; k++) out[k] = 0.0;
      } else {
        const int iee = a.ee[g], ine = a.ne[g], ise = a.se[g];
        Corners cr;
        cr.ucc = a.u_in[g];
        cr.vcc = a.v_in[g];
        cr.uee = a.u_in[iee];
        cr.vee = a.v_in[iee];
        cr.une = a.u_in[ine];
        cr.vne = a.v_in[ine];
        cr.use = a.u_in[ise];
        cr.vse = a.v_in[ise];
        const Geom gm = make_geom(a.dxT[g], a.dyT[g], a.HTE[g], a.HTN[g],
                                  a.HTEm1[g], a.HTNm1[g], p.deltaminEVP);
        const Strain sr = strain_rates(cr, gm, p.e_factor);
        double st[12];
#pragma unroll
        for (int k = 0; k < 12; k++) st[k] = a.s_in[k][g];
        stress_update(st, out, sr, a.strength[g], gm, p);
        if (owned) {
#pragma unroll
          for (int k = 0; k < 12; k++) a.s_out[k][g] = st[k];
        }
      }
#pragma unroll
      for (int k = 0; k < 8; k++) s_str[b][k][c] = out[k];
      if (kLast && owned) {
#pragma unroll
        for (int k = 0; k < 8; k++) a.str_out[k][g] = out[k];
      }
    }
    __syncthreads();

    // ---------------- phase 2: stepu on owned points ----------------------
    if (tid < own) {
      const int g = base + tid;
      if (!(a.flags[g] & kSkipU)) {
        const uint32_t pk = a.lnb[g];
        const uint32_t vnw = pk & kLnbMask, vsw = (pk >> kLnbBits) & kLnbMask;
        const uint32_t vsse = (pk >> (2 * kLnbBits)) & kLnbMask;
        const int bnw = (vnw & kStrPrev) ? b ^ 1 : b, bsw = (vsw & kStrPrev) ? b ^ 1 : b;
        const int bsse = (vsse & kStrPrev) ? b ^ 1 : b;
        const int lnw = vnw & (kStrPrev - 1), lsw = vsw & (kStrPrev - 1);
        const int lsse = vsse & (kStrPrev - 1);
        StepuIn in;
        in.uold = a.u_in[g];
        in.vold = a.v_in[g];
        in.kvrel = a.kvrel[g];
        in.uocn = a.uocn[g];
        in.vocn = a.vocn[g];
        in.waterx = a.waterx[g];
        in.watery = a.watery[g];
        in.forcex = a.forcex[g];
        in.forcey = a.forcey[g];
        in.umassdti = a.umassdti[g];
        in.fm = a.fm[g];
        in.uarear = a.uarear[g];
        in.Tbu = a.Tbu[g];
        in.uinit = a.uinit[g];
        in.vinit = a.vinit[g];
        in.s1 = s_str[b][0][tid];
        in.s2nw = s_str[bnw][1][lnw];
        in.s3sse = s_str[bsse][2][lsse];
        in.s4sw = s_str[bsw][3][lsw];
        in.s5 = s_str[b][4][tid];
        in.s6sse = s_str[bsse][5][lsse];
        in.s7nw = s_str[bnw][6][lnw];
        in.s8sw = s_str[bsw][7][lsw];
        const StepuOut o = stepu_point(in, p);
        a.u_out[g] = o.u;
        a.v_out[g] = o.v;
        if (kLast) {
          a.strintx[g] = o.strintx;
          a.strinty[g] = o.strinty;
          a.Cb[g] = o.Cb;
        }
      }
    }
  }
}

__global__ void k_scatter(PermBatch b, int nslots, const int32_t *pos) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots;
       s += gridDim.x * blockDim.x) {
    const int p = pos[s];
    for (int f = 0; f < b.n; f++) {
      const double v = p >= 0 ? b.src[f][p] : 0.0;
      b.dst[f][s] = v;
      if (b.dst2[f]) b.dst2[f][s] = v;
    }
  }
}

__global__ void k_gather(PermBatch b, int na, const int32_t *sop) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < na;
       q += gridDim.x * blockDim.x) {
    const int s = sop[q];
    for (int f = 0; f < b.n; f++) b.dst[f][q] = b.src[f][s];
  }
}

__global__ void k_flags(int nslots, const int32_t *pos, const int32_t *skipT,
                        const int32_t *skipU, uint8_t *flags,
                        const uint32_t *lnb, uint32_t *meta) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots;
       s += gridDim.x * blockDim.x) {
    const int p = pos[s];
    const uint8_t f = p < 0 ? (uint8_t)(kSkipT | kSkipU)
                            : (uint8_t)((skipT[p] ? kSkipT : 0) | (skipU[p] ? kSkipU : 0));
    flags[s] = f;
    meta[s] = lnb[s] | ((uint32_t)f << 30);
  }
}

__global__ void k_drag(int n, const double *aiu, const double *Cw, double rhow,
                       double *kv) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += gridDim.x * blockDim.x)
    kv[s] = drag_factor(aiu[s], rhow, Cw[s]);
}

int blocks_for(int n) {
  int b = (n + 255) / 256;
  return b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b);
}

}  // namespace

void launch_fused(const FusedArgs &a, const Params &p, bool last,
                  cudaStream_t st) {
  if (a.ntiles <= 0 || a.nruns <= 0) return;
  if (last)
    k_fused<true><<<a.nruns, kTileCompute, 0, st>>>(a, p);
  else
    k_fused<false><<<a.nruns, kTileCompute, 0, st>>>(a, p);
}

void launch_scatter(const PermBatch &b, int nslots, const int32_t *pos,
                    cudaStream_t st) {
  if (nslots <= 0 || b.n <= 0) return;
  k_scatter<<<blocks_for(nslots), 256, 0, st>>>(b, nslots, pos);
}

void launch_gather(const PermBatch &b, int na, const int32_t *sop,
                   cudaStream_t st) {
  if (na <= 0 || b.n <= 0) return;
  k_gather<<<blocks_for(na), 256, 0, st>>>(b, na, sop);
}

void launch_flags(int nslots, const int32_t *pos, const int32_t *skipT,
                  const int32_t *skipU, uint8_t *flags, const uint32_t *lnb,
                  uint32_t *meta, cudaStream_t st) {
  if (nslots <= 0) return;
  k_flags<<<blocks_for(nslots), 256, 0, st>>>(nslots, pos, skipT, skipU, flags, lnb, meta);
}

void launch_drag_factor(int n, const double *aiu, const double *Cw,
                        double rhow, double *kv, cudaStream_t st) {
  if (n <= 0) return;
  k_drag<<<blocks_for(n), 256, 0, st>>>(n, aiu, Cw, rhow, kv);
}

namespace {
struct ConstSrc {
  const double *f[kConstFields - 1];
};

__global__ void k_const_blocks(int ntiles, const int32_t *tile_off, const int32_t *tile_cnt,
                               ConstSrc src, const uint32_t *meta, const uint32_t *lcor,
                               double *cblk, int *cflags) {
  constexpr int kTbuSrc = kConstFields - 4, kUinitSrc = kConstFields - 3;
  constexpr int kVinitSrc = kConstFields - 2;
  const long long total = (long long)ntiles * kConstFields * kConstTileSlots;
  int flags = 0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(e % kConstTileSlots);
    const long long tf = e / kConstTileSlots;
    const int f = (int)(tf % kConstFields);
    const int t = (int)(tf / kConstFields);
    double v = 0.0;
    if (l < tile_cnt[t]) {
      const int s = tile_off[t] + l;
      if (f == kConstStressFields - 1) {
        const unsigned long long su =
            (unsigned long long)__double_as_longlong(src.f[kUinitSrc][s]) >> 63;
        const unsigned long long sv =
            (unsigned long long)__double_as_longlong(src.f[kVinitSrc][s]) >> 63;
        v = __longlong_as_double((long long)((unsigned long long)meta[s] |
                                             ((unsigned long long)lcor[s] << 32) | su << 62 |
                                             sv << 63));
      } else {
        const int k = f < kConstStressFields ? f : f - 1;
        v = src.f[k][s];
        if (k == kTbuSrc && __double_as_longlong(v) != 0) flags |= 1;
        if ((k == kUinitSrc || k == kVinitSrc) && !isfinite(v)) flags |= 2;
      }
    }
    cblk[e] = v;
  }
  if (flags) atomicOr(cflags, flags);
}
}  // namespace

void launch_const_blocks(int ntiles, const int32_t *tile_off, const int32_t *tile_cnt,
                         const double *const src[kConstFields - 1], const uint32_t *meta,
                         const uint32_t *lcor, double *cblk, int *cflags, cudaStream_t st) {
  if (ntiles <= 0) return;
  ConstSrc cs;
  for (int f = 0; f < kConstFields - 1; f++) cs.f[f] = src[f];
  const long long total = (long long)ntiles * kConstFields * kConstTileSlots;
  const long long b = (total + 255) / 256;
  k_const_blocks<<<(int)(b < 148 * 32 ? b : 148 * 32), 256, 0, st>>>(
      ntiles, tile_off, tile_cnt, cs, meta, lcor, cblk, cflags);
}

}  // namespace evp
