// evp_kernels_ref.cu -- stress and stepu as two grid-stride kernels over the
// reference's 1D order (src/bench_v2b.F90:62-312, 444-549).
//
// One thread per list point; neighbour values are gathered through the
// 0-based ee/ne/se (stress) and nw/sw/sse (stepu) vectors.  These kernels
// carry the lindividual-style entry points (stress alone, stepu alone) and
// are the reference-order cross-check of the fused solver.
#include "evp_kernels.cuh"

namespace evp {

namespace {

constexpr int kThreads = 256;

// At most 128 registers: two blocks (16 warps) per SM.  kStd: parameters
// with std_params(p) (stress_update_std).
template <bool kStd>
__global__ void __launch_bounds__(kThreads, 2)
k_stress_ref(DevState s, Params p) {
  const int n = s.na;
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n;
       w += gridDim.x * blockDim.x) {
    if (s.flags[w] & kSkipT) continue;
    const int iee = s.ee[w], ine = s.ne[w], ise = s.se[w];
    Corners c;
    c.ucc = s.u[w];
    c.vcc = s.v[w];
    c.uee = s.u[iee];
    c.vee = s.v[iee];
    c.une = s.u[ine];
    c.vne = s.v[ine];
    c.use = s.u[ise];
    c.vse = s.v[ise];
    const Geom g = make_geom(s.dxT[w], s.dyT[w], s.HTE[w], s.HTN[w],
                             s.HTEm1[w], s.HTNm1[w], p.deltaminEVP);
    const Strain sr = strain_rates(c, g, p.e_factor);
    double st[12], out[8];
#pragma unroll
    for (int k = 0; k < 12; k++) st[k] = s.stress[k][w];
    if (kStd)
      stress_update_std(st, out, sr, s.strength[w], g, p);
    else
      stress_update(st, out, sr, s.strength[w], g, p);
#pragma unroll
    for (int k = 0; k < 12; k++) s.stress[k][w] = st[k];
#pragma unroll
    for (int k = 0; k < 8; k++) s.str[k][w] = out[k];
  }
}

__global__ void __launch_bounds__(kThreads)
k_stepu_ref(DevState s, Params p) {
  const int n = s.na;
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n;
       w += gridDim.x * blockDim.x) {
    if (s.flags[w] & kSkipU) continue;
    const int inw = s.nw[w], isw = s.sw[w], isse = s.sse[w];
    StepuIn in;
    in.uold = s.u[w];
    in.vold = s.v[w];
    in.kvrel = drag_factor(s.aiu[w], p.rhow, s.Cw[w]);
    in.uocn = s.uocn[w];
    in.vocn = s.vocn[w];
    in.waterx = s.waterx[w];
    in.watery = s.watery[w];
    in.forcex = s.forcex[w];
    in.forcey = s.forcey[w];
    in.umassdti = s.umassdti[w];
    in.fm = s.fm[w];
    in.uarear = s.uarear[w];
    in.Tbu = s.Tbu[w];
    in.uinit = s.uinit[w];
    in.vinit = s.vinit[w];
    in.s1 = s.str[0][w];
    in.s2nw = s.str[1][inw];
    in.s3sse = s.str[2][isse];
    in.s4sw = s.str[3][isw];
    in.s5 = s.str[4][w];
    in.s6sse = s.str[5][isse];
    in.s7nw = s.str[6][inw];
    in.s8sw = s.str[7][isw];
    const StepuOut o = stepu_point(in, p);
    s.Cb[w] = o.Cb;
    s.strintx[w] = o.strintx;
    s.strinty[w] = o.strinty;
    s.u[w] = o.u;
    s.v[w] = o.v;
  }
}

int grid_for(int n) {
  int b = (n + kThreads - 1) / kThreads;
  return b < 1 ? 1 : b;
}

}  // namespace

void launch_stress(const DevState &s, const Params &p, cudaStream_t st) {
  if (s.na <= 0) return;
  if (std_params(p))
    k_stress_ref<true><<<grid_for(s.na), kThreads, 0, st>>>(s, p);
  else
    k_stress_ref<false><<<grid_for(s.na), kThreads, 0, st>>>(s, p);
}

void launch_stepu(const DevState &s, const Params &p, cudaStream_t st) {
  if (s.na <= 0) return;
  k_stepu_ref<<<grid_for(s.na), kThreads, 0, st>>>(s, p);
}

}  // namespace evp
