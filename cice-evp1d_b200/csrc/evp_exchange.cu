// evp_exchange.cu -- the velocity exchange of include/evp1d.h
// (evp1d_exchange_*) for one state split over several handles.
//
// A handle's local 1D problem is a band of the global list plus ghost points.
// After every subcycle the ghosts' velocities are stale: the caller packs the
// band's boundary velocities into a device buffer, moves the buffers between
// handles (NCCL send/recv, or device copies when the handles share a GPU) and
// unpacks them into the ghosts' places in the current state.  The kernels
// read and write the slot-ordered state directly: list point i (1-based) is
// at slot_of_point[i-1], halo slot i > na at nslots + (i-1-na).
#include <cstdint>
#include <vector>

#include "evp1d.h"
#include "evp_handle.h"
#include "evp_internal.h"

namespace {

constexpr int kBlock = 256;

int cuda_fail(cudaError_t e, const char *what) {
  return evp::error(e == cudaErrorMemoryAllocation ? EVP1D_ERR_NOMEM : EVP1D_ERR_CUDA,
                    "%s: %s", what, cudaGetErrorString(e));
}

int blocks_for(int n) { return (n + kBlock - 1) / kBlock; }

// 1-based local positions -> device state positions, in place.
__global__ void k_exchange_positions(int n, int na, int nslots,
                                     const int32_t *__restrict__ slot_of_point, int32_t *pos) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = pos[k];
  pos[k] = i <= na ? slot_of_point[i - 1] : nslots + (i - 1 - na);
}

__global__ void k_exchange_pack(int n, const int32_t *__restrict__ pos,
                                const double *__restrict__ u, const double *__restrict__ v,
                                double *buf) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int s = pos[k];
  buf[2 * k] = u[s];
  buf[2 * k + 1] = v[s];
}

__global__ void k_exchange_unpack(int n, const int32_t *__restrict__ pos,
                                  const double *__restrict__ buf, double *u, double *v) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int s = pos[k];
  u[s] = buf[2 * k];
  v[s] = buf[2 * k + 1];
}

int usable(evp1d_t *h) {
  if (!h) return evp::error(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (h->nmembers > 1)
    return evp::error(EVP1D_ERR_STATE, "the velocity exchange is for single-state handles");
  cudaError_t e = cudaSetDevice(h->d.device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  return EVP1D_OK;
}

}  // namespace

namespace evp {
void exchange_release(evp1d_t *h) {
  if (h->xpos) cudaFree(h->xpos);
  h->xpos = nullptr;
  h->xbuf = nullptr;
  h->nsend = h->nrecv = 0;
}
}  // namespace evp

int evp1d_exchange_setup(evp1d_t *h, int n_send, const int32_t *send_idx, int n_recv,
                         const int32_t *recv_idx) {
  int rc = usable(h);
  if (rc != EVP1D_OK) return rc;
  const int na = h->d.na, navel = h->d.navel;
  if (n_send < 0 || n_recv < 0)
    return evp::error(EVP1D_ERR_INVALID_ARG, "n_send = %d, n_recv = %d", n_send, n_recv);
  if ((n_send > 0 && !send_idx) || (n_recv > 0 && !recv_idx))
    return evp::error(EVP1D_ERR_INVALID_ARG, "NULL index array");
  for (int k = 0; k < n_send; k++)
    if (send_idx[k] < 1 || send_idx[k] > na)
      return evp::error(EVP1D_ERR_INVALID_ARG, "send_idx[%d] = %d outside 1..%d", k,
                        send_idx[k], na);
  std::vector<char> seen((size_t)navel + 1, 0);
  for (int k = 0; k < n_recv; k++) {
    const int i = recv_idx[k];
    if (i < 1 || i > navel)
      return evp::error(EVP1D_ERR_INVALID_ARG, "recv_idx[%d] = %d outside 1..%d", k, i, navel);
    if (seen[i]) return evp::error(EVP1D_ERR_INVALID_ARG, "recv_idx repeats %d", i);
    seen[i] = 1;
  }
  evp::exchange_release(h);
  const int n = n_send + n_recv;
  if (n == 0) return EVP1D_OK;
  cudaStream_t st = h->d.stream;
  // one allocation: the positions, then (256-byte aligned) the send and the
  // receive buffer of u, v pairs
  const size_t pos_bytes = (sizeof(int32_t) * (size_t)n + 255) & ~(size_t)255;
  cudaError_t e = evp::device_alloc(&h->xpos, pos_bytes + sizeof(double) * 2 * (size_t)n);
  if (e != cudaSuccess) {
    h->xpos = nullptr;
    return cuda_fail(e, "cudaMalloc");
  }
  h->xbuf = reinterpret_cast<double *>(reinterpret_cast<char *>(h->xpos) + pos_bytes);
  std::vector<int32_t> all((size_t)n);
  for (int k = 0; k < n_send; k++) all[k] = send_idx[k];
  for (int k = 0; k < n_recv; k++) all[n_send + k] = recv_idx[k];
  e = cudaMemcpyAsync(h->xpos, all.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice,
                      st);
  if (e == cudaSuccess) {
    k_exchange_positions<<<blocks_for(n), kBlock, 0, st>>>(n, na, h->d.nslots,
                                                           h->d.slot_of_point, h->xpos);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // `all` is pageable
  if (e != cudaSuccess) {
    evp::exchange_release(h);
    return cuda_fail(e, "exchange setup");
  }
  h->nsend = n_send;
  h->nrecv = n_recv;
  return EVP1D_OK;
}

int evp1d_exchange_pack(evp1d_t *h, double *buf) {
  evp::NvtxRange nvtx_range("evp1d_exchange_pack");
  int rc = usable(h);
  if (rc != EVP1D_OK) return rc;
  if (!h->uploaded) return evp::error(EVP1D_ERR_STATE, "evp1d_upload has not been called");
  if (h->nsend == 0) return EVP1D_OK;
  if (!buf) buf = h->xbuf;
  const int c = h->d.cur;
  k_exchange_pack<<<blocks_for(h->nsend), kBlock, 0, h->d.stream>>>(h->nsend, h->xpos,
                                                                   h->d.u[c], h->d.v[c], buf);
  h->launches++;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? EVP1D_OK : cuda_fail(e, "k_exchange_pack");
}

int evp1d_exchange_unpack(evp1d_t *h, const double *buf) {
  evp::NvtxRange nvtx_range("evp1d_exchange_unpack");
  int rc = usable(h);
  if (rc != EVP1D_OK) return rc;
  if (!h->uploaded) return evp::error(EVP1D_ERR_STATE, "evp1d_upload has not been called");
  if (h->nrecv == 0) return EVP1D_OK;
  if (!buf) buf = h->xbuf + 2 * (size_t)h->nsend;
  const int c = h->d.cur;
  k_exchange_unpack<<<blocks_for(h->nrecv), kBlock, 0, h->d.stream>>>(
      h->nrecv, h->xpos + h->nsend, buf, h->d.u[c], h->d.v[c]);
  h->launches++;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? EVP1D_OK : cuda_fail(e, "k_exchange_unpack");
}

int evp1d_exchange_buffers(evp1d_t *h, double **send, double **recv) {
  int rc = usable(h);
  if (rc != EVP1D_OK) return rc;
  if (!send || !recv) return evp::error(EVP1D_ERR_INVALID_ARG, "NULL argument");
  *send = h->nsend > 0 ? h->xbuf : nullptr;
  *recv = h->nrecv > 0 ? h->xbuf + 2 * (size_t)h->nsend : nullptr;
  return EVP1D_OK;
}
