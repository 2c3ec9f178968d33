// Segmented dot products for the device SCF tail: per output slot, the sums over its segments
// of products of up to four packed FP64 vectors (x_i * x_j, or x_i alone).
//
// The SCF tail of many molecules reduces packed arrays (every molecule's nbf x nbf blocks back
// to back) per molecule: the density-DIIS matrix B_xy = sum d_x . d_y of the last four residuals
// (conv_diis4, reference src/conv.c:606-844), the RMS density change, and the energy.  An
// index_add_ of every element into its molecule's slot is one FP64 atomic per element, all on a
// few hundred addresses; here each CTA reduces one chunk of one segment for all products at once
// (one pass over HBM for the ten B entries), writes its partial sums, and a second kernel adds
// each slot's partials in chunk order, so the result does not depend on scheduling.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/sqb200.h"

namespace sqb {
int set_error(int code, const std::string& msg);   // jk_engine.cu
}

namespace {

constexpr int kChunk = 16384;       // elements per CTA
constexpr int kThreads = 256;
constexpr int kMaxVec = 4, kMaxPair = 10;

struct Chunk { long long start; int len; int slot; };

struct Vecs {
  const double* v[kMaxVec];
  int pi[kMaxPair], pj[kMaxPair];   // product pi * pj; pj < 0: pi alone
  int npair;
};

template <int NP>
__global__ void __launch_bounds__(kThreads) k_seg_partial(Vecs a, const Chunk* __restrict__ chunks,
                                                          double* __restrict__ partial) {
  const Chunk c = chunks[blockIdx.x];
  double acc[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) acc[p] = 0.0;
  const double *v0 = a.v[0], *v1 = a.v[1], *v2 = a.v[2], *v3 = a.v[3];
  for (int e = threadIdx.x; e < c.len; e += kThreads) {
    const long long g = c.start + e;
    const double x0 = __ldg(v0 + g);
    const double x1 = v1 ? __ldg(v1 + g) : 0.0;
    const double x2 = v2 ? __ldg(v2 + g) : 0.0;
    const double x3 = v3 ? __ldg(v3 + g) : 0.0;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const int i = a.pi[p], j = a.pj[p];
      const double xi = i == 0 ? x0 : i == 1 ? x1 : i == 2 ? x2 : x3;
      const double xj = j < 0 ? 1.0 : j == 0 ? x0 : j == 1 ? x1 : j == 2 ? x2 : x3;
      acc[p] = fma(xi, xj, acc[p]);
    }
  }
  __shared__ double red[kThreads / 32][NP];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    double v = acc[p];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][p] = v;
  }
  __syncthreads();
  if (threadIdx.x < NP) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) v += red[w][threadIdx.x];
    partial[(size_t)blockIdx.x * NP + threadIdx.x] = v;
  }
}

// out[slot * npair + p] = sum over the slot's chunks, in chunk order, of partial[chunk][p]
__global__ void k_seg_final(const double* __restrict__ partial, const int* __restrict__ slot_first, int nslot,
                            int npair, double* __restrict__ out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nslot * npair) return;
  const int s = idx / npair, p = idx - s * npair;
  double v = 0.0;
  for (int c = slot_first[s]; c < slot_first[s + 1]; ++c) v += partial[(size_t)c * npair + p];
  out[idx] = v;
}

}  // namespace

struct sqb200_segdots {
  int device = 0, nslot = 0, nchunk = 0;
  Chunk* d_chunks = nullptr;
  int* d_slot_first = nullptr;
  double* d_partial = nullptr;   // nchunk x kMaxPair
  void* d_base = nullptr;
};

extern "C" {

int sqb200_segdots_create(sqb200_segdots** out, int device, int nseg, const long long* seg_start,
                          const long long* seg_len, const int* seg_slot, int nslot) {
  if (!out || nseg < 0 || nslot <= 0 || (nseg > 0 && (!seg_start || !seg_len || !seg_slot)))
    return sqb::set_error(SQB200_EINVAL, "sqb200_segdots_create: null argument or no slot");
  *out = nullptr;
  std::vector<int> order(nseg);
  for (int s = 0; s < nseg; ++s) {
    if (seg_slot[s] < 0 || seg_slot[s] >= nslot || seg_len[s] < 0 || seg_start[s] < 0)
      return sqb::set_error(SQB200_EINVAL, "sqb200_segdots_create: bad segment");
    order[s] = s;
  }
  // chunks grouped by slot, segments of a slot in the caller's order
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return seg_slot[a] < seg_slot[b]; });
  std::vector<Chunk> ch;
  std::vector<int> first(nslot + 1, 0);
  for (int s : order) {
    for (long long o = 0; o < seg_len[s]; o += kChunk)
      ch.push_back({seg_start[s] + o, (int)std::min<long long>(kChunk, seg_len[s] - o), seg_slot[s]});
  }
  for (const Chunk& c : ch) first[c.slot + 1] += 1;
  for (int s = 0; s < nslot; ++s) first[s + 1] += first[s];
  if (cudaSetDevice(device) != cudaSuccess) return sqb::set_error(SQB200_ECUDA, "sqb200_segdots_create: cudaSetDevice");
  sqb200_segdots* p = new sqb200_segdots();
  p->device = device;
  p->nslot = nslot;
  p->nchunk = (int)ch.size();
  const size_t bc = std::max<size_t>(1, ch.size()) * sizeof(Chunk);
  const size_t bf = (nslot + 1) * sizeof(int);
  const size_t bp = std::max<size_t>(1, ch.size()) * kMaxPair * sizeof(double);
  const size_t oc = 0, of = (bc + 255) / 256 * 256, op = of + (bf + 255) / 256 * 256;
  if (cudaMalloc(&p->d_base, op + bp) != cudaSuccess) {
    delete p;
    return sqb::set_error(SQB200_ENOMEM, "sqb200_segdots_create: cudaMalloc");
  }
  p->d_chunks = (Chunk*)((char*)p->d_base + oc);
  p->d_slot_first = (int*)((char*)p->d_base + of);
  p->d_partial = (double*)((char*)p->d_base + op);
  // the copies land before this returns (pageable memory, then a synchronised stream)
  cudaStream_t st = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess && !ch.empty())
    e = cudaMemcpyAsync(p->d_chunks, ch.data(), ch.size() * sizeof(Chunk), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p->d_slot_first, first.data(), bf, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    cudaFree(p->d_base);
    delete p;
    return sqb::set_error(SQB200_ECUDA, std::string("sqb200_segdots_create: ") + cudaGetErrorString(e));
  }
  *out = p;
  return SQB200_OK;
}

int sqb200_segdots_run(sqb200_segdots* p, int nvec, const double* const* vecs, int npair, const int* pair_i,
                       const int* pair_j, double* out, void* stream) {
  if (!p || nvec < 1 || nvec > kMaxVec || !vecs || npair < 1 || npair > kMaxPair || !pair_i || !pair_j || !out)
    return sqb::set_error(SQB200_EINVAL, "sqb200_segdots_run: bad argument");
  Vecs a;
  for (int k = 0; k < kMaxVec; ++k) a.v[k] = k < nvec ? vecs[k] : nullptr;
  for (int k = 0; k < nvec; ++k)
    if (!a.v[k]) return sqb::set_error(SQB200_EINVAL, "sqb200_segdots_run: null vector");
  for (int q = 0; q < kMaxPair; ++q) { a.pi[q] = 0; a.pj[q] = -1; }
  for (int q = 0; q < npair; ++q) {
    if (pair_i[q] < 0 || pair_i[q] >= nvec || pair_j[q] >= nvec)
      return sqb::set_error(SQB200_EINVAL, "sqb200_segdots_run: bad vector index");
    a.pi[q] = pair_i[q];
    a.pj[q] = pair_j[q] < 0 ? -1 : pair_j[q];
  }
  a.npair = npair;
  if (cudaSetDevice(p->device) != cudaSuccess) return sqb::set_error(SQB200_ECUDA, "sqb200_segdots_run: cudaSetDevice");
  cudaStream_t st = (cudaStream_t)stream;
  if (p->nchunk > 0) {
    switch (npair) {
#define SQB_SEG_CASE(N) \
      case N: k_seg_partial<N><<<p->nchunk, kThreads, 0, st>>>(a, p->d_chunks, p->d_partial); break;
      SQB_SEG_CASE(1) SQB_SEG_CASE(2) SQB_SEG_CASE(3) SQB_SEG_CASE(4) SQB_SEG_CASE(5)
      SQB_SEG_CASE(6) SQB_SEG_CASE(7) SQB_SEG_CASE(8) SQB_SEG_CASE(9) SQB_SEG_CASE(10)
#undef SQB_SEG_CASE
    }
  }
  const int tot = p->nslot * npair;
  k_seg_final<<<(tot + 127) / 128, 128, 0, st>>>(p->d_partial, p->d_slot_first, p->nslot, npair, out);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SQB200_OK
                          : sqb::set_error(SQB200_ECUDA, std::string("sqb200_segdots_run: ") + cudaGetErrorString(e));
}

int sqb200_segdots_destroy(sqb200_segdots* p) {
  if (!p) return SQB200_OK;
  cudaSetDevice(p->device);
  cudaFree(p->d_base);
  delete p;
  return SQB200_OK;
}

}  // extern "C"
