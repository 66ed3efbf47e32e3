// sort.cu -- device scan and stable LSD radix sort used by the scene builder
// (Morton-ordered LBVH leaves, half-edge grouping for the edge list).
#include "psdr_internal.h"

namespace psdr {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;  // elements per thread per block
constexpr int kScanBlock = kScanThreads * kScanPer;

template <class T>
__device__ T block_exclusive_scan(T v, T* smem_warp, T& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    T w = lane < nw ? smem_warp[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) smem_warp[lane] = w;
  }
  __syncthreads();
  T base = wid > 0 ? smem_warp[wid - 1] : T(0);
  total = smem_warp[(blockDim.x >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

template <class T>
__global__ void k_reduce(const T* __restrict__ in, int n, T* __restrict__ sums) {
  __shared__ T sw[32];
  const int base = blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
  T acc = T(0);
#pragma unroll
  for (int k = 0; k < kScanPer; ++k)
    if (base + k < n) acc += in[base + k];
  T tot;
  block_exclusive_scan<T>(acc, sw, tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Single block: exclusive scan of `n` block sums in place (n <= kScanBlock * 64).
template <class T>
__global__ void k_scan_sums(T* data, int n) {
  __shared__ T sw[32];
  T carry = T(0);
  for (int start = 0; start < n; start += kScanBlock) {
    const int base = start + threadIdx.x * kScanPer;
    T loc[kScanPer];
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
      loc[k] = base + k < n ? data[base + k] : T(0);
      acc += loc[k];
    }
    T tot;
    T ex = block_exclusive_scan<T>(acc, sw, tot);
    T run = carry + ex;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
      if (base + k < n) data[base + k] = run;
      run += loc[k];
    }
    carry += tot;
    __syncthreads();
  }
}

template <class T, bool INCL>
__global__ void k_scan_apply(const T* __restrict__ in, T* __restrict__ out, int n, const T* __restrict__ offs) {
  __shared__ T sw[32];
  const int base = blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
  T loc[kScanPer];
  T acc = T(0);
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    loc[k] = base + k < n ? in[base + k] : T(0);
    acc += loc[k];
  }
  T tot;
  T run = offs[blockIdx.x] + block_exclusive_scan<T>(acc, sw, tot);
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    if (INCL) run += loc[k];
    if (base + k < n) out[base + k] = run;
    if (!INCL) run += loc[k];
  }
}

template <class T, bool INCL>
void scan_impl(const T* in, T* out, int n, T* tmp, cudaStream_t st) {
  if (n <= 0) return;
  const int nb = (n + kScanBlock - 1) / kScanBlock;
  k_reduce<T><<<nb, kScanThreads, 0, st>>>(in, n, tmp);
  k_scan_sums<T><<<1, kScanThreads, 0, st>>>(tmp, nb);
  k_scan_apply<T, INCL><<<nb, kScanThreads, 0, st>>>(in, out, n, tmp);
  PSDR_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------- radix sort
constexpr int kSortThreads = 256;
constexpr int kSortChunk = 4096;  // elements per block

__global__ void k_hist(const uint64_t* __restrict__ keys, int n, int shift, int* __restrict__ hist, int nb) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int lo = blockIdx.x * kSortChunk, hi = min(n, lo + kSortChunk);
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&h[(keys[i] >> shift) & 255u], 1);
  __syncthreads();
  hist[threadIdx.x * nb + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: each block walks its chunk in order, 256 elements at a time; ranks
// among equal digits come from warp match + per-warp digit counts.
__global__ void k_scatter(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                          uint64_t* __restrict__ kout, uint32_t* __restrict__ vout, int n, int shift,
                          const int* __restrict__ hist, int nb) {
  __shared__ int offs[256];
  __shared__ int wcnt[8][256];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  offs[threadIdx.x] = hist[threadIdx.x * nb + blockIdx.x];
  for (int w = 0; w < 8; ++w) wcnt[w][threadIdx.x] = 0;
  __syncthreads();
  const int lo = blockIdx.x * kSortChunk, hi = min(n, lo + kSortChunk);
  for (int base = lo; base < hi; base += kSortThreads) {
    const int i = base + threadIdx.x;
    const bool ok = i < hi;
    uint64_t key = ok ? kin[i] : 0;
    uint32_t val = ok ? vin[i] : 0;
    const uint32_t dig = ok ? (uint32_t)((key >> shift) & 255u) : 256u + (uint32_t)wid;
    const uint32_t peers = __match_any_sync(0xffffffffu, dig);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    const int leader = __ffs(peers) - 1;
    if (ok && lane == leader) wcnt[wid][dig] = __popc(peers);
    __syncthreads();
    // per digit: exclusive prefix over warps
    {
      const int d = threadIdx.x;
      int run = 0;
      for (int w = 0; w < 8; ++w) {
        int c = wcnt[w][d];
        wcnt[w][d] = run;
        run += c;
      }
      __syncthreads();
      if (ok) {
        const int pos = offs[dig] + wcnt[wid][dig] + rank;
        kout[pos] = key;
        vout[pos] = val;
      }
      __syncthreads();
      offs[d] += run;
      for (int w = 0; w < 8; ++w) wcnt[w][d] = 0;
      __syncthreads();
    }
  }
}

}  // namespace

size_t scan_tmp_ints(int n) { return (size_t)((n + kScanBlock - 1) / kScanBlock + 1); }
size_t scan_tmp_doubles(int n) { return scan_tmp_ints(n); }

void exclusive_scan_int(const int* in, int* out, int n, int* tmp, cudaStream_t st) {
  scan_impl<int, false>(in, out, n, tmp, st);
}
void inclusive_scan_double(const double* in, double* out, int n, double* tmp, cudaStream_t st) {
  scan_impl<double, true>(in, out, n, tmp, st);
}

void radix_sort_pairs(uint64_t* keys, uint32_t* vals, int n, int bits, SortTmp& tmp, cudaStream_t st) {
  if (n <= 1) return;
  const int nb = (n + kSortChunk - 1) / kSortChunk;
  tmp.keys2.alloc(sizeof(uint64_t) * n, st);
  tmp.vals2.alloc(sizeof(uint32_t) * n, st);
  tmp.hist.alloc(sizeof(int) * (256 * (size_t)nb + scan_tmp_ints(256 * nb)), st);
  int* hist = tmp.hist.as<int>();
  int* hscan_tmp = hist + 256 * (size_t)nb;
  uint64_t* ka = keys;
  uint32_t* va = vals;
  uint64_t* kb = tmp.keys2.as<uint64_t>();
  uint32_t* vb = tmp.vals2.as<uint32_t>();
  int passes = (bits + 7) / 8;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    k_hist<<<nb, 256, 0, st>>>(ka, n, shift, hist, nb);
    exclusive_scan_int(hist, hist, 256 * nb, hscan_tmp, st);
    k_scatter<<<nb, kSortThreads, 0, st>>>(ka, va, kb, vb, n, shift, hist, nb);
    PSDR_CUDA(cudaGetLastError());
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    PSDR_CUDA(cudaMemcpyAsync(keys, ka, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, st));
    PSDR_CUDA(cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
  }
}

}  // namespace psdr
