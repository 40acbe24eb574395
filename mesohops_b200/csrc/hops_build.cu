// Structure builder for full triangular hierarchies on the GPU.
//
// The aux of a triangular hierarchy over M modes and depth <= D are the
// multisets of modes of size <= D, ordered by size and then lexicographically
// by their sorted mode tuple (the order of basis/hops_hierarchy.py:340-368 and
// the id sort of basis/hops_aux.py:171-201,460-480).  A size-k tuple
// t_0 <= ... <= t_{k-1} is the k-combination c_i = t_i + i of M + k - 1
// elements, so its place in the order is the combinatorial-number-system rank
// of c plus the count of smaller multisets, C(M + k - 1, k - 1).  Every aux is
// unranked and every connection ranked independently, one thread each, which
// replaces the host-side construction of the hierarchy connections
// (hops_hierarchy.py:470-523) and of K2_k (eom_hops_ksuper.py:36-90).
//
// binom: int64 table C(n, j) for n <= M + D + 1, j <= D + 1, row stride D + 2.
#include <cuda_runtime.h>
#include <stdint.h>
#include "hops_common.cuh"

using namespace hops;

void hops_set_error_text(const char* msg);

namespace {

constexpr int kTriMaxDepth = 16;

struct Tri {
  int M, D, stride;
  const int64_t* B;
  __device__ int64_t C(int n, int j) const {
    return (n < 0 || j < 0 || j > n) ? 0 : B[(size_t)n * stride + j];
  }
  // number of aux with depth < k
  __device__ int64_t off(int k) const { return k == 0 ? 0 : C(M + k - 1, k - 1); }
  // global index -> (depth, sorted tuple)
  __device__ int unrank(int64_t g, int* t) const {
    int k = 0;
    while (k < D && g >= off(k + 1)) ++k;
    int64_t r = g - off(k);
    const int n = M + k - 1;
    int prev = -1;
    for (int i = 0; i < k; ++i) {
      int v = prev + 1;
      for (; v < n; ++v) {
        const int64_t cnt = C(n - 1 - v, k - 1 - i);
        if (r < cnt) break;
        r -= cnt;
      }
      t[i] = min(v - i, M - 1);  // v < n for every index below the aux count
      prev = v;
    }
    return k;
  }
  // sorted tuple of size k -> global index
  __device__ int64_t rank(const int* t, int k) const {
    if (k == 0) return 0;
    const int n = M + k - 1;
    int64_t r = 0;
    int prev = -1;
    for (int i = 0; i < k; ++i) {
      const int b = t[i] + i;
      r += C(n - 1 - prev, k - i) - C(n - b, k - i);
      prev = b;
    }
    return off(k) + r;
  }
};

// k_decay[g] = -sum_i w[t_i] (complex) and the number of distinct modes of g
__global__ void k_tri_pass1(Tri tri, int64_t N, const double* w, double* k_decay,
                            int32_t* dn_count) {
  int t[kTriMaxDepth];
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < N;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int k = tri.unrank(g, t);
    double re = 0.0, im = 0.0;
    int distinct = 0;
    for (int i = 0; i < k; ++i) {
      re -= w[2 * t[i]];
      im -= w[2 * t[i] + 1];
      if (i == 0 || t[i] != t[i - 1]) ++distinct;
    }
    k_decay[2 * g] = re;
    k_decay[2 * g + 1] = im;
    dn_count[g] = distinct;
  }
}

// up connections of the aux below the truncation depth: (g, m) -> g + e_m
__global__ void k_tri_up(Tri tri, int64_t n_below, int32_t* up_aux, int32_t* up_mode) {
  int t[kTriMaxDepth + 1], u[kTriMaxDepth + 1];
  const int64_t total = n_below * tri.M;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = q / tri.M;
    const int m = (int)(q - g * tri.M);
    const int k = tri.unrank(g, t);
    int j = 0, i = 0;
    while (i < k && t[i] <= m) u[j++] = t[i++];
    u[j++] = m;
    while (i < k) u[j++] = t[i++];
    up_aux[q] = (int32_t)tri.rank(u, k + 1);
    up_mode[q] = m;
  }
}

// down connections: for each distinct mode m of g (increasing), g - e_m and
// the depth k_m(g) of g in m
__global__ void k_tri_dn(Tri tri, int64_t N, const int32_t* dn_ptr, int32_t* dn_aux,
                         int32_t* dn_mode, int32_t* dn_k) {
  int t[kTriMaxDepth], u[kTriMaxDepth];
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < N;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int k = tri.unrank(g, t);
    int p = dn_ptr[g];
    for (int i = 0; i < k; ++i) {
      if (i > 0 && t[i] == t[i - 1]) continue;
      const int m = t[i];
      int cnt = 0;
      for (int l = i; l < k && t[l] == m; ++l) ++cnt;
      int j = 0;
      for (int l = 0; l < k; ++l)
        if (l != i) u[j++] = t[l];
      dn_aux[p] = (int32_t)tri.rank(u, k - 1);
      dn_mode[p] = m;
      dn_k[p] = cnt;
      ++p;
    }
  }
}

int tri_check(int32_t n_mode, int32_t depth, const int64_t* binom) {
  if (n_mode < 1 || depth < 0 || depth > kTriMaxDepth || !binom) {
    hops_set_error_text("hops_tri: need n_mode >= 1, 0 <= depth <= 16 and a binomial table");
    return HOPS_EINVAL;
  }
  return HOPS_OK;
}

int grid_of(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

extern "C" int32_t hops_tri_max_depth(void) { return kTriMaxDepth; }

extern "C" int hops_tri_pass1(int32_t n_mode, int32_t depth, const int64_t* binom_dev,
                              int64_t n_hier, const double* w_dev, double* k_decay_dev,
                              int32_t* dn_count_dev, void* stream) {
  int rc = tri_check(n_mode, depth, binom_dev);
  if (rc) return rc;
  if (n_hier <= 0 || !w_dev || !k_decay_dev || !dn_count_dev) {
    hops_set_error_text("hops_tri_pass1: bad arguments");
    return HOPS_EINVAL;
  }
  const Tri tri{n_mode, depth, depth + 2, binom_dev};
  k_tri_pass1<<<grid_of(n_hier), 256, 0, (cudaStream_t)stream>>>(tri, n_hier, w_dev, k_decay_dev,
                                                                 dn_count_dev);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    hops_set_error_text(cudaGetErrorString(e));
    return HOPS_ECUDA;
  }
  return HOPS_OK;
}

extern "C" int hops_tri_pass2(int32_t n_mode, int32_t depth, const int64_t* binom_dev,
                              int64_t n_hier, int64_t n_below, const int32_t* dn_ptr_dev,
                              int32_t* up_aux_dev, int32_t* up_mode_dev, int32_t* dn_aux_dev,
                              int32_t* dn_mode_dev, int32_t* dn_k_dev, void* stream) {
  int rc = tri_check(n_mode, depth, binom_dev);
  if (rc) return rc;
  if (n_hier <= 0 || n_below < 0 || !dn_ptr_dev ||
      (n_below > 0 && (!up_aux_dev || !up_mode_dev)) ||
      (n_hier > 1 && (!dn_aux_dev || !dn_mode_dev || !dn_k_dev))) {
    hops_set_error_text("hops_tri_pass2: bad arguments");
    return HOPS_EINVAL;
  }
  const Tri tri{n_mode, depth, depth + 2, binom_dev};
  cudaStream_t s = (cudaStream_t)stream;
  if (n_below > 0)
    k_tri_up<<<grid_of(n_below * n_mode), 256, 0, s>>>(tri, n_below, up_aux_dev, up_mode_dev);
  if (n_hier > 1)
    k_tri_dn<<<grid_of(n_hier), 256, 0, s>>>(tri, n_hier, dn_ptr_dev, dn_aux_dev, dn_mode_dev,
                                             dn_k_dev);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    hops_set_error_text(cudaGetErrorString(e));
    return HOPS_ECUDA;
  }
  return HOPS_OK;
}
