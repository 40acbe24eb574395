// FFT-filtered complex noise in FP64 (Percival circulant embedding), the GPU
// replacement of noise/hops_noise.py:630-716.  The three length-2(n_t-1)
// transforms are cuFFT Z2Z plans; embedding, clipping, filtering and the
// phase (un)rotation are the kernels below.
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdio.h>
#include <stdarg.h>
#include <mutex>
#include <vector>
#include "hops_common.cuh"

using namespace hops;

void hops_set_error_text(const char* msg);  // defined in hops_rk4.cu
static thread_local char g_nerr[512];

static int nerr(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_nerr, sizeof(g_nerr), fmt, ap);
  va_end(ap);
  hops_set_error_text(g_nerr);
  return code;
}

// Rounded alpha as the reference stores it (complex64, hops_noise.py:236).
__device__ __forceinline__ double2 alpha64(const double* alpha, size_t i) {
  double2 a = reinterpret_cast<const double2*>(alpha)[i];
  return mk((double)(float)a.x, (double)(float)a.y);
}

// nu_l = angle(c[l, n_t-1]) / ((n_t-1) 2 pi): rotation that makes the last sample real.
__device__ __forceinline__ double rot_nu(const double* alpha, int l, int n_t) {
  double2 c = alpha64(alpha, (size_t)l * n_t + (n_t - 1));
  return atan2(c.y, c.x) / ((n_t - 1.0) * 2.0 * 3.14159265358979323846);
}

// exp(-2 pi i nu k)
__device__ __forceinline__ double2 rot(double nu, long k) {
  double sn, cs;
  // reduce nu*k to [0,1) turns before the trig call
  double x = nu * (double)k;
  x -= floor(x);
  sincospi(-2.0 * x, &sn, &cs);
  return mk(cs, sn);
}

// emb[r][k], k < N = 2(n_t-1): rotated correlation function of alpha row
// l = r % n_alpha and its Hermitian mirror.
__global__ void k_embed(const double* alpha, int n_alpha, int n_rows, int n_t, double2* emb) {
  const long N = 2L * (n_t - 1);
  const long total = (long)n_rows * N;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long r = i / N;
    const long k = i - r * N;
    const int l = (int)(r % n_alpha);
    const double nu = rot_nu(alpha, l, n_t);
    double2 v;
    if (k < n_t) {
      v = cmul(alpha64(alpha, (size_t)l * n_t + k), rot(nu, k));
    } else {
      const long kk = N - k;  // 1 .. n_t-2
      v = cconj(cmul(alpha64(alpha, (size_t)l * n_t + kk), rot(nu, kk)));
    }
    emb[i] = v;
  }
}

// z (complex64) -> complex128 work array.
__global__ void k_widen(const float2* z, long total, double2* zw) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x)
    zw[i] = to_d(z[i]);
}

// zw <- zw * sqrt(max(Re(S), 0) / 2); counts clipped spectral values.
__global__ void k_filter(const double2* spec, long total, double2* zw, unsigned long long* nneg) {
  unsigned long long cnt = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    double s = spec[i].x;
    if (s < 0.0) {
      s = 0.0;
      ++cnt;
    }
    zw[i] = cscale(zw[i], sqrt(s / 2.0));
  }
  if (cnt) atomicAdd(nneg, cnt);
}

// out[l][k] = ifft(...)[k] / N * conj(rot(k)), k < n_t; row l unrotated with
// alpha row l % n_alpha.
__global__ void k_unrotate(const double* alpha, int n_alpha, const double2* y, int n_lop,
                           int n_t, double2* out, float2* out64) {
  const long N = 2L * (n_t - 1);
  const long total = (long)n_lop * n_t;
  const double invN = 1.0 / (double)N;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int l = (int)(i / n_t);
    const long k = i - (long)l * n_t;
    const double nu = rot_nu(alpha, l % n_alpha, n_t);
    double2 v = cscale(y[(long)l * N + k], invN);
    v = cmul(v, cconj(rot(nu, k)));
    if (out) out[i] = v;
    if (out64) out64[i] = mkf((float)v.x, (float)v.y);
  }
}

static int grid_for(long n) {
  long b = (n + 255) / 256;
  if (b > 148L * 16) b = 148L * 16;
  if (b < 1) b = 1;
  return (int)b;
}

extern "C" size_t hops_noise_filter_work_doubles(int32_t n_lop, int32_t n_t) {
  return (size_t)4 * n_lop * 2 * (size_t)(n_t - 1) + 2;
}

// Batched Z2Z plans kept for reuse: making a plan costs milliseconds (tens of
// milliseconds for lengths with large prime factors), and an ensemble, the
// trajectories of an adaptive worker or repeated set-ups ask for the same
// (device, length, batch) again.  A plan is lent to one call at a time and
// taken back only after that call has synchronised its stream, so two calls
// never share a plan's work area; at most kPlanKeep idle plans are kept.
namespace {
struct PlanKey {
  int dev, n, batch;
};
struct IdlePlan {
  PlanKey key;
  cufftHandle plan;
};
std::mutex g_plan_mu;
std::vector<IdlePlan> g_plans;
constexpr size_t kPlanKeep = 8;

bool plan_take(int n, int batch, cufftHandle* out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    for (size_t i = 0; i < g_plans.size(); ++i)
      if (g_plans[i].key.dev == dev && g_plans[i].key.n == n && g_plans[i].key.batch == batch) {
        *out = g_plans[i].plan;
        g_plans.erase(g_plans.begin() + (long)i);
        return true;
      }
  }
  return cufftPlan1d(out, n, CUFFT_Z2Z, batch) == CUFFT_SUCCESS;
}

// `synced`: the call's work on the plan has completed.
void plan_give(int n, int batch, cufftHandle plan, bool synced) {
  int dev = 0;
  if (synced && cudaGetDevice(&dev) == cudaSuccess) {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    g_plans.push_back({{dev, n, batch}, plan});
    if (g_plans.size() <= kPlanKeep) return;
    plan = g_plans.front().plan;  // the oldest idle plan goes
    g_plans.erase(g_plans.begin());
  }
  cufftDestroy(plan);
}
}  // namespace

extern "C" int hops_noise_filter_shared(const double* alpha_dev, int32_t n_alpha,
                                        const float* z_dev, int32_t n_rows, int32_t n_t,
                                        double* work_dev, double* out_dev, float* out64_dev,
                                        int64_t* n_negative_host, void* stream) {
  if (!alpha_dev || !z_dev || !work_dev || n_alpha <= 0 || n_rows <= 0 || n_rows % n_alpha ||
      n_t < 3)
    return nerr(HOPS_EINVAL, "hops_noise_filter: bad arguments (n_alpha=%d n_rows=%d n_t=%d)",
                n_alpha, n_rows, n_t);
  cudaStream_t s = (cudaStream_t)stream;
  const int N = 2 * (n_t - 1);
  const long total = (long)n_rows * N;
  double2* emb = reinterpret_cast<double2*>(work_dev);
  double2* zw = emb + total;
  unsigned long long* nneg = reinterpret_cast<unsigned long long*>(zw + total);
  cufftHandle plan;
  if (!plan_take(N, n_rows, &plan))
    return nerr(HOPS_ECUDA, "cufftPlan1d(%d, batch %d) failed", N, n_rows);
  int rc = HOPS_OK;
  bool synced = false;
  do {
    if (cufftSetStream(plan, s) != CUFFT_SUCCESS) { rc = nerr(HOPS_ECUDA, "cufftSetStream failed"); break; }
    if (cudaMemsetAsync(nneg, 0, sizeof(unsigned long long), s) != cudaSuccess) {
      rc = nerr(HOPS_ECUDA, "memset failed");
      break;
    }
    // every row's embedding from its alpha row: one batched plan serves all
    // three transforms
    k_embed<<<grid_for(total), 256, 0, s>>>(alpha_dev, n_alpha, n_rows, n_t, emb);
    if (cufftExecZ2Z(plan, (cufftDoubleComplex*)emb, (cufftDoubleComplex*)emb, CUFFT_FORWARD) != CUFFT_SUCCESS) {
      rc = nerr(HOPS_ECUDA, "cufftExecZ2Z (embedding) failed");
      break;
    }
    k_widen<<<grid_for(total), 256, 0, s>>>(reinterpret_cast<const float2*>(z_dev), total, zw);
    if (cufftExecZ2Z(plan, (cufftDoubleComplex*)zw, (cufftDoubleComplex*)zw, CUFFT_FORWARD) != CUFFT_SUCCESS) {
      rc = nerr(HOPS_ECUDA, "cufftExecZ2Z (noise) failed");
      break;
    }
    k_filter<<<grid_for(total), 256, 0, s>>>(emb, total, zw, nneg);
    if (cufftExecZ2Z(plan, (cufftDoubleComplex*)zw, (cufftDoubleComplex*)zw, CUFFT_INVERSE) != CUFFT_SUCCESS) {
      rc = nerr(HOPS_ECUDA, "cufftExecZ2Z (inverse) failed");
      break;
    }
    k_unrotate<<<grid_for((long)n_rows * n_t), 256, 0, s>>>(alpha_dev, n_alpha, zw, n_rows, n_t,
                                                            reinterpret_cast<double2*>(out_dev),
                                                            reinterpret_cast<float2*>(out64_dev));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      rc = nerr(HOPS_ECUDA, "noise filter launch: %s", cudaGetErrorString(e));
      break;
    }
    if (n_negative_host) {
      unsigned long long h = 0;
      if (cudaMemcpyAsync(&h, nneg, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        rc = nerr(HOPS_ECUDA, "reading the clip count failed");
        break;
      }
      synced = true;
      *n_negative_host = (int64_t)h;
    }
  } while (0);
  plan_give(N, n_rows, plan, synced);
  return rc;
}

extern "C" int hops_noise_filter(const double* alpha_dev, const float* z_dev, int32_t n_lop,
                                 int32_t n_t, double* work_dev, double* out_dev, float* out64_dev,
                                 int64_t* n_negative_host, void* stream) {
  return hops_noise_filter_shared(alpha_dev, n_lop, z_dev, n_lop, n_t, work_dev, out_dev,
                                  out64_dev, n_negative_host, stream);
}

// ------------------------------------------------ effective-noise windows ----
// EFFECTIVE_NOISE_INTEGRATION (integrator/integrator_rk.py:115-128) replaces
// the noise samples at t, t + tau/2, t + tau by the means of three windows of
// k = tau / (2 TAU) consecutive complex64 samples.  The reference takes them
// with numpy's mean, so the sums follow numpy's pairwise summation exactly:
// fewer than 8 floats added in order, up to 128 floats in 8 running partial
// sums (for complex data: 4 complex partials) combined as ((0+1)+(2+3)) +
// ((4+5)+(6+7)) with the tail added in order, larger blocks split in halves
// rounded down to 8 floats; then each component is divided by k in single
// precision.  With real_only (FLAG_REAL noise: numpy sums the float32 real
// parts alone) the real parts use the float32 form of the same scheme.
__device__ void pw_complex(const float2* a, int m, float& rr, float& ri) {
  const int n = 2 * m;
  if (n < 8) {
    rr = -0.0f;
    ri = -0.0f;
    for (int i = 0; i < m; ++i) {
      rr = __fadd_rn(rr, a[i].x);
      ri = __fadd_rn(ri, a[i].y);
    }
    return;
  }
  if (n <= 128) {
    float r[8] = {a[0].x, a[0].y, a[1].x, a[1].y, a[2].x, a[2].y, a[3].x, a[3].y};
    int i = 4;
    for (; i + 4 <= m; i += 4) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        r[2 * j] = __fadd_rn(r[2 * j], a[i + j].x);
        r[2 * j + 1] = __fadd_rn(r[2 * j + 1], a[i + j].y);
      }
    }
    rr = __fadd_rn(__fadd_rn(r[0], r[2]), __fadd_rn(r[4], r[6]));
    ri = __fadd_rn(__fadd_rn(r[1], r[3]), __fadd_rn(r[5], r[7]));
    for (; i < m; ++i) {
      rr = __fadd_rn(rr, a[i].x);
      ri = __fadd_rn(ri, a[i].y);
    }
    return;
  }
  int n2 = n / 2;
  n2 -= n2 % 8;
  const int m2 = n2 / 2;
  float r1, i1, r2, i2;
  pw_complex(a, m2, r1, i1);
  pw_complex(a + m2, m - m2, r2, i2);
  rr = __fadd_rn(r1, r2);
  ri = __fadd_rn(i1, i2);
}

// Real parts a[i].x, i < n, as numpy sums a float32 row.
__device__ float pw_real(const float2* a, int n) {
  if (n < 8) {
    float r = -0.0f;
    for (int i = 0; i < n; ++i) r = __fadd_rn(r, a[i].x);
    return r;
  }
  if (n <= 128) {
    float r[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) r[j] = a[j].x;
    int i = 8;
    for (; i + 8 <= n; i += 8) {
#pragma unroll
      for (int j = 0; j < 8; ++j) r[j] = __fadd_rn(r[j], a[i + j].x);
    }
    float s = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                        __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
    for (; i < n; ++i) s = __fadd_rn(s, a[i].x);
    return s;
  }
  int n2 = n / 2;
  n2 -= n2 % 8;
  return __fadd_rn(pw_real(a, n2), pw_real(a + n2, n - n2));
}

// out[r][w] = mean(in[r][start + w k .. start + (w+1) k - 1]), w < n_out.
__global__ void k_window_mean(const float2* in, long rows, int n_t, int start, int k, int n_out,
                              int real_only, float2* out) {
  const long total = rows * (long)n_out;
  const float fk = (float)k;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total;
       q += (long)gridDim.x * blockDim.x) {
    const long r = q / n_out;
    const int w = (int)(q - r * n_out);
    const float2* a = in + r * n_t + start + (long)w * k;
    float sr, si = 0.0f;
    if (real_only)
      sr = pw_real(a, k);
    else
      pw_complex(a, k, sr, si);
    out[q] = make_float2(__fdiv_rn(sr, fk), real_only ? 0.0f : __fdiv_rn(si, fk));
  }
}

extern "C" int hops_noise_window_mean(const float* noise_dev, int64_t rows, int32_t n_t,
                                      int32_t start, int32_t k, int32_t n_out,
                                      int32_t real_only, float* out_dev, void* stream) {
  if (!noise_dev || !out_dev || rows < 0 || n_t <= 0 || start < 0 || k < 1 || n_out < 0 ||
      (int64_t)start + (int64_t)n_out * k > n_t)
    return nerr(HOPS_EINVAL, "hops_noise_window_mean: windows [%d, %d + %d*%d) outside %d samples",
                start, start, n_out, k, n_t);
  if (rows == 0 || n_out == 0) return HOPS_OK;
  const long total = rows * (long)n_out;
  k_window_mean<<<grid_for(total), 128, 0, (cudaStream_t)stream>>>(
      reinterpret_cast<const float2*>(noise_dev), rows, n_t, start, k, n_out, real_only,
      reinterpret_cast<float2*>(out_dev));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return nerr(HOPS_ECUDA, "window mean launch: %s", cudaGetErrorString(e));
  return HOPS_OK;
}
