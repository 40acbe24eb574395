// B200 kernels of the HOPS trajectory hot path: batched RK4 over the auxiliary
// hierarchy (streaming stage kernels) and the resident one-CTA-per-trajectory
// propagator.  See hops_b200.h for the C ABI and the reference functions each
// entry point replaces.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <stdarg.h>
#include <algorithm>
#include "hops_common.cuh"

using namespace hops;

// ------------------------------------------------------------ error state ----
static thread_local char g_err[512] = "";

static int set_err(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

#define CUDA_TRY(expr)                                                        \
  do {                                                                        \
    cudaError_t e_ = (expr);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return set_err(HOPS_ECUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                     __FILE__, __LINE__);                                     \
  } while (0)

#define LAUNCH_CHECK()                                                        \
  do {                                                                        \
    cudaError_t e_ = cudaGetLastError();                                      \
    if (e_ != cudaSuccess)                                                    \
      return set_err(HOPS_ECUDA, "kernel launch: %s (%s:%d)",                 \
                     cudaGetErrorString(e_), __FILE__, __LINE__);             \
  } while (0)

extern "C" const char* hops_last_error(void) { return g_err; }
void hops_set_error_text(const char* msg) { snprintf(g_err, sizeof(g_err), "%s", msg); }
extern "C" int hops_version(void) { return 10000; }

extern "C" int hops_device_query(int device, int* sm_count, int* smem_optin) {
  CUDA_TRY(cudaDeviceGetAttribute(sm_count, cudaDevAttrMultiProcessorCount, device));
  CUDA_TRY(cudaDeviceGetAttribute(smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  return HOPS_OK;
}

extern "C" size_t hops_scalar_workspace_doubles(int32_t S, int32_t M, int32_t L, int32_t B) {
  ScalarLayout lay(S, M, L);
  return (size_t)lay.stride * (size_t)B;
}

// ------------------------------------------------------------- precision ----
template <typename R> struct Prec;
template <> struct Prec<double> {
  using T = double2;
  static __device__ __forceinline__ T kdec(const hops_structure& st, int a) { return ld2(st.k_decay, a); }
  static __device__ __forceinline__ T dncoef(const hops_structure& st, int p) { return ld2(st.dn_coef, p); }
  static __device__ __forceinline__ T gw(const hops_structure& st, int m) { return ld2(st.mode_gw, m); }
  static __device__ __forceinline__ T lval(const hops_structure& st, int q) { return ld2(st.l_val, q); }
  static __device__ __forceinline__ T lhval(const hops_structure& st, int q) { return ld2(st.lh_val, q); }
  static __device__ __forceinline__ T hval(const hops_structure& st, int q) { return ld2(st.h_val, q); }
  static __device__ __forceinline__ T sval(const hops_structure& st, int j) { return ld2(st.lop_sval, j); }
  static __device__ __forceinline__ T diag(const double* ws, const ScalarLayout& l, int s) { return ld2(ws + l.diagD(), s); }
  static __device__ __forceinline__ T upc(const double* ws, const ScalarLayout& l, int m) { return ld2(ws + l.upc(), m); }
  static __device__ __forceinline__ T cz(const double* ws, const ScalarLayout& l, int j) { return ld2(ws + l.cz(), j); }
};
template <> struct Prec<float> {
  using T = float2;
  static __device__ __forceinline__ T kdec(const hops_structure& st, int a) { return ld2f(st.k_decay_f, a); }
  static __device__ __forceinline__ T dncoef(const hops_structure& st, int p) { return ld2f(st.dn_coef_f, p); }
  static __device__ __forceinline__ T gw(const hops_structure& st, int m) { return ld2f(st.mode_gw_f, m); }
  static __device__ __forceinline__ T lval(const hops_structure& st, int q) { return ld2f(st.l_val_f, q); }
  static __device__ __forceinline__ T lhval(const hops_structure& st, int q) { return ld2f(st.lh_val_f, q); }
  static __device__ __forceinline__ T hval(const hops_structure& st, int q) { return ld2f(st.h_val_f, q); }
  static __device__ __forceinline__ T sval(const hops_structure& st, int j) {
    double2 v = ld2(st.lop_sval, j);
    return mkf((float)v.x, (float)v.y);
  }
  static __device__ __forceinline__ T diag(const double* ws, const ScalarLayout& l, int s) {
    return reinterpret_cast<const float2*>(ws + l.diagD_f())[s];
  }
  static __device__ __forceinline__ T upc(const double* ws, const ScalarLayout& l, int m) {
    return reinterpret_cast<const float2*>(ws + l.upc_f())[m];
  }
  static __device__ __forceinline__ T cz(const double* ws, const ScalarLayout& l, int j) {
    double2 v = ld2(ws + l.cz(), j);
    return mkf((float)v.x, (float)v.y);
  }
};

// ------------------------------------------------- derivative of one element --
// k(a, b, s) of hops_eom.py:389-425 for one trajectory b, reading the stage
// input Y through the row accessor `row(a)` (pointer to Y[a][b][0]).
//   K2_k:      k_decay[a] * y
//   -iH:       sum_s' (-iH)[s,s'] Y[a][s']
//   noise/nc:  (zhat_j - i z2_j) (L_j Y[a])[s] - nc y
//   flux up:   sum_{m, u=a+e_m} (g_m/w_m) (conj<L> Y[u][s] - (L Y[u])[s])
//   flux down: sum_{m, d=a-e_m} k_m(a) w_m (L^H Y[d])[s]
template <typename R, bool SITE, class Row>
__device__ __forceinline__ typename Prec<R>::T deriv_elem(const hops_structure& st, const double* ws,
                                                          const ScalarLayout& lay, int a, int s,
                                                          Row row) {
  using P = Prec<R>;
  using T = typename P::T;
  const T* ya = row(a);
  T y = ya[s];
  T k;
  if (SITE) {
    k = cmul(cadd(P::kdec(st, a), P::diag(ws, lay, s)), y);
  } else {
    T d = P::kdec(st, a);
    d.x -= (R)ws[lay.nc()];
    k = cmul(d, y);
    for (int j = 0; j < st.n_lop; ++j) {
      const int base = j * (st.n_state + 1);
      int q0 = st.l_ptr[base + s], q1 = st.l_ptr[base + s + 1];
      if (q0 == q1) continue;
      T acc = czero<T>();
      for (int q = q0; q < q1; ++q) acc = cfma(P::lval(st, q), ya[st.l_col[q]], acc);
      k = cfma(P::cz(ws, lay, j), acc, k);
    }
  }
  for (int q = st.h_ptr[s]; q < st.h_ptr[s + 1]; ++q) k = cfma(P::hval(st, q), ya[st.h_col[q]], k);
  const int u0 = st.up_ptr[a], u1 = st.up_ptr[a + 1];
  for (int p = u0; p < u1; ++p) {
    const int u = st.up_aux[p], m = st.up_mode[p];
    const T* yu = row(u);
    T c = P::upc(ws, lay, m);
    if (SITE) {
      const int j = st.mode_lop[m];
      if (st.lop_site[j] == s) c = csub(c, cmul(P::gw(st, m), P::sval(st, j)));
      k = cfma(c, yu[s], k);
    } else {
      k = cfma(c, yu[s], k);
      const int j = st.mode_lop[m];
      const int base = j * (st.n_state + 1);
      int q0 = st.l_ptr[base + s], q1 = st.l_ptr[base + s + 1];
      if (q0 != q1) {
        T acc = czero<T>();
        for (int q = q0; q < q1; ++q) acc = cfma(P::lval(st, q), yu[st.l_col[q]], acc);
        k = csub(k, cmul(P::gw(st, m), acc));
      }
    }
  }
  const int d0 = st.dn_ptr[a], d1 = st.dn_ptr[a + 1];
  for (int p = d0; p < d1; ++p) {
    const int d = st.dn_aux[p], m = st.dn_mode[p];
    const int j = st.mode_lop[m];
    const T* yd = row(d);
    if (SITE) {
      if (st.lop_site[j] == s) k = cfma(cmul(P::dncoef(st, p), cconj(P::sval(st, j))), yd[s], k);
    } else {
      const int base = j * (st.n_state + 1);
      int q0 = st.lh_ptr[base + s], q1 = st.lh_ptr[base + s + 1];
      if (q0 != q1) {
        T acc = czero<T>();
        for (int q = q0; q < q1; ++q) acc = cfma(P::lhval(st, q), yd[st.lh_col[q]], acc);
        k = cfma(P::dncoef(st, p), acc, k);
      }
    }
  }
  return k;
}


// ----------------------------------------------------------- stage update ----
template <typename T, typename R>
__device__ __forceinline__ T cdiv6(T a) {
  a.x = a.x / (R)6;
  a.y = a.y / (R)6;
  return a;
}

// RK4 bookkeeping of one element (integrator_rk.py:66-73); phis = phi at the
// start of the step (normalised).  Stage 4 = plain derivative output.
template <typename T, typename R>
__device__ __forceinline__ void rk_update(int stage, R h, T k, T phis, T* acc, T* yout, T* phi,
                                          size_t e) {
  switch (stage) {
    case 0:
      acc[e] = k;
      yout[e] = cadd(phis, cscale(k, h * (R)0.5));
      break;
    case 1:
      acc[e] = cadd(acc[e], cscale(k, (R)2));
      yout[e] = cadd(phis, cscale(k, h * (R)0.5));
      break;
    case 2:
      acc[e] = cadd(acc[e], cscale(k, (R)2));
      yout[e] = cadd(phis, cscale(k, h));
      break;
    case 3: {
      T sum = cadd(acc[e], k);
      phi[e] = cadd(phis, cdiv6<T, R>(cscale(sum, h)));
    } break;
    default:
      yout[e] = k;
  }
}

// ------------------------------------------------ streaming stage kernel ----
// One RK stage for B trajectories sharing a structure.  Groups of G lanes own
// one aux a at a time (warp-uniform connection lists); lanes stride over the
// B*S elements of that aux.  Stage 0 reads the un-normalised phi and folds the
// pending per-trajectory scale into k (the derivative is linear in Y once the
// stage scalars are fixed).
template <typename R, bool SITE>
__global__ void __launch_bounds__(256) k_stage(hops_structure st, int B, int stage, R h,
                                               const typename Prec<R>::T* __restrict__ yin,
                                               typename Prec<R>::T* yout,
                                               typename Prec<R>::T* phi,
                                               typename Prec<R>::T* acc,
                                               const double* __restrict__ ws_all, int G) {
  using T = typename Prec<R>::T;
  const int S = st.n_state;
  const int BS = B * S;
  const ScalarLayout lay(S, st.n_mode, st.n_lop);
  const int lane = threadIdx.x & 31;
  const int gpw = 32 / G;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int sub = lane / G, r0 = lane - sub * G;
  for (int a = warp * gpw + sub; a < st.n_hier; a += nwarps * gpw) {
    for (int r = r0; r < BS; r += G) {
      const int b = r / S, s = r - b * S;
      const double* ws = ws_all + (size_t)b * lay.stride;
      auto row = [&](int x) { return yin + ((size_t)x * B + b) * S; };
      T k = deriv_elem<R, SITE>(st, ws, lay, a, s, row);
      const size_t e = (size_t)a * BS + r;
      const R sc = (R)ws[lay.scale()];
      T phis;
      if (stage == 0 || stage == 4) {
        k = cscale(k, sc);
        phis = cscale(yin[e], sc);
      } else {
        phis = cscale(phi[e], sc);
      }
      rk_update<T, R>(stage, h, k, phis, acc, yout, phi, e);
    }
  }
}

// ----------------------------------------------- streaming scalar kernel ----
// One CTA per trajectory: FP64 stage scalars (stage_scalars) of stage `stage`
// from the stage input yin.  With recompute_scale, first renormalises the state
// produced by the previous step (hops_trajectory.py:616-634) by recording the
// factor 1/||psi_0|| that the stage kernels apply on the fly.
template <typename R>
__global__ void __launch_bounds__(128) k_scalars(hops_structure st, hops_batch bt, int stage, int it,
                                                 double h, const void* yin, int recompute_scale,
                                                 double* psi_prev, const float* z1s,
                                                 const float* z2s, double* dz_out) {
  using T = typename Prec<R>::T;
  extern __shared__ double shm[];
  double* red = shm;
  double* sh = shm + 32;
  const int b = blockIdx.x;
  const int S = st.n_state, M = st.n_mode, L = st.n_lop, B = bt.n_traj;
  const ScalarLayout lay(S, M, L);
  double* ws = bt.work + (size_t)b * lay.stride;
  const T* ph = static_cast<const T*>(bt.phi);
  if (recompute_scale || psi_prev) {
    double sc = ws[lay.scale()];
    if (recompute_scale) {
      double p = 0.0;
      for (int s = threadIdx.x; s < S; s += blockDim.x) {
        double2 v = to_d(ph[(size_t)b * S + s]);
        p += v.x * v.x + v.y * v.y;
      }
      const double n2 = block_sum(p, red);
      sc = 1.0 / sqrt(n2);
      if (!(n2 > 0.0) || !isfinite(sc)) {
        if (threadIdx.x == 0) bt.status[b] = HOPS_ENONFINITE;
        sc = 1.0;
      }
      __syncthreads();
      if (threadIdx.x == 0) ws[lay.scale()] = sc;
    }
    if (psi_prev)
      for (int s = threadIdx.x; s < S; s += blockDim.x)
        reinterpret_cast<double2*>(psi_prev)[(size_t)b * S + s] = cscale(to_d(ph[(size_t)b * S + s]), sc);
    __syncthreads();
  }
  const double sc = (stage == 0 || stage == 4) ? ws[lay.scale()] : 1.0;
  StageIO io;
  io.zmem = bt.zmem + (size_t)b * M * 2;
  if (stage == 4) {
    io.noise1 = z1s ? reinterpret_cast<const float2*>(z1s) + (size_t)b * L : nullptr;
    io.noise2 = z2s ? reinterpret_cast<const float2*>(z2s) + (size_t)b * L : nullptr;
    io.n_t1 = 1;
    io.n_t2 = 1;
    io.it = 0;
    io.zmem_out = dz_out + (size_t)b * M * 2;
  } else {
    io.noise1 = bt.noise1 ? reinterpret_cast<const float2*>(bt.noise1) + (size_t)b * L * bt.n_t1 : nullptr;
    io.noise2 = bt.noise2 ? reinterpret_cast<const float2*>(bt.noise2) + (size_t)b * L * bt.n_t2 : nullptr;
    io.n_t1 = bt.n_t1;
    io.n_t2 = bt.n_t2;
    io.it = it;
    io.zmem_out = bt.zmem + (size_t)b * M * 2;
  }
  io.stage = stage;
  io.eom = bt.eom;
  io.h = h;
  io.ws = ws;
  const T* y = static_cast<const T*>(yin);
  auto get = [&](int a, int s) -> double2 {
    return cscale(to_d(y[((size_t)a * B + b) * S + s]), sc);
  };
  stage_scalars(st, io, get, red, sh);
}

// Normalisation after the last step of a call: records 1/||psi_0|| per
// trajectory and writes the last psi_0.
template <typename R>
__global__ void __launch_bounds__(128) k_finalize(hops_structure st, hops_batch bt, double* psi_last,
                                                  int normalize) {
  using T = typename Prec<R>::T;
  __shared__ double red[32];
  const int b = blockIdx.x, S = st.n_state;
  const ScalarLayout lay(S, st.n_mode, st.n_lop);
  double* ws = bt.work + (size_t)b * lay.stride;
  const T* ph = static_cast<const T*>(bt.phi);
  double sc = 1.0;
  if (normalize) {
    double p = 0.0;
    for (int s = threadIdx.x; s < S; s += blockDim.x) {
      double2 v = to_d(ph[(size_t)b * S + s]);
      p += v.x * v.x + v.y * v.y;
    }
    const double n2 = block_sum(p, red);
    sc = 1.0 / sqrt(n2);
    if (!(n2 > 0.0) || !isfinite(sc)) {
      if (threadIdx.x == 0) bt.status[b] = HOPS_ENONFINITE;
      sc = 1.0;
    }
  }
  if (threadIdx.x == 0) ws[lay.scale()] = sc;
  if (psi_last)
    for (int s = threadIdx.x; s < S; s += blockDim.x)
      reinterpret_cast<double2*>(psi_last)[(size_t)b * S + s] = cscale(to_d(ph[(size_t)b * S + s]), sc);
}

template <typename R>
__global__ void k_apply_scale(typename Prec<R>::T* phi, int B, int S, size_t E,
                              const double* ws, int stride) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < E;
       e += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)((e / S) % B);
    phi[e] = cscale(phi[e], (R)ws[(size_t)b * stride]);
  }
}

__global__ void k_reset(double* ws, int stride, int B, int32_t* status, int clear_status) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < B) {
    ws[(size_t)b * stride] = 1.0;
    if (clear_status && status) status[b] = 0;
  }
}

// --------------------------------------------------------- resident kernel ----
// One CTA owns one trajectory for all n_steps steps: stage scalars, the four
// RK stages and the renormalisation run back to back with only __syncthreads
// between them (no grid-wide synchronisation).  Vectors live in shared memory
// when they fit (mode 2: phi, acc, y0, y1; mode 1: y0, y1), else in the task's
// scratch.  Tasks may carry different structures (uneven adaptive bases).
template <typename R, bool SITE>
__global__ void __launch_bounds__(512) k_resident(hops_task* tasks, int mode, int max_elems,
                                                  int sc_doubles) {
  using T = typename Prec<R>::T;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ hops_structure st;
  __shared__ double red[32];
  hops_task* tk = tasks + blockIdx.x;
  if (threadIdx.x == 0) st = *tk->st;
  __syncthreads();
  const int S = st.n_state, M = st.n_mode, L = st.n_lop;
  const int E = st.n_hier * S;
  const ScalarLayout lay(S, M, L);
  double* ws = reinterpret_cast<double*>(smraw);
  double* zm = ws + lay.stride;
  double* sh = zm + 2 * M;
  T* vec = reinterpret_cast<T*>(smraw + (size_t)sc_doubles * sizeof(double));
  T *phi, *acc, *y0, *y1;
  T* gphi = static_cast<T*>(tk->phi);
  if (mode == 2) {
    phi = vec;
    acc = vec + max_elems;
    y0 = vec + 2 * max_elems;
    y1 = vec + 3 * max_elems;
  } else if (mode == 1) {
    y0 = vec;
    y1 = vec + max_elems;
    phi = gphi;
    acc = static_cast<T*>(tk->scratch);
  } else {
    phi = gphi;
    acc = static_cast<T*>(tk->scratch);
    y0 = acc + E;
    y1 = acc + 2 * E;
  }
  const R sc0 = (R)tk->scale;
  for (int e = threadIdx.x; e < E; e += blockDim.x) phi[e] = cscale(gphi[e], sc0);
  for (int m = threadIdx.x; m < M; m += blockDim.x)
    reinterpret_cast<double2*>(zm)[m] = reinterpret_cast<const double2*>(tk->zmem)[m];
  __syncthreads();
  const bool normalized = tk->eom == HOPS_EOM_NORMALIZED_NONLINEAR;
  const R h = (R)tk->tau_over_hbar;
  int status = 0;
  StageIO io;
  io.zmem = zm;
  io.zmem_out = zm;
  io.noise1 = reinterpret_cast<const float2*>(tk->noise1);
  io.noise2 = reinterpret_cast<const float2*>(tk->noise2);
  io.n_t1 = tk->n_t1;
  io.n_t2 = tk->n_t2;
  io.eom = tk->eom;
  io.h = tk->tau_over_hbar;
  io.ws = ws;
  for (int n = 0; n < tk->n_steps; ++n) {
    for (int stage = 0; stage < 4; ++stage) {
      const T* yin = stage == 0 ? phi : (stage == 1 ? y0 : (stage == 2 ? y1 : y0));
      T* yout = stage == 0 ? y0 : (stage == 1 ? y1 : (stage == 2 ? y0 : nullptr));
      io.it = tk->it0 + 2 * n * tk->di + rk_noise_slot(stage) * tk->di;
      io.stage = stage;
      auto get = [&](int a, int s) -> double2 { return to_d(yin[a * S + s]); };
      stage_scalars(st, io, get, red, sh);
      auto row = [&](int x) { return yin + x * S; };
      for (int e = threadIdx.x; e < E; e += blockDim.x) {
        const int a = e / S, s = e - a * S;
        T k = deriv_elem<R, SITE>(st, ws, lay, a, s, row);
        rk_update<T, R>(stage, h, k, phi[e], acc, yout, phi, (size_t)e);
      }
      __syncthreads();
    }
    if (normalized) {
      double p = 0.0;
      for (int s = threadIdx.x; s < S; s += blockDim.x) {
        double2 v = to_d(phi[s]);
        p += v.x * v.x + v.y * v.y;
      }
      const double n2 = block_sum(p, red);
      double sc = 1.0 / sqrt(n2);
      if (!(n2 > 0.0) || !isfinite(sc)) {
        status = HOPS_ENONFINITE;
        sc = 1.0;
      }
      for (int e = threadIdx.x; e < E; e += blockDim.x) phi[e] = cscale(phi[e], (R)sc);
      __syncthreads();
    }
    if (tk->psi_out)
      for (int s = threadIdx.x; s < S; s += blockDim.x)
        reinterpret_cast<double2*>(tk->psi_out)[(size_t)n * S + s] = to_d(phi[s]);
  }
  __syncthreads();
  if (mode == 2)
    for (int e = threadIdx.x; e < E; e += blockDim.x) gphi[e] = phi[e];
  for (int m = threadIdx.x; m < M; m += blockDim.x)
    reinterpret_cast<double2*>(tk->zmem)[m] = reinterpret_cast<const double2*>(zm)[m];
  if (threadIdx.x == 0) {
    tk->status = status;
    tk->scale = 1.0;
  }
}

// ============================================================= C ABI =========
static int g_sm_count = 0;

static int sm_count() {
  if (g_sm_count == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      g_sm_count = 148;
  }
  return g_sm_count;
}

static int check_structure(const hops_structure* st) {
  if (!st) return set_err(HOPS_EINVAL, "null structure");
  if (st->n_hier <= 0 || st->n_state <= 0 || st->n_mode < 0 || st->n_lop < 0)
    return set_err(HOPS_EINVAL, "bad structure sizes n_hier=%d n_state=%d n_mode=%d n_lop=%d",
                   st->n_hier, st->n_state, st->n_mode, st->n_lop);
  if (!st->k_decay || !st->up_ptr || !st->dn_ptr || !st->h_ptr || !st->l_ptr || !st->lop_active)
    return set_err(HOPS_EINVAL, "structure has null tables");
  if (st->site_projector && (!st->lop_site || !st->lop_sval))
    return set_err(HOPS_EINVAL, "site-projector structure without lop_site/lop_sval");
  return HOPS_OK;
}

static int check_batch(const hops_structure* st, const hops_batch* bt) {
  if (!bt) return set_err(HOPS_EINVAL, "null batch");
  if (bt->n_traj <= 0) return set_err(HOPS_EINVAL, "n_traj must be positive");
  if (bt->precision != HOPS_PREC_C128 && bt->precision != HOPS_PREC_C64)
    return set_err(HOPS_EINVAL, "unknown precision %d", bt->precision);
  if (bt->eom < 0 || bt->eom > 2) return set_err(HOPS_EINVAL, "unknown eom %d", bt->eom);
  if (!bt->phi || !bt->acc || !bt->y0 || !bt->y1 || !bt->zmem || !bt->work || !bt->status)
    return set_err(HOPS_EINVAL, "batch has null buffers");
  if (bt->precision == HOPS_PREC_C64 &&
      (!st->k_decay_f || !st->dn_coef_f || !st->mode_gw_f || !st->h_val_f || !st->l_val_f ||
       !st->lh_val_f))
    return set_err(HOPS_EINVAL, "complex64 batch needs the float coefficient tables");
  (void)st;
  return HOPS_OK;
}

static int group_lanes(int bs) {
  if (bs >= 32) return 32;
  int g = 1;
  while (g < bs) g <<= 1;
  return g;
}

static int stage_grid(const hops_structure* st, int G) {
  const int gpw = 32 / G;
  const long warps = (st->n_hier + gpw - 1) / gpw;
  long blocks = (warps * 32 + 255) / 256;
  const long cap = (long)sm_count() * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

template <typename R>
static int run_stage(const hops_structure* st, int B, int stage, double h, const void* yin,
                     void* yout, void* phi, void* acc, const double* ws, cudaStream_t s) {
  using T = typename Prec<R>::T;
  const int G = group_lanes(B * st->n_state);
  const int grid = stage_grid(st, G);
  if (st->site_projector)
    k_stage<R, true><<<grid, 256, 0, s>>>(*st, B, stage, (R)h, (const T*)yin, (T*)yout, (T*)phi,
                                          (T*)acc, ws, G);
  else
    k_stage<R, false><<<grid, 256, 0, s>>>(*st, B, stage, (R)h, (const T*)yin, (T*)yout, (T*)phi,
                                           (T*)acc, ws, G);
  LAUNCH_CHECK();
  return HOPS_OK;
}

static size_t scalar_smem(const hops_structure* st) {
  return (size_t)(32 + 4 * st->n_lop + 2) * sizeof(double);
}

template <typename R>
static int propagate_impl(const hops_structure* st, hops_batch* bt, int32_t it0, int32_t di,
                          int32_t n_steps, double h, double* psi_out, cudaStream_t s) {
  using T = typename Prec<R>::T;
  const int B = bt->n_traj, S = st->n_state;
  const size_t smem = scalar_smem(st);
  const bool normalized = bt->eom == HOPS_EOM_NORMALIZED_NONLINEAR;
  const size_t psi_stride = (size_t)B * S * 2;
  for (int n = 0; n < n_steps; ++n) {
    for (int i = 0; i < 4; ++i) {
      const int slot = i == 0 ? 0 : (i == 3 ? 2 : 1);
      const int it = it0 + 2 * n * di + slot * di;
      const void* yin = i == 0 ? bt->phi : (i == 1 ? bt->y0 : (i == 2 ? bt->y1 : bt->y0));
      void* yout = i == 0 ? bt->y0 : (i == 1 ? bt->y1 : (i == 2 ? bt->y0 : nullptr));
      const int recompute = (i == 0 && n > 0 && normalized) ? 1 : 0;
      double* psi_prev = (i == 0 && n > 0 && psi_out) ? psi_out + (size_t)(n - 1) * psi_stride : nullptr;
      k_scalars<R><<<B, 128, smem, s>>>(*st, *bt, i, it, h, yin, recompute, psi_prev, nullptr,
                                        nullptr, nullptr);
      LAUNCH_CHECK();
      int rc = run_stage<R>(st, B, i, h, yin, yout, bt->phi, bt->acc, bt->work, s);
      if (rc) return rc;
    }
  }
  if (n_steps > 0) {
    double* psi_last = psi_out ? psi_out + (size_t)(n_steps - 1) * psi_stride : nullptr;
    k_finalize<R><<<B, 128, 0, s>>>(*st, *bt, psi_last, normalized ? 1 : 0);
    LAUNCH_CHECK();
    if (normalized) {
      const size_t E = (size_t)st->n_hier * B * S;
      long blocks = (long)((E + 255) / 256);
      if (blocks > (long)sm_count() * 8) blocks = (long)sm_count() * 8;
      const ScalarLayout lay(S, st->n_mode, st->n_lop);
      k_apply_scale<R><<<(int)blocks, 256, 0, s>>>((T*)bt->phi, B, S, E, bt->work, lay.stride);
      LAUNCH_CHECK();
      k_reset<<<(B + 127) / 128, 128, 0, s>>>(bt->work, lay.stride, B, nullptr, 0);
      LAUNCH_CHECK();
    }
  }
  return HOPS_OK;
}

extern "C" int hops_batch_reset(const hops_structure* st, hops_batch* bt, void* stream) {
  int rc = check_structure(st);
  if (rc) return rc;
  if ((rc = check_batch(st, bt))) return rc;
  const ScalarLayout lay(st->n_state, st->n_mode, st->n_lop);
  k_reset<<<(bt->n_traj + 127) / 128, 128, 0, (cudaStream_t)stream>>>(bt->work, lay.stride,
                                                                       bt->n_traj, bt->status, 1);
  LAUNCH_CHECK();
  return HOPS_OK;
}

extern "C" int hops_rk4_propagate(const hops_structure* st, hops_batch* bt, int32_t it0,
                                  int32_t di, int32_t n_steps, double tau_over_hbar,
                                  double* psi_out_dev, void* stream) {
  int rc = check_structure(st);
  if (rc) return rc;
  if ((rc = check_batch(st, bt))) return rc;
  if (n_steps < 0 || it0 < 0 || di < 0) return set_err(HOPS_EINVAL, "negative step/noise index");
  if (!bt->noise1 && bt->eom != HOPS_EOM_LINEAR && false) return set_err(HOPS_EINVAL, "no noise");
  const long last = (long)it0 + 2L * n_steps * di;
  if (n_steps > 0 && bt->noise1 && last >= bt->n_t1)
    return set_err(HOPS_EINVAL, "noise 1 too short: needs index %ld, has %d samples", last, bt->n_t1);
  if (n_steps > 0 && bt->noise2 && last >= bt->n_t2)
    return set_err(HOPS_EINVAL, "noise 2 too short: needs index %ld, has %d samples", last, bt->n_t2);
  if (scalar_smem(st) > 48 * 1024) return set_err(HOPS_ENOTSUP, "too many L operators (%d)", st->n_lop);
  cudaStream_t s = (cudaStream_t)stream;
  if (bt->precision == HOPS_PREC_C128)
    return propagate_impl<double>(st, bt, it0, di, n_steps, tau_over_hbar, psi_out_dev, s);
  return propagate_impl<float>(st, bt, it0, di, n_steps, tau_over_hbar, psi_out_dev, s);
}

extern "C" int hops_dsystem_dt(const hops_structure* st, hops_batch* bt, const float* z1_dev,
                               const float* z2_dev, void* dphi_dev, double* dzmem_dev,
                               void* stream) {
  int rc = check_structure(st);
  if (rc) return rc;
  if ((rc = check_batch(st, bt))) return rc;
  if (!dphi_dev || !dzmem_dev) return set_err(HOPS_EINVAL, "null outputs");
  if (scalar_smem(st) > 48 * 1024) return set_err(HOPS_ENOTSUP, "too many L operators (%d)", st->n_lop);
  cudaStream_t s = (cudaStream_t)stream;
  const size_t smem = scalar_smem(st);
  if (bt->precision == HOPS_PREC_C128) {
    k_scalars<double><<<bt->n_traj, 128, smem, s>>>(*st, *bt, 4, 0, 0.0, bt->phi, 0, nullptr,
                                                    z1_dev, z2_dev, dzmem_dev);
    LAUNCH_CHECK();
    return run_stage<double>(st, bt->n_traj, 4, 0.0, bt->phi, dphi_dev, bt->phi, bt->acc, bt->work, s);
  }
  k_scalars<float><<<bt->n_traj, 128, smem, s>>>(*st, *bt, 4, 0, 0.0, bt->phi, 0, nullptr, z1_dev,
                                                 z2_dev, dzmem_dev);
  LAUNCH_CHECK();
  return run_stage<float>(st, bt->n_traj, 4, 0.0, bt->phi, dphi_dev, bt->phi, bt->acc, bt->work, s);
}

static size_t resident_sc_doubles(int max_sc) {
  // scalar block + z_mem copy + stage scratch, rounded to 16 bytes
  return (size_t)((max_sc + 1) & ~1);
}

template <typename R>
static int resident_impl(hops_task* tasks, int n_tasks, int max_elems, int max_sc,
                         int site, cudaStream_t s) {
  using T = typename Prec<R>::T;
  int dev = 0, optin = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t scb = resident_sc_doubles(max_sc) * sizeof(double);
  const size_t budget = (size_t)optin - sizeof(hops_structure) - 32 * sizeof(double) - 64;
  int mode = 0;
  size_t smem = scb;
  if (scb + 4 * (size_t)max_elems * sizeof(T) <= budget) {
    mode = 2;
    smem = scb + 4 * (size_t)max_elems * sizeof(T);
  } else if (scb + 2 * (size_t)max_elems * sizeof(T) <= budget) {
    mode = 1;
    smem = scb + 2 * (size_t)max_elems * sizeof(T);
  } else if (scb > budget) {
    return set_err(HOPS_ENOTSUP, "resident scalar block of %zu bytes exceeds shared memory", scb);
  }
  int threads = ((max_elems + 31) / 32) * 32;
  if (threads < 64) threads = 64;
  if (threads > 512) threads = 512;
  if (site) {
    CUDA_TRY(cudaFuncSetAttribute(k_resident<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_resident<R, true><<<n_tasks, threads, smem, s>>>(tasks, mode, max_elems,
                                                       (int)resident_sc_doubles(max_sc));
  } else {
    CUDA_TRY(cudaFuncSetAttribute(k_resident<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_resident<R, false><<<n_tasks, threads, smem, s>>>(tasks, mode, max_elems,
                                                        (int)resident_sc_doubles(max_sc));
  }
  LAUNCH_CHECK();
  return HOPS_OK;
}

extern "C" int hops_resident_propagate(hops_task* tasks_dev, int32_t n_tasks, int32_t max_elems,
                                       int32_t max_scalar_doubles, int32_t precision,
                                       int32_t all_site_projector, void* stream) {
  if (!tasks_dev || n_tasks <= 0 || max_elems <= 0 || max_scalar_doubles <= 0)
    return set_err(HOPS_EINVAL, "bad resident launch arguments");
  if (n_tasks > 2147483647 / 2) return set_err(HOPS_EINVAL, "too many tasks");
  cudaStream_t s = (cudaStream_t)stream;
  if (precision == HOPS_PREC_C128)
    return resident_impl<double>(tasks_dev, n_tasks, max_elems, max_scalar_doubles,
                                 all_site_projector, s);
  if (precision == HOPS_PREC_C64)
    return resident_impl<float>(tasks_dev, n_tasks, max_elems, max_scalar_doubles,
                                all_site_projector, s);
  return set_err(HOPS_EINVAL, "unknown precision %d", precision);
}

extern "C" int32_t hops_resident_scalar_doubles(int32_t n_state, int32_t n_mode, int32_t n_lop) {
  const ScalarLayout lay(n_state, n_mode, n_lop);
  return lay.stride + 2 * n_mode + 4 * n_lop + 2;
}
