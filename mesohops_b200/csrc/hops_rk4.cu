// B200 kernels of the HOPS trajectory hot path: batched RK4 over the auxiliary
// hierarchy (streaming stage kernels) and the resident one-CTA-per-trajectory
// propagator.  See hops_b200.h for the C ABI and the reference functions each
// entry point replaces.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <stdarg.h>
#include <algorithm>
#include <utility>
#include <vector>
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

// ------------------------------------------- programmatic dependent launch ----
// The scalar and stage kernels of a propagate call form a chain in one stream
// (k_scalars -> stage kernel -> k_scalars ...).  With HOPS_PDL they are
// launched with programmatic stream serialisation: each kernel lets its
// dependent launch at once (griddepcontrol.launch_dependents) and waits for
// its predecessor's completion and memory (griddepcontrol.wait) before it
// reads anything, so the dependent's launch and CTA placement overlap the
// running kernel instead of following it.  A dependent launches only once
// every CTA of its predecessor is resident and has triggered, and no kernel
// waits on its dependent, so the waits always end.
#ifndef HOPS_PDL
#define HOPS_PDL 1
#endif
// the stage kernels: let the next k_scalars launch at once, then wait
__device__ __forceinline__ void pdl_enter() {
#if HOPS_PDL
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}
// k_scalars waits at entry and lets the next stage kernel launch only at its
// end, so that the stage kernel's one-wave grid is placed all at once rather
// than partly beside the scalar CTAs
__device__ __forceinline__ void pdl_wait() {
#if HOPS_PDL
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}
__device__ __forceinline__ void pdl_trigger() {
#if HOPS_PDL
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}
template <typename... KArgs, typename... Args>
static cudaError_t launch_chain(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                cudaStream_t s, Args&&... args) {
#if HOPS_PDL
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
#else
  kern<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
  return cudaGetLastError();
#endif
}

// ------------------------------------------------------------- precision ----
// Structure coefficients in the arithmetic precision R.
template <typename R> struct Prec;
template <> struct Prec<double> {
  using T = double2;
  static __device__ __forceinline__ T kdec(const hops_structure& st, int a) { return ld2(st.k_decay, a); }
  static __device__ __forceinline__ T dncoef(const hops_structure& st, int p) { return ld2(st.dn_coef, p); }
  static __device__ __forceinline__ T dncs(const hops_structure& st, int p) { return ld2(st.dn_coef_site, p); }
  static __device__ __forceinline__ T gw(const hops_structure& st, int m) { return ld2(st.mode_gw, m); }
  static __device__ __forceinline__ T gwv(const hops_structure& st, int m) { return ld2(st.mode_gwv, m); }
  static __device__ __forceinline__ T lval(const hops_structure& st, int q) { return ld2(st.l_val, q); }
  static __device__ __forceinline__ T lhval(const hops_structure& st, int q) { return ld2(st.lh_val, q); }
  static __device__ __forceinline__ T hval(const hops_structure& st, int q) { return ld2(st.h_val, q); }
  static __device__ __forceinline__ T hdiag(const hops_structure& st, int s) { return ld2(st.h_diag, s); }
};
template <> struct Prec<float> {
  using T = float2;
  static __device__ __forceinline__ T kdec(const hops_structure& st, int a) { return ld2f(st.k_decay_f, a); }
  static __device__ __forceinline__ T dncoef(const hops_structure& st, int p) { return ld2f(st.dn_coef_f, p); }
  static __device__ __forceinline__ T dncs(const hops_structure& st, int p) { return ld2f(st.dn_coef_site_f, p); }
  static __device__ __forceinline__ T gw(const hops_structure& st, int m) { return ld2f(st.mode_gw_f, m); }
  static __device__ __forceinline__ T gwv(const hops_structure& st, int m) { return ld2f(st.mode_gwv_f, m); }
  static __device__ __forceinline__ T lval(const hops_structure& st, int q) { return ld2f(st.l_val_f, q); }
  static __device__ __forceinline__ T lhval(const hops_structure& st, int q) { return ld2f(st.lh_val_f, q); }
  static __device__ __forceinline__ T hval(const hops_structure& st, int q) { return ld2f(st.h_val_f, q); }
  static __device__ __forceinline__ T hdiag(const hops_structure& st, int s) {
    const double2 v = ld2(st.h_diag, s);
    return mkf((float)v.x, (float)v.y);
  }
};

extern "C" size_t hops_scalar_workspace_doubles(int32_t S, int32_t M, int32_t L, int32_t B) {
  return BatchLayout(S, M, L, B).total;
}

// Per-thread stage coefficients of trajectory b read from the transposed arrays.
template <typename R> struct CoefT {
  using T = typename Prec<R>::T;
  const double* ws;
  BatchLayout bl;
  int B, b;
  __device__ __forceinline__ T diag(int s) const {
    if constexpr (sizeof(R) == 8) return ld2(ws + bl.diagT, s * B + b);
    else return ld2f(reinterpret_cast<const float*>(ws + bl.diagT_f), s * B + b);
  }
  __device__ __forceinline__ T upc(int m) const {
    if constexpr (sizeof(R) == 8) return ld2(ws + bl.upcT, m * B + b);
    else return ld2f(reinterpret_cast<const float*>(ws + bl.upcT_f), m * B + b);
  }
  __device__ __forceinline__ T cz(int j) const {
    if constexpr (sizeof(R) == 8) return ld2(ws + bl.czT, j * B + b);
    else return ld2f(reinterpret_cast<const float*>(ws + bl.czT_f), j * B + b);
  }
  __device__ __forceinline__ R nc() const { return (R)ws[bl.ncB + b]; }
  __device__ __forceinline__ T phys(int s) const {
    if constexpr (sizeof(R) == 8) return ld2(ws + bl.physT, s * B + b);
    else return ld2f(reinterpret_cast<const float*>(ws + bl.physT_f), s * B + b);
  }
};

// Stage coefficients of one trajectory read from its ScalarLayout block
// (resident kernel, block in shared memory).
template <typename R> struct CoefWS {
  using T = typename Prec<R>::T;
  const double* ws;
  ScalarLayout lay;
  __device__ __forceinline__ T diag(int s) const {
    if constexpr (sizeof(R) == 8) return ld2(ws + lay.diagD(), s);
    else return ld2f(reinterpret_cast<const float*>(ws + lay.diagD_f()), s);
  }
  __device__ __forceinline__ T upc(int m) const {
    if constexpr (sizeof(R) == 8) return ld2(ws + lay.upc(), m);
    else return ld2f(reinterpret_cast<const float*>(ws + lay.upc_f()), m);
  }
  __device__ __forceinline__ T cz(int j) const {
    double2 v = ld2(ws + lay.cz(), j);
    if constexpr (sizeof(R) == 8) return v;
    else return mkf((float)v.x, (float)v.y);
  }
  __device__ __forceinline__ R nc() const { return (R)ws[lay.nc()]; }
  __device__ __forceinline__ T phys(int s) const {
    if constexpr (sizeof(R) == 8) return ld2(ws + lay.phys(), s);
    else return ld2f(reinterpret_cast<const float*>(ws + lay.phys_f()), s);
  }
};

// ------------------------------------------------- derivative of one element --
// k(a, s) of hops_eom.py:389-425 for one trajectory, reading the stage input
// through y(aux, state) and the stage coefficients through cf:
//   K2_k + noise + norm:  (k_decay[a] + diag(s)) y            (site projectors)
//                         (k_decay[a] - nc) y + sum_j cz_j (L_j Y[a])[s]   (general L)
//   -iH:                  sum_s' (-iH)[s,s'] Y[a][s']
//   flux up (K2_kp1+Z2):  sum_{m, u=a+e_m} (g_m/w_m)(conj<L> Y[u][s] - (L Y[u])[s])
//   flux down (K2_km1):   sum_{m, d=a-e_m} k_m(a) w_m (L^H Y[d])[s]
template <typename R, bool SITE, class Y, class Cf>
__device__ __forceinline__ typename Prec<R>::T deriv_elem(const hops_structure& st, int a, int s,
                                                          Y y, const Cf& cf) {
  using P = Prec<R>;
  using T = typename P::T;
  T k;
  if (SITE) {
    k = cmul(cadd(P::kdec(st, a), cf.diag(s)), y(a, s));
  } else {
    T d = P::kdec(st, a);
    d.x -= cf.nc();
    // a site-projector structure evaluated by the general path: the diagonal
    // of -iH is not in its H CSR
    if (st.h_diag) d = cadd(d, P::hdiag(st, s));
    k = cmul(d, y(a, s));
    const int base_s = s;
    for (int j = 0; j < st.n_lop; ++j) {
      const int base = j * (st.n_state + 1);
      const int q0 = st.l_ptr[base + base_s], q1 = st.l_ptr[base + base_s + 1];
      if (q0 == q1) continue;
      T acc = czero<T>();
      for (int q = q0; q < q1; ++q) acc = cfma(P::lval(st, q), y(a, st.l_col[q]), acc);
      k = cfma(cf.cz(j), acc, k);
    }
  }
  for (int q = st.h_ptr[s]; q < st.h_ptr[s + 1]; ++q) k = cfma(P::hval(st, q), y(a, st.h_col[q]), k);
  const int u0 = st.up_ptr[a], u1 = st.up_ptr[a + 1];
  for (int p = u0; p < u1; ++p) {
    const int u = st.up_aux[p], m = st.up_mode[p];
    T c = cf.upc(m);
    if (SITE) {
      if (st.up_site[p] == s) c = csub(c, P::gwv(st, m));
      k = cfma(c, y(u, s), k);
    } else {
      k = cfma(c, y(u, s), k);
      const int base = st.mode_lop[m] * (st.n_state + 1);
      const int q0 = st.l_ptr[base + s], q1 = st.l_ptr[base + s + 1];
      if (q0 != q1) {
        T acc = czero<T>();
        for (int q = q0; q < q1; ++q) acc = cfma(P::lval(st, q), y(u, st.l_col[q]), acc);
        k = csub(k, cmul(P::gw(st, m), acc));
      }
    }
  }
  const int d0 = st.dn_ptr[a], d1 = st.dn_ptr[a + 1];
  for (int p = d0; p < d1; ++p) {
    const int d = st.dn_aux[p];
    if (SITE) {
      if (st.dn_site[p] == s) k = cfma(P::dncs(st, p), y(d, s), k);
    } else {
      const int m = st.dn_mode[p];
      const int base = st.mode_lop[m] * (st.n_state + 1);
      const int q0 = st.lh_ptr[base + s], q1 = st.lh_ptr[base + s + 1];
      if (q0 != q1) {
        T acc = czero<T>();
        for (int q = q0; q < q1; ++q) acc = cfma(P::lhval(st, q), y(d, st.lh_col[q]), acc);
        k = cfma(P::dncoef(st, p), acc, k);
      }
    }
  }
  return k;
}

// ------------------------------------------------------- type conversion ----
template <typename To> __device__ __forceinline__ To cv(double2 a);
template <typename To> __device__ __forceinline__ To cv(float2 a);
template <> __device__ __forceinline__ double2 cv<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ double2 cv<double2>(float2 a) { return mk(a.x, a.y); }
template <> __device__ __forceinline__ float2 cv<float2>(float2 a) { return a; }
template <> __device__ __forceinline__ float2 cv<float2>(double2 a) { return mkf((float)a.x, (float)a.y); }

// Division by a run-time constant d < 2^31 with one multiply-high and a shift
// (Granlund & Montgomery, "Division by invariant integers using
// multiplication", 1994): l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (mulhi(m, n) + n) >> l for every 32-bit n.
struct FastDiv {
  unsigned d, m, l;
  FastDiv() : d(1), m(1), l(0) {}
  explicit FastDiv(unsigned dd) : d(dd) {
    l = 0;
    while ((1ull << l) < dd) ++l;
    m = (unsigned)((((1ull << 32) * ((1ull << l) - dd)) / dd) + 1);
  }
  __device__ __forceinline__ unsigned div(unsigned n) const {
    const unsigned hi = __umulhi(m, n);
    return (unsigned)(((unsigned long long)hi + n) >> l);
  }
};

// ----------------------------------------------------------- stage update ----
// L2 eviction priorities of the batched stage kernel (HOPS_WIDE_HINTS bit 0:
// the read-once streams -- phi, acc and the stage outputs -- evict-first;
// bit 1: the stage input Y, which the neighbour gathers re-read, evict-last).
// Bit 0 alone is the default: on the 20-site ring it took 5 % off the
// complex128 stage (3 % mixed, none complex64); bit 1 gained nothing more.
#ifndef HOPS_WIDE_HINTS
#define HOPS_WIDE_HINTS 1
#endif
// RK4 bookkeeping of one element (integrator_rk.py:66-73).  ph: the state at
// the start of the step (already scaled) in the state type PT; k in the
// arithmetic type T; acc, the stage inputs and phi's complex64 copy stored in
// the stage type ST.  Stage inputs and the new state are formed in PT
// arithmetic and rounded once to their storage types.  GHINT (stage kernels,
// whose buffers are always in global memory): the accumulator is touched only
// by its owner thread, so it is loaded and stored evict-first.  The resident
// kernel keeps acc in shared memory and must not use the global-only hints.
// Stage 4 = plain derivative output.
template <bool GHINT, typename ST>
__device__ __forceinline__ ST acc_load(const ST* p) {
  if constexpr (GHINT) return __ldcs(p);
  else return *p;
}
template <bool GHINT, typename ST>
__device__ __forceinline__ void acc_store(ST* p, ST v) {
  if constexpr (GHINT) __stcs(p, v);
  else *p = v;
}
// store of a stage output or the new state (evict-first when OHINT: the
// batched stage kernel with HOPS_WIDE_HINTS bit 0)
template <bool OHINT, typename V>
__device__ __forceinline__ void out_store(V* p, V v) {
  if constexpr (OHINT) __stcs(p, v);
  else *p = v;
}

// Partial-sum form of the stage kernels: the third stage does not store the
// accumulated slope k1 + 2 k2 + 2 k3 but the partial sum
// P = phi + h/6 (k1 + 2 k2 + 2 k3) in the state's precision, and the fourth
// stage reads P in place of phi and the slope: phi' = P + h/6 k4.  With the
// stage vectors in the state's precision (complex128, complex64) P takes the
// accumulator's buffer and the fourth stage skips the read of phi: 16 vector
// passes per step instead of 17.  Mixed precision (complex128 state,
// complex64 stage vectors) splits P -- real parts in the accumulator's
// buffer, imaginary parts in the buffer of phi's complex64 copy, which no
// kernel reads between the second stage and the fourth: the same bytes move
// as with the slope, and one complex64 rounding of the largest slope term is
// gone.  The sum is rounded as phi + h/6 (k1 + 2 k2 + 2 k3) + h/6 k4 instead
// of phi + h/6 (k1 + 2 k2 + 2 k3 + k4): a difference in the last bit.
template <typename ST, typename PT>
constexpr bool psum_mode() { return true; }
template <typename ST, typename PT>
constexpr bool psum_split() { return sizeof(PT) == 16 && sizeof(ST) == 8; }

__device__ __forceinline__ double* psum_re(void* acc) { return static_cast<double*>(acc); }
__device__ __forceinline__ double* psum_im(void* shadow) { return static_cast<double*>(shadow); }

// rk_finish: the same update with the accumulated slope acc[e] already loaded
// (accv; read at stages 1-3 only), so that a caller can load the operands of
// several elements before it stores any of them.  PSUM: the partial-sum form
// above (the caller passes P as ph at the fourth stage).
template <bool GHINT, bool PSUM, typename T, typename ST, typename PT, bool OHINT = false>
__device__ __forceinline__ void rk_finish(int stage, double h, T k, PT ph, ST accv, ST* acc,
                                          ST* yout, PT* phi, ST* shadow, size_t e) {
  using RP = decltype(ph.x);
  const RP hh = (RP)h;
  // h / 6 rounded once: the reference divides h (k1 + 2 k2 + 2 k3 + k4) by 6
  // (integrator_rk.py:75); the product with h/6 differs in the last bit and
  // spares every element an IEEE division
  const RP h6 = (RP)(h / 6.0);
  if constexpr (PSUM) {
    if (stage == 2) {
      PT sum = cv<PT>(cadd(cv<T>(accv), cscale(k, (decltype(k.x))2)));
      const PT hs = cscale(sum, h6);
      const PT pp = cadd(ph, hs);
      if constexpr (psum_split<ST, PT>()) {
        __stcs(psum_re(acc) + e, (double)pp.x);
        __stcs(psum_im(shadow) + e, (double)pp.y);
      } else {
        acc_store<GHINT>(acc + e, cv<ST>(pp));
      }
      out_store<OHINT>(yout + e, cv<ST>(cadd(ph, cscale(cv<PT>(k), hh))));
      return;
    }
    if (stage == 3) {
      const PT hs = cscale(cv<PT>(k), h6);
      const PT nw = cadd(ph, hs);
      out_store<OHINT>(phi + e, nw);
      if (psum_split<ST, PT>() || shadow) out_store<OHINT>(shadow + e, cv<ST>(nw));
      return;
    }
  }
  switch (stage) {
    case 0: {
      acc_store<GHINT>(acc + e, cv<ST>(k));
      out_store<OHINT>(yout + e, cv<ST>(cadd(ph, cscale(cv<PT>(k), hh * (RP)0.5))));
    } break;
    case 1:
    case 2: {
      const T a0 = cv<T>(accv);
      acc_store<GHINT>(acc + e, cv<ST>(cadd(a0, cscale(k, (decltype(k.x))2))));
      const RP c = stage == 1 ? hh * (RP)0.5 : hh;
      out_store<OHINT>(yout + e, cv<ST>(cadd(ph, cscale(cv<PT>(k), c))));
    } break;
    case 3: {
      PT sum = cv<PT>(cadd(cv<T>(accv), k));
      const PT hs = cscale(sum, h6);
      const PT nw = cadd(ph, hs);
      out_store<OHINT>(phi + e, nw);
      if (shadow) out_store<OHINT>(shadow + e, cv<ST>(nw));
    } break;
    default:
      out_store<OHINT>(yout + e, cv<ST>(k));
  }
}

template <bool GHINT, typename T, typename ST, typename PT>
__device__ __forceinline__ void rk_update(int stage, double h, T k, PT ph, ST* acc, ST* yout,
                                          PT* phi, ST* shadow, size_t e) {
  const ST accv = (stage >= 1 && stage <= 3) ? acc_load<GHINT>(acc + e) : ST{};
  rk_finish<GHINT, false, T, ST, PT>(stage, h, k, ph, accv, acc, yout, phi, shadow, e);
}

// L2 cache policies for the hints above.
__device__ __forceinline__ unsigned long long policy_evict_first() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long policy_evict_last() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
// load of one stage-vector element with an L2 cache policy
__device__ __forceinline__ double2 ld_pol(const double2* p, unsigned long long pol) {
  double2 v;
  asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;\n"
               : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float2 ld_pol(const float2* p, unsigned long long pol) {
  float2 v;
  asm volatile("ld.global.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;\n"
               : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(pol));
  return v;
}

// Asynchronous global -> shared copies (cp.async, no register staging).
template <int BYTES>
__device__ __forceinline__ void cp_async(void* sdst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(gsrc), "n"(BYTES)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
// the same with an L2 cache policy
template <int BYTES>
__device__ __forceinline__ void cp_async_pol(void* sdst, const void* gsrc,
                                             unsigned long long pol) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;\n"
                 ::"r"(d), "l"(gsrc), "l"(pol) : "memory");
  else
    asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], %2, %3;\n"
                 ::"r"(d), "l"(gsrc), "n"(BYTES), "l"(pol) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Shared memory of k_wide: per warp, two buffers of one work item's streamed
// operands (phi, acc and the item's own row of Y; 32*NB trajectories each).
template <typename ST, typename PT, int NB>
constexpr size_t wide_smem_bytes(int warps) {
  return (size_t)warps * 2 * 32 * NB * (sizeof(PT) + 2 * sizeof(ST));
}

// ---------------------------------------------------- wide stage kernel ----
// B >= 32 trajectories: one warp per (aux a, state s, chunk of 32*NB
// trajectories); lane l owns the trajectories bg + l + 32 j, j < NB.
// Connection lists, coefficients and the site test are warp-uniform and loaded
// once per neighbour for the whole chunk; every Y load is a coalesced
// 32-trajectory segment and the NB loads per neighbour are in flight together.
// chunk_major (the task order):
//   0  tasks (a, s), s fastest; each warp walks every chunk of its (a, s);
//   1  the chunk is the outermost task index, so the warps in flight all
//      gather from one chunk's slice of Y (a slice of 32 trajectories of the
//      20-site ring is 54 MB in complex64);
//   2  chunk outermost, then the state s, the aux a fastest.  With site
//      projectors an item (a, s) gathers only rows (a +- e_k, s) and the
//      H-neighbour rows (a, s'), so the warps in flight touch a few state
//      slices of one chunk (10626 aux x 128 trajectories x 16 B = 22 MB each
//      on the 20-site ring): the up-gathers, which re-read every leaf row up
//      to four times, hit L2; the H-neighbour rows, adjacent in memory in
//      order 0, are read again one slice later;
//   3  chunk outermost, then the aux below st.n_up_prefix (those with up
//      connections) in order 2, then the others in order 0.  The gathers of
//      the interior aux run state by state against one slice of the leaf rows
//      (8855 leaves x 2 KB = 18 MB per state on the 20-site ring), while the
//      leaves, 83 % of the items, keep the sequential (aux, state) streaming
//      and their H rows' locality.
// The stage is bound by load latency at the occupancy registers allow.  NB <= 2
// is held to 64 registers (4 CTAs of 256 threads, 32 warps per SM), NB = 4 to
// 128 (4 CTAs of 128 threads); both measured faster than the registers the
// compiler would otherwise take.  NB = 8 is left nearly uncapped.
// Resident CTAs per SM that the NB = 4 stage kernel is compiled for (its
// register budget: 65536 / (128 threads x this) per thread).  4 is the
// fastest on the 20-site ring: 5 or 6 (96 / 80 registers, more warps, more of
// the SM's on-chip memory as shared memory) made the mixed-precision stage
// 1.4x / 1.8x slower, 3 (148 registers, 12 warps per SM) 1.24x slower.
#ifndef HOPS_WIDE_MIN_BLOCKS4
#define HOPS_WIDE_MIN_BLOCKS4 4
#endif
// CTA size of k_wide: 256 threads for NB <= 2, else 128 (finer occupancy
// steps at the register counts the wider tasks take).
constexpr int wide_threads(int nb) { return nb <= 2 ? 256 : 128; }

// Resident CTAs per SM of a shape.  With FP64 arithmetic the NB = 2 task holds
// twice the complex accumulators of the single-precision one: at 4 CTAs (64
// registers) it spilled; 3 CTAs leave it 85 registers.
constexpr int wide_min_blocks(int nb, int rbytes) {
  return nb == 1 ? 4 : (nb == 2 ? (rbytes == 8 ? 3 : 4) : (nb == 4 ? HOPS_WIDE_MIN_BLOCKS4 : 2));
}

// The work items of one stage, run by the calling CTA's warps (the body of
// k_wide and of the stage phases of the persistent step kernel).  wide_smem:
// the CTA's wide_smem_bytes of shared memory.  The persistent kernel passes
// pointers without __restrict__: its Y and stage coefficients are rewritten
// within the kernel, so they must not be read through the read-only path.
template <typename R, typename ST, typename PT, bool SITE, int NB, bool LT>
__device__ __forceinline__ void wide_items(const hops_structure& st, int B, int stage, double h,
                                           const ST* yin, ST* yout, PT* phi, ST* shadow, ST* acc,
                                           const double* ws, FastDiv divS, FastDiv divAS,
                                           FastDiv divH, FastDiv divP, unsigned n_pre_s,
                                           int chunk_major, unsigned char* wide_smem) {
  using P = Prec<R>;
  using T = typename P::T;
  const int S = st.n_state;
  const BatchLayout bl(S, st.n_mode, st.n_lop, B);
  const T* upcT = reinterpret_cast<const T*>(ws + (sizeof(R) == 8 ? bl.upcT : bl.upcT_f));
  const T* diagT = reinterpret_cast<const T*>(ws + (sizeof(R) == 8 ? bl.diagT : bl.diagT_f));
  const T* czT = reinterpret_cast<const T*>(ws + (sizeof(R) == 8 ? bl.czT : bl.czT_f));
  const double* ncB = ws + bl.ncB;
  const double* scaleB = ws + bl.scaleB;
  const int lane = threadIdx.x & 31;
  constexpr int CH = 32 * NB;
  const unsigned n_as = (unsigned)st.n_hier * (unsigned)S;
  const unsigned nchunk = (unsigned)((B + CH - 1) / CH);
  const unsigned ntask = chunk_major ? n_as * nchunk : n_as;
  const unsigned nw = (gridDim.x * blockDim.x) >> 5;

  // A work item is one (task, chunk).  The streamed operands of the warp's
  // next item are copied into shared memory while the current item gathers
  // its neighbours, so no item waits for its own DRAM reads.
  [[maybe_unused]] const unsigned long long pol_stream = policy_evict_first();
  [[maybe_unused]] const unsigned long long pol_keep = policy_evict_last();
  auto yl = [&](size_t i) -> ST {
    if constexpr ((HOPS_WIDE_HINTS & 2) != 0) return ld_pol(yin + i, pol_keep);
    else return yin[i];
  };
  // row index a * S + s of task t in chunk ci
  auto task_as = [&](unsigned t, unsigned ci) -> unsigned {
    const unsigned r = chunk_major ? t - ci * n_as : t;
    if (chunk_major == 2) {
      const unsigned sm = divH.div(r);
      return (r - sm * (unsigned)st.n_hier) * (unsigned)S + sm;
    }
    if (chunk_major == 3 && r < n_pre_s) {  // divP divides by the prefix length
      const unsigned sm = divP.div(r);
      return (r - sm * divP.d) * (unsigned)S + sm;
    }
    return r;
  };
  const int nwb = blockDim.x >> 5;
  const int wib = threadIdx.x >> 5;
  PT* ph_s = reinterpret_cast<PT*>(wide_smem) + (size_t)wib * 2 * CH;
  ST* ac_s = reinterpret_cast<ST*>(wide_smem + (size_t)nwb * 2 * CH * sizeof(PT)) +
             (size_t)wib * 2 * CH;
  ST* ys_s = reinterpret_cast<ST*>(wide_smem + (size_t)nwb * 2 * CH * (sizeof(PT) + sizeof(ST))) +
             (size_t)wib * 2 * CH;
  constexpr bool PSUM = psum_mode<ST, PT>();
  // fourth stage of the partial-sum form: P (re, im) in place of phi and acc
  const bool want_psum = PSUM && stage == 3;
  const bool want_phi = stage != 4 && !want_psum;
  const bool want_acc = stage >= 1 && stage <= 3 && !want_psum;
  auto prefetch = [&](unsigned t, unsigned ci, int buf) {
    const unsigned as = task_as(t, ci);
    const size_t row = (size_t)as * B;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const int b = (int)ci * CH + lane + 32 * j;
      if (b < B) {
        const int o = buf * CH + lane + 32 * j;
        if constexpr ((HOPS_WIDE_HINTS & 2) != 0) cp_async_pol<sizeof(ST)>(ys_s + o, yin + row + b, pol_keep);
        else cp_async<sizeof(ST)>(ys_s + o, yin + row + b);
        if constexpr ((HOPS_WIDE_HINTS & 1) != 0) {
          if (want_phi) cp_async_pol<sizeof(PT)>(ph_s + o, phi + row + b, pol_stream);
          if (want_acc) cp_async_pol<sizeof(ST)>(ac_s + o, acc + row + b, pol_stream);
        } else {
          if (want_phi) cp_async<sizeof(PT)>(ph_s + o, phi + row + b);
          if (want_acc) cp_async<sizeof(ST)>(ac_s + o, acc + row + b);
        }
        if constexpr (PSUM) {
          if (want_psum) {
            if constexpr (psum_split<ST, PT>()) {
              double* pd = reinterpret_cast<double*>(ph_s + o);
              cp_async<8>(pd, psum_re(acc) + row + b);
              cp_async<8>(pd + 1, psum_im(shadow) + row + b);
            } else {
              cp_async<sizeof(PT)>(ph_s + o, reinterpret_cast<const PT*>(acc) + row + b);
            }
          }
        }
      }
    }
  };

  unsigned t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  unsigned ci = (t < ntask && chunk_major) ? divAS.div(t) : 0u;
  if (t < ntask) prefetch(t, ci, 0);
  cp_async_commit();
  int buf = 0;
  while (t < ntask) {
    unsigned tn = t, cn = ci + 1;
    if (chunk_major || cn >= nchunk) {
      tn = t + nw;
      cn = (tn < ntask && chunk_major) ? divAS.div(tn) : 0u;
    }
    if (tn < ntask) prefetch(tn, cn, buf ^ 1);
    cp_async_commit();  // one group per item, empty past the last one

    const unsigned as = task_as(t, ci);
    const int a = (int)divS.div(as);
    const int s = (int)as - a * S;
    const size_t rowa = (size_t)as * B;
    const T kd = P::kdec(st, a);
    const int u0 = st.up_ptr[a], u1 = st.up_ptr[a + 1];
    const int d0 = st.dn_ptr[a], d1 = st.dn_ptr[a + 1];
    const int h0 = st.h_ptr[s], h1 = st.h_ptr[s + 1];
    const int bg = (int)ci * CH;
    cp_async_wait<1>();  // this item's copies have landed (each lane reads only its own)
    T k[NB];
    bool ok[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const int b = bg + lane + 32 * j;
      ok[j] = b < B;
      k[j] = czero<T>();
      if (ok[j]) {
        T c = kd;
        if (SITE) {
          c = cadd(c, diagT[(size_t)s * B + b]);
        } else {
          c.x -= (R)ncB[b];
        }
        k[j] = cmul(c, cv<T>(ys_s[buf * CH + lane + 32 * j]));
      }
    }
    if (!SITE) {
      for (int jl = 0; jl < st.n_lop; ++jl) {
        const int base = jl * (S + 1);
        const int q0 = st.l_ptr[base + s], q1 = st.l_ptr[base + s + 1];
        for (int q = q0; q < q1; ++q) {
          const T lv = P::lval(st, q);
          const size_t rb = ((size_t)a * S + st.l_col[q]) * B + bg + lane;
#pragma unroll
          for (int j = 0; j < NB; ++j)
            if (ok[j])
              k[j] = cfma(cmul(czT[(size_t)jl * B + bg + lane + 32 * j], lv), cv<T>(yl(rb + 32 * j)), k[j]);
        }
      }
    }
    for (int q = h0; q < h1; ++q) {
      const T hv = P::hval(st, q);
      const size_t rb = ((size_t)a * S + st.h_col[q]) * B + bg + lane;
#pragma unroll
      for (int j = 0; j < NB; ++j)
        if (ok[j]) k[j] = cfma(hv, cv<T>(yl(rb + 32 * j)), k[j]);
    }
    int p0 = u0;
    if (SITE) {
      // two neighbours per iteration: their 2 x NB row segments are loaded
      // before either is consumed, so twice as many loads are in flight
      for (; p0 + 2 <= u1; p0 += 2) {
        const int ua = __ldg(st.up_aux + p0), ma = __ldg(st.up_mode + p0);
        const int ub = __ldg(st.up_aux + p0 + 1), mb = __ldg(st.up_mode + p0 + 1);
        const int sa = __ldg(st.up_site + p0), sb = __ldg(st.up_site + p0 + 1);
        const size_t ra = ((size_t)ua * S + s) * B + bg + lane;
        const size_t rb = ((size_t)ub * S + s) * B + bg + lane;
        ST ya[NB], yb[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j) {
          if (ok[j]) {
            ya[j] = yl(ra + 32 * j);
            yb[j] = yl(rb + 32 * j);
          }
        }
        const T* upa = upcT + (size_t)ma * B + bg + lane;
        const T* upb = upcT + (size_t)mb * B + bg + lane;
        const T corra = sa == s ? P::gwv(st, ma) : czero<T>();
        const T corrb = sb == s ? P::gwv(st, mb) : czero<T>();
#pragma unroll
        for (int j = 0; j < NB; ++j) {
          if (ok[j]) {
            k[j] = cfma(csub(upa[32 * j], corra), cv<T>(ya[j]), k[j]);
            k[j] = cfma(csub(upb[32 * j], corrb), cv<T>(yb[j]), k[j]);
          }
        }
      }
    }
    for (int p = p0; p < u1; ++p) {
      const int u = st.up_aux[p], m = st.up_mode[p];
      const size_t rb = ((size_t)u * S + s) * B + bg + lane;
      const T* up = upcT + (size_t)m * B + bg + lane;
      if (SITE) {
        const bool hit = st.up_site[p] == s;
        const T corr = hit ? P::gwv(st, m) : czero<T>();
#pragma unroll
        for (int j = 0; j < NB; ++j)
          if (ok[j]) k[j] = cfma(csub(up[32 * j], corr), cv<T>(yl(rb + 32 * j)), k[j]);
      } else {
#pragma unroll
        for (int j = 0; j < NB; ++j)
          if (ok[j]) k[j] = cfma(up[32 * j], cv<T>(yl(rb + 32 * j)), k[j]);
        const int base = st.mode_lop[m] * (S + 1);
        const int q0 = st.l_ptr[base + s], q1 = st.l_ptr[base + s + 1];
        for (int q = q0; q < q1; ++q) {
          const T lv = cmul(P::gw(st, m), P::lval(st, q));
          const size_t rb2 = ((size_t)u * S + st.l_col[q]) * B + bg + lane;
#pragma unroll
          for (int j = 0; j < NB; ++j)
            if (ok[j]) k[j] = csub(k[j], cmul(lv, cv<T>(yl(rb2 + 32 * j))));
        }
      }
    }
    for (int p = d0; p < d1; ++p) {
      if (SITE) {
        if (__ldg(st.dn_site + p) != s) continue;
        const int d = __ldg(st.dn_aux + p);
        const T cf = P::dncs(st, p);
        const size_t rb = ((size_t)d * S + s) * B + bg + lane;
#pragma unroll
        for (int j = 0; j < NB; ++j)
          if (ok[j]) k[j] = cfma(cf, cv<T>(yl(rb + 32 * j)), k[j]);
      } else {
        const int d = st.dn_aux[p], m = st.dn_mode[p];
        const int base = st.mode_lop[m] * (S + 1);
        const int q0 = st.lh_ptr[base + s], q1 = st.lh_ptr[base + s + 1];
        for (int q = q0; q < q1; ++q) {
          const T cf = cmul(P::dncoef(st, p), P::lhval(st, q));
          const size_t rb = ((size_t)d * S + st.lh_col[q]) * B + bg + lane;
#pragma unroll
          for (int j = 0; j < NB; ++j)
            if (ok[j]) k[j] = cfma(cf, cv<T>(yl(rb + 32 * j)), k[j]);
        }
      }
    }
    PT ph[NB];
    ST accv[NB];
    double sc[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const int o = buf * CH + lane + 32 * j;
      ph[j] = PT{};
      accv[j] = ST{};
      sc[j] = 1.0;
      if (!ok[j]) continue;
      sc[j] = scaleB[bg + lane + 32 * j];
      if (want_phi || want_psum) ph[j] = ph_s[o];
      if (want_acc) accv[j] = ac_s[o];
    }
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      if (!ok[j]) continue;
      const size_t e = rowa + bg + lane + 32 * j;
      T kk = k[j];
      if (stage == 0 || stage == 4) kk = cscale(kk, (R)sc[j]);
      if (LT && a == 0) {  // LT term of psi_0 (computed from the scaled state)
        if constexpr (sizeof(R) == 8) kk = cadd(kk, ld2(ws + bl.physT, s * B + bg + lane + 32 * j));
        else kk = cadd(kk, ld2f(reinterpret_cast<const float*>(ws + bl.physT_f), s * B + bg + lane + 32 * j));
      }
      // P was formed from the scaled state: no scale at the partial-sum stage
      const PT p = stage == 4 ? PT{} : (want_psum ? ph[j] : cscale(ph[j], (decltype(PT{}.x))sc[j]));
      rk_finish<true, PSUM, T, ST, PT, (HOPS_WIDE_HINTS & 1) != 0>(stage, h, kk, p, accv[j], acc,
                                                                  yout, phi, shadow, e);
    }
    t = tn;
    ci = cn;
    buf ^= 1;
  }
  cp_async_wait<0>();
}

template <typename R, typename ST, typename PT, bool SITE, int NB, bool LT>
__global__ void __launch_bounds__(wide_threads(NB), wide_min_blocks(NB, sizeof(R)))
    k_wide(hops_structure st, int B, int stage, double h, const ST* __restrict__ yin,
           ST* __restrict__ yout, PT* phi, ST* shadow, ST* acc, const double* __restrict__ ws,
           FastDiv divS, FastDiv divAS, FastDiv divH, FastDiv divP, unsigned n_pre_s,
           int chunk_major) {
  extern __shared__ __align__(16) unsigned char wide_smem[];
  pdl_enter();
  wide_items<R, ST, PT, SITE, NB, LT>(st, B, stage, h, yin, yout, phi, shadow, acc, ws, divS,
                                      divAS, divH, divP, n_pre_s, chunk_major, wide_smem);
}


// -------------------------------------------------- narrow stage kernel ----
// B < 32 trajectories: one warp per aux a (warp-uniform connection lists),
// lanes over the S*B elements (state s, trajectory b) of that aux.
// MINB: resident CTAs per SM the kernel is compiled for.  Complex128 stage
// vectors on aux of >= 64 elements (large single trajectories) run with
// MINB = 5 (48 registers, 40 warps per SM), everything else with MINB = 4
// (64 registers).  Stage launch, ms, MINB 4 / 5 / 6: 120-site chain depth 3
// complex128 1.054 / 1.019 / 1.029, mixed 0.969 / 0.954 / 0.994; 200-site
// chain complex128 8.84 / 8.45 / 8.56, mixed 7.90 / 7.99 / 8.24; the
// one-trajectory 20-site ring (20 elements per aux) is unaffected.
#ifndef HOPS_NARROW_BIG_MINB
#define HOPS_NARROW_BIG_MINB 5
#endif
template <typename R, typename ST, typename PT, bool SITE, int MINB>
__global__ void __launch_bounds__(256, MINB) k_narrow(hops_structure st, int B, int stage, double h,
                                                const ST* __restrict__ yin,
                                                ST* __restrict__ yout, PT* phi, ST* shadow,
                                                ST* acc, const double* __restrict__ ws,
                                                FastDiv divB) {
  using T = typename Prec<R>::T;
  pdl_enter();
  const int S = st.n_state;
  const int SB = S * B;
  const BatchLayout bl(S, st.n_mode, st.n_lop, B);
  const double* scaleB = ws + bl.scaleB;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < st.n_hier; a += nw) {
    for (int r = lane; r < SB; r += 32) {
      const int s = (int)divB.div((unsigned)r);
      const int b = r - s * B;
      const size_t e = (size_t)a * SB + r;
      // the element's own streamed operands first: their DRAM latency then
      // overlaps the neighbour gather instead of following it; the fourth
      // stage of the partial-sum form reads P (already scaled) instead
      constexpr bool PSUM = psum_mode<ST, PT>();
      const bool want_psum = PSUM && stage == 3;
      PT ph0 = PT{};
      if (want_psum) {
        if constexpr (psum_split<ST, PT>())
          ph0 = PT{__ldcs(psum_re(acc) + e), __ldcs(psum_im(shadow) + e)};
        else if constexpr (PSUM)
          ph0 = __ldcs(reinterpret_cast<const PT*>(acc) + e);
      } else if (stage != 4) {
        ph0 = phi[e];
      }
      const ST accv = (stage >= 1 && stage <= 3 && !want_psum) ? acc_load<true>(acc + e) : ST{};
      const double sc = scaleB[b];
      auto y = [&](int x, int sp) { return cv<T>(yin[((size_t)x * S + sp) * B + b]); };
      const CoefT<R> cf{ws, bl, B, b};
      T k = deriv_elem<R, SITE>(st, a, s, y, cf);
      if (stage == 0 || stage == 4) k = cscale(k, (R)sc);
      if (st.lt_coef && a == 0) k = cadd(k, cf.phys(s));  // LT term of psi_0 (already scaled)
      const PT ph = want_psum ? ph0 : cscale(ph0, (decltype(PT{}.x))sc);
      rk_finish<true, PSUM, T, ST, PT>(stage, h, k, ph, accv, acc, yout, phi, shadow, e);
    }
  }
}

// ----------------------------------------------- streaming scalar kernel ----
// One CTA per trajectory b: FP64 stage scalars (stage_scalars) of stage
// `stage`, then published in trajectory-fastest layout for the stage kernels.
// Stage 0 / 4 read the state phi (precision PT) with the pending scale; the
// other stages read the stage input (precision T).  With recompute_scale the
// CTA first renormalises the state produced by the previous step
// (hops_trajectory.py:616-634) by recording 1/||psi_0||, which every stage
// kernel applies on the fly.
__device__ void publish(const hops_structure& st, const BatchLayout& bl, double* wsall, int B,
                        int b, const double* ws) {
  const int S = st.n_state, M = st.n_mode, L = st.n_lop;
  const ScalarLayout lay(S, M, L);
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    double2 v = ld2(ws + lay.upc(), m);
    reinterpret_cast<double2*>(wsall + bl.upcT)[(size_t)m * B + b] = v;
    reinterpret_cast<float2*>(wsall + bl.upcT_f)[(size_t)m * B + b] = mkf((float)v.x, (float)v.y);
  }
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double2 v = ld2(ws + lay.diagD(), s);
    reinterpret_cast<double2*>(wsall + bl.diagT)[(size_t)s * B + b] = v;
    reinterpret_cast<float2*>(wsall + bl.diagT_f)[(size_t)s * B + b] = mkf((float)v.x, (float)v.y);
  }
  for (int j = threadIdx.x; j < L; j += blockDim.x) {
    double2 v = ld2(ws + lay.cz(), j);
    reinterpret_cast<double2*>(wsall + bl.czT)[(size_t)j * B + b] = v;
    reinterpret_cast<float2*>(wsall + bl.czT_f)[(size_t)j * B + b] = mkf((float)v.x, (float)v.y);
  }
  if (st.lt_coef)
    for (int s = threadIdx.x; s < S; s += blockDim.x) {
      double2 v = ld2(ws + lay.phys(), s);
      reinterpret_cast<double2*>(wsall + bl.physT)[(size_t)s * B + b] = v;
      reinterpret_cast<float2*>(wsall + bl.physT_f)[(size_t)s * B + b] = mkf((float)v.x, (float)v.y);
    }
  if (threadIdx.x == 0) {
    wsall[bl.ncB + b] = ws[lay.nc()];
    wsall[bl.scaleB + b] = ws[lay.scale()];
  }
}

// The stage scalars of trajectory b, computed by the calling CTA (all its
// threads; shm: the CTA's scalar shared memory, scalar_smem / scalar_smem_rows
// bytes).  Used by k_scalars (one CTA per trajectory) and by the persistent
// step kernel.
template <typename R, typename ST, typename PT>
__device__ __forceinline__ void scalars_cta(const hops_structure& st, const hops_batch& bt, int b,
                                            int stage, int it, double h, const void* yin,
                                            int recompute_scale, double* psi_prev,
                                            const float* z1s, const float* z2s, double* dz_out,
                                            int stage_rows, double* shm) {
  using T = typename Prec<R>::T;
  double* red = shm;
  double* sh = shm + 32;
  const int S = st.n_state, M = st.n_mode, L = st.n_lop, B = bt.n_traj;
  const ScalarLayout lay(S, M, L);
  const BatchLayout bl(S, M, L, B);
  double* ws = bt.work + (size_t)b * lay.stride;
  const PT* ph = static_cast<const PT*>(bt.phi);
  if (recompute_scale || psi_prev) {
    double sc = ws[lay.scale()];
    if (recompute_scale) {
      double p = 0.0;
      for (int s = threadIdx.x; s < S; s += blockDim.x) {
        double2 v = to_d(ph[(size_t)s * B + b]);
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
        reinterpret_cast<double2*>(psi_prev)[(size_t)b * S + s] = cscale(to_d(ph[(size_t)s * B + b]), sc);
    __syncthreads();
  }
  const bool from_phi = stage == 0 || stage == 4;
  const double sc = from_phi ? ws[lay.scale()] : 1.0;
  StageIO io;
  io.zmem = bt.zmem + (size_t)b * M * 2;
  if (stage == 4) {
    io.noise1 = z1s ? reinterpret_cast<const float2*>(z1s) + (size_t)b * L : nullptr;
    io.noise2 = z2s ? reinterpret_cast<const float2*>(z2s) + (size_t)b * L : nullptr;
    io.n_t1 = 1;
    io.n_t2 = 1;
    io.noise_c128 = 0;
    io.it = 0;
    io.zmem_out = dz_out + (size_t)b * M * 2;
  } else {
    const size_t esz = bt.noise_c128 ? 16 : 8;
    io.noise1 = bt.noise1 ? reinterpret_cast<const char*>(bt.noise1) + (size_t)b * L * bt.n_t1 * esz
                          : nullptr;
    io.noise2 = bt.noise2 ? reinterpret_cast<const char*>(bt.noise2) + (size_t)b * L * bt.n_t2 * esz
                          : nullptr;
    io.n_t1 = bt.n_t1;
    io.n_t2 = bt.n_t2;
    io.noise_c128 = bt.noise_c128;
    io.it = it;
    io.zmem_out = bt.zmem + (size_t)b * M * 2;
  }
  io.stage = stage;
  io.eom = bt.eom;
  io.h = h;
  io.ws = ws;
  const ST* y = static_cast<const ST*>(yin);
  auto get = [&](int a, int s) -> double2 {
    const size_t i = ((size_t)a * S + s) * B + b;
    return from_phi ? cscale(to_d(ph[i]), sc) : to_d(y[i]);
  };
  if (stage_rows) {
    // The rows the scalars read (psi_0 and the first-order aux) are loaded
    // once, all in flight together, instead of by dependent loads in the
    // per-mode loops.
    double2* rows = reinterpret_cast<double2*>(sh + 4 * L + 2);
    const int nr = (1 + st.n_first) * S;
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
      const int f = i / S, r = i - f * S;
      rows[i] = get(f == 0 ? 0 : st.first_aux[f - 1], r);
    }
    __syncthreads();
    stage_scalars(
        st, io, [&](int a, int r) { return a == 0 ? rows[r] : get(a, r); },
        [&](int f, int r) { return rows[(size_t)(f + 1) * S + r]; }, red, sh);
  } else {
    stage_scalars(st, io, get, red, sh);
  }
  publish(st, bl, bt.work, B, b, ws);
}

template <typename R, typename ST, typename PT>
__global__ void __launch_bounds__(128) k_scalars(hops_structure st, hops_batch bt, int stage, int it,
                                                 double h, const void* yin, int recompute_scale,
                                                 double* psi_prev, const float* z1s,
                                                 const float* z2s, double* dz_out, int stage_rows) {
  extern __shared__ double shm[];
  pdl_wait();
  scalars_cta<R, ST, PT>(st, bt, blockIdx.x, stage, it, h, yin, recompute_scale, psi_prev, z1s,
                         z2s, dz_out, stage_rows, shm);
  pdl_trigger();
}

// --------------------------------------------- persistent step kernel ----
// One cooperative launch runs every RK4 step of a call: for each stage the
// stage scalars of every trajectory (CTA b mod gridDim, as k_scalars), a grid
// barrier, the stage's work items (wide_items), a grid barrier.  It replaces
// the 8 launches per step of the separate kernels and the gaps between them.
//
// Grid barrier: bar[0] counts arrivals, bar[1] is the generation, bar[2] the
// error word.  The last CTA to arrive resets the count and bumps the
// generation; the others wait on the generation with a time limit (limit_ns
// of %globaltimer; HOPS_BARRIER_NS in the step kernel), after which they set
// the error word and return; a CTA that sees the error word set returns too.
// The host zeroes bar before the launch.  A cooperative launch guarantees
// that every CTA is resident, so the barrier cannot wait on a CTA that never
// runs.  The longest phase between two barriers is one stage (~0.5 ms on the
// 20-site ring at 128 trajectories, tens of ms for the largest batches).
#ifndef HOPS_BARRIER_NS
#define HOPS_BARRIER_NS 2000000000ull
#endif
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Relaxed (not acquire) load for the polling: an acquire at gpu scope
// invalidates the SM's L1, and a CTA polling with acquires kept emptying the
// L1 of the CTAs still working on its SM (1.7x the instructions and half the
// L1 hit rate of the separate launches).  One fence after the wait acquires.
__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// false: the barrier failed (time limit, or another CTA's failure)
__device__ __forceinline__ bool grid_sync(unsigned* bar, unsigned& gen,
                                          unsigned long long limit_ns = HOPS_BARRIER_NS) {
  __shared__ unsigned ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned ok = 1;
    __threadfence();  // this CTA's writes before the arrival
    const unsigned g = gen;
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicExch(bar + 1, g + 1u);
    } else {
      const unsigned long long t0 = global_ns();
      unsigned ns = 32;
      while (ld_relaxed_u32(bar + 1) == g) {
        if (ld_relaxed_u32(bar + 2) != 0u) {
          ok = 0;
          break;
        }
        if (global_ns() - t0 > limit_ns) {
          atomicExch(bar + 2, 1u);
          ok = 0;
          break;
        }
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
      }
    }
    __threadfence();  // acquire: the other CTAs' writes before the barrier are seen
    if (ld_relaxed_u32(bar + 2) != 0u) ok = 0;
    ok_s = ok;
  }
  ++gen;
  __syncthreads();
  return ok_s != 0u;
}

// Self-test of the grid barrier: every CTA but `absent` passes n_sync
// barriers; out[c] = 1 if CTA c passed them all, 0 if one failed (time limit
// or another CTA's failure), 2 for the absent CTA, which returns at once.
__global__ void k_barrier_test(unsigned* bar, int32_t* out, int n_sync, int absent,
                               unsigned long long limit_ns) {
  if ((int)blockIdx.x == absent) {
    if (threadIdx.x == 0) out[blockIdx.x] = 2;
    return;
  }
  unsigned gen = 0;
  bool ok = true;
  for (int i = 0; i < n_sync && ok; ++i) ok = grid_sync(bar, gen, limit_ns);
  if (threadIdx.x == 0) out[blockIdx.x] = ok ? 1 : 0;
}

#ifndef HOPS_PERSIST_NOINLINE
#define HOPS_PERSIST_NOINLINE 0
#endif
#if HOPS_PERSIST_NOINLINE
// The stage phase as a call: the callee gets the register budget of the
// kernel, the caller's few live values are saved across it.
template <typename R, typename ST, typename PT, bool SITE, int NB, bool LT>
__device__ __noinline__ void wide_phase(const hops_structure& st, const hops_batch& bt, int i,
                                        double h, FastDiv divS, FastDiv divAS, FastDiv divH,
                                        FastDiv divP, unsigned n_pre_s, int chunk_major,
                                        unsigned char* smem) {
  ST* shadow = bt.precision == HOPS_PREC_MIXED ? static_cast<ST*>(bt.phi_lo) : nullptr;
  const void* yin = i == 0 ? (shadow ? static_cast<const void*>(shadow) : bt.phi)
                           : (i == 1 ? bt.y0 : (i == 2 ? bt.y1 : bt.y0));
  void* yout = i == 0 ? bt.y0 : (i == 1 ? bt.y1 : (i == 2 ? bt.y0 : nullptr));
  wide_items<R, ST, PT, SITE, NB, LT>(st, bt.n_traj, i, h, static_cast<const ST*>(yin),
                                      static_cast<ST*>(yout), static_cast<PT*>(bt.phi), shadow,
                                      static_cast<ST*>(bt.acc), bt.work, divS, divAS, divH, divP,
                                      n_pre_s, chunk_major, smem);
}
#define HOPS_PERSIST_PARAM const __grid_constant__
#else
#define HOPS_PERSIST_PARAM
#endif

// The step loop keeps one counter q = 4 n + i live across the stage phase;
// everything else is recomputed from the kernel parameters, so the stage
// phase has (nearly) the register budget of k_wide.
template <typename R, typename ST, typename PT, bool SITE, int NB, bool LT>
__global__ void __launch_bounds__(wide_threads(NB), wide_min_blocks(NB, sizeof(R)))
    k_persist(HOPS_PERSIST_PARAM hops_structure st, HOPS_PERSIST_PARAM hops_batch bt, int it0,
              int di, int n_steps, double h, double* psi_out, int stage_rows, FastDiv divS,
              FastDiv divAS, FastDiv divH, FastDiv divP, unsigned n_pre_s, int chunk_major) {
  extern __shared__ __align__(16) unsigned char pers_smem[];
  for (int q = 0; q < 4 * n_steps; ++q) {
    const int n = q >> 2, i = q & 3;
    const int B = bt.n_traj;
    unsigned* bar = reinterpret_cast<unsigned*>(
        bt.work + BatchLayout(st.n_state, st.n_mode, st.n_lop, B).bar);
    unsigned gen = 2u * (unsigned)q;
    {
      ST* shadow = bt.precision == HOPS_PREC_MIXED ? static_cast<ST*>(bt.phi_lo) : nullptr;
      const int it = it0 + 2 * n * di + rk_noise_slot(i) * di;
      // stage 0 gathers from the state (or its complex64 copy in mixed mode)
      const void* yin = i == 0 ? (shadow ? static_cast<const void*>(shadow) : bt.phi)
                               : (i == 1 ? bt.y0 : (i == 2 ? bt.y1 : bt.y0));
      const int recompute = (i == 0 && n > 0 && bt.eom == HOPS_EOM_NORMALIZED_NONLINEAR) ? 1 : 0;
      double* psi_prev = (i == 0 && n > 0 && psi_out)
                             ? psi_out + (size_t)(n - 1) * (size_t)B * st.n_state * 2
                             : nullptr;
      for (int b = blockIdx.x; b < B; b += gridDim.x) {
        scalars_cta<R, ST, PT>(st, bt, b, i, it, h, yin, recompute, psi_prev, nullptr, nullptr,
                               nullptr, stage_rows, reinterpret_cast<double*>(pers_smem));
        __syncthreads();  // the next trajectory reuses the shared memory
      }
    }
    bool ok = grid_sync(bar, gen);
    if (ok) {
#if HOPS_PERSIST_NOINLINE
      wide_phase<R, ST, PT, SITE, NB, LT>(st, bt, i, h, divS, divAS, divH, divP, n_pre_s,
                                          chunk_major, pers_smem);
#else
      ST* shadow = bt.precision == HOPS_PREC_MIXED ? static_cast<ST*>(bt.phi_lo) : nullptr;
      const void* yin = i == 0 ? (shadow ? static_cast<const void*>(shadow) : bt.phi)
                               : (i == 1 ? bt.y0 : (i == 2 ? bt.y1 : bt.y0));
      void* yout = i == 0 ? bt.y0 : (i == 1 ? bt.y1 : (i == 2 ? bt.y0 : nullptr));
      wide_items<R, ST, PT, SITE, NB, LT>(st, B, i, h, static_cast<const ST*>(yin),
                                          static_cast<ST*>(yout), static_cast<PT*>(bt.phi),
                                          shadow, static_cast<ST*>(bt.acc), bt.work, divS, divAS,
                                          divH, divP, n_pre_s, chunk_major, pers_smem);
#endif
      bar = reinterpret_cast<unsigned*>(
          bt.work + BatchLayout(st.n_state, st.n_mode, st.n_lop, bt.n_traj).bar);
      ok = grid_sync(bar, gen);
    }
    if (!ok) {  // every trajectory of this CTA ends with the timeout status
      if (threadIdx.x == 0)
        for (int b = blockIdx.x; b < bt.n_traj; b += gridDim.x) bt.status[b] = HOPS_ETIMEOUT;
      return;
    }
  }
}


// Normalisation after the last step of a call: records 1/||psi_0|| per
// trajectory and writes the last psi_0.
template <typename PT>
__global__ void __launch_bounds__(128) k_finalize(hops_structure st, hops_batch bt, double* psi_last,
                                                  int normalize) {
  __shared__ double red[32];
  const int b = blockIdx.x, S = st.n_state, B = bt.n_traj;
  const ScalarLayout lay(S, st.n_mode, st.n_lop);
  const BatchLayout bl(S, st.n_mode, st.n_lop, B);
  double* ws = bt.work + (size_t)b * lay.stride;
  const PT* ph = static_cast<const PT*>(bt.phi);
  double sc = 1.0;
  if (normalize) {
    double p = 0.0;
    for (int s = threadIdx.x; s < S; s += blockDim.x) {
      double2 v = to_d(ph[(size_t)s * B + b]);
      p += v.x * v.x + v.y * v.y;
    }
    const double n2 = block_sum(p, red);
    sc = 1.0 / sqrt(n2);
    if (!(n2 > 0.0) || !isfinite(sc)) {
      if (threadIdx.x == 0) bt.status[b] = HOPS_ENONFINITE;
      sc = 1.0;
    }
  }
  if (threadIdx.x == 0) {
    ws[lay.scale()] = sc;
    bt.work[bl.scaleB + b] = sc;
  }
  if (psi_last)
    for (int s = threadIdx.x; s < S; s += blockDim.x)
      reinterpret_cast<double2*>(psi_last)[(size_t)b * S + s] = cscale(to_d(ph[(size_t)s * B + b]), sc);
}

template <typename PT, typename T>
__global__ void k_apply_scale(PT* phi, T* shadow, int B, size_t E, const double* scaleB) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < E;
       e += (size_t)gridDim.x * blockDim.x) {
    const PT v = cscale(phi[e], (decltype(PT{}.x))scaleB[e % B]);
    phi[e] = v;
    if (shadow) shadow[e] = cv<T>(v);
  }
}

__global__ void k_reset(double* ws, int stride, size_t scale_off, int B, int32_t* status,
                        int clear_status) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < B) {
    ws[(size_t)b * stride] = 1.0;
    ws[scale_off + b] = 1.0;
    if (clear_status && status) status[b] = 0;
  }
}

// --------------------------------------------------------- resident kernel ----
// One CTA owns one trajectory for all n_steps steps: stage scalars, the four
// RK stages and the renormalisation run back to back with only __syncthreads
// between them (no grid-wide synchronisation).  Vectors live in shared memory
// when they fit (mode 2: phi, acc, y0, y1; mode 1: y0, y1), else in the task's
// scratch.  Tasks may carry different structures (uneven adaptive bases).
template <typename R, typename ST, typename PT, bool SITE>
__global__ void __launch_bounds__(512, 1) k_resident(hops_task* tasks, int mode, int max_elems,
                                                     int sc_doubles) {
  using T = typename Prec<R>::T;
  using RP = decltype(PT{}.x);
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
  unsigned char* vbase = smraw + (size_t)sc_doubles * sizeof(double);
  PT* gphi = static_cast<PT*>(tk->phi);
  PT* phi;
  ST *acc, *y0, *y1;
  if (mode == 2) {
    phi = reinterpret_cast<PT*>(vbase);
    ST* v = reinterpret_cast<ST*>(vbase + (size_t)max_elems * sizeof(PT));
    acc = v;
    y0 = v + max_elems;
    y1 = v + 2 * max_elems;
  } else if (mode == 1) {
    y0 = reinterpret_cast<ST*>(vbase);
    y1 = y0 + max_elems;
    phi = gphi;
    acc = static_cast<ST*>(tk->scratch);
  } else {
    phi = gphi;
    acc = static_cast<ST*>(tk->scratch);
    y0 = acc + E;
    y1 = acc + 2 * E;
  }
  const RP sc0 = (RP)tk->scale;
  for (int e = threadIdx.x; e < E; e += blockDim.x) phi[e] = cscale(gphi[e], sc0);
  for (int m = threadIdx.x; m < M; m += blockDim.x)
    reinterpret_cast<double2*>(zm)[m] = reinterpret_cast<const double2*>(tk->zmem)[m];
  __syncthreads();
  const bool normalized = tk->eom == HOPS_EOM_NORMALIZED_NONLINEAR;
  int status = 0;
  StageIO io;
  io.zmem = zm;
  io.zmem_out = zm;
  io.noise1 = tk->noise1;
  io.noise2 = tk->noise2;
  io.n_t1 = tk->n_t1;
  io.n_t2 = tk->n_t2;
  io.noise_c128 = tk->noise_c128;
  io.eom = tk->eom;
  io.h = tk->tau_over_hbar;
  io.ws = ws;
  const CoefWS<R> cf{ws, lay};
  for (int n = 0; n < tk->n_steps; ++n) {
    for (int stage = 0; stage < 4; ++stage) {
      const ST* yin = stage == 1 ? y0 : (stage == 2 ? y1 : y0);
      ST* yout = stage == 0 ? y0 : (stage == 1 ? y1 : (stage == 2 ? y0 : nullptr));
      io.it = tk->it0 + 2 * n * tk->di + rk_noise_slot(stage) * tk->di;
      io.stage = stage;
      if (stage == 0) {
        auto get = [&](int a, int s) -> double2 { return to_d(phi[a * S + s]); };
        stage_scalars(st, io, get, red, sh);
        auto y = [&](int x, int sp) { return cv<T>(phi[x * S + sp]); };
        for (int e = threadIdx.x; e < E; e += blockDim.x) {
          const int a = e / S, s = e - a * S;
          T k = deriv_elem<R, SITE>(st, a, s, y, cf);
          if (st.lt_coef && a == 0) k = cadd(k, cf.phys(s));  // LT term of psi_0
          rk_update<false, T, ST, PT>(stage, io.h, k, phi[e], acc, yout, phi, (ST*)nullptr, (size_t)e);
        }
      } else {
        auto get = [&](int a, int s) -> double2 { return to_d(yin[a * S + s]); };
        stage_scalars(st, io, get, red, sh);
        auto y = [&](int x, int sp) { return cv<T>(yin[x * S + sp]); };
        for (int e = threadIdx.x; e < E; e += blockDim.x) {
          const int a = e / S, s = e - a * S;
          T k = deriv_elem<R, SITE>(st, a, s, y, cf);
          if (st.lt_coef && a == 0) k = cadd(k, cf.phys(s));  // LT term of psi_0
          rk_update<false, T, ST, PT>(stage, io.h, k, phi[e], acc, yout, phi, (ST*)nullptr, (size_t)e);
        }
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
      for (int e = threadIdx.x; e < E; e += blockDim.x) phi[e] = cscale(phi[e], (RP)sc);
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

// Optional CUDA-event timing of the stage kernels (profiling aid; one host
// thread at a time).  Each stage-kernel launch is bracketed by two events on
// its stream; hops_kernel_timing_read sums the elapsed times.
static bool g_timing = false;
static std::vector<cudaEvent_t> g_ev;
static size_t g_ev_used = 0;

static cudaEvent_t timing_event() {
  if (g_ev_used == g_ev.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    g_ev.push_back(e);
  }
  return g_ev[g_ev_used++];
}

extern "C" int hops_kernel_timing(int enable) {
  g_timing = enable != 0;
  g_ev_used = 0;
  return HOPS_OK;
}

extern "C" int hops_kernel_timing_read(double* total_ms, int64_t* n_launches) {
  double tot = 0.0;
  int64_t n = 0;
  for (size_t i = 0; i + 1 < g_ev_used; i += 2) {
    float ms = 0.f;
    CUDA_TRY(cudaEventSynchronize(g_ev[i + 1]));
    CUDA_TRY(cudaEventElapsedTime(&ms, g_ev[i], g_ev[i + 1]));
    tot += ms;
    ++n;
  }
  if (total_ms) *total_ms = tot;
  if (n_launches) *n_launches = n;
  g_ev_used = 0;
  return HOPS_OK;
}

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
  if ((long)st->n_hier * st->n_state >= (1L << 31))
    return set_err(HOPS_ENOTSUP, "n_hier * n_state must be below 2^31");
  if (!st->k_decay || !st->up_ptr || !st->dn_ptr || !st->h_ptr || !st->l_ptr || !st->lop_active)
    return set_err(HOPS_EINVAL, "structure has null tables");
  if (st->site_projector && (!st->lop_site || !st->lop_sval || !st->mode_site || !st->mode_gwv ||
                             !st->mode_gwv_f || !st->dn_coef_site || !st->dn_coef_site_f))
    return set_err(HOPS_EINVAL, "site-projector structure without its site tables");
  return HOPS_OK;
}

static int check_batch(const hops_structure* st, const hops_batch* bt) {
  if (!bt) return set_err(HOPS_EINVAL, "null batch");
  if (bt->n_traj <= 0) return set_err(HOPS_EINVAL, "n_traj must be positive");
  if (bt->precision != HOPS_PREC_C128 && bt->precision != HOPS_PREC_C64 &&
      bt->precision != HOPS_PREC_MIXED)
    return set_err(HOPS_EINVAL, "unknown precision %d", bt->precision);
  if (bt->eom < 0 || bt->eom > 2) return set_err(HOPS_EINVAL, "unknown eom %d", bt->eom);
  if (!bt->phi || !bt->acc || !bt->y0 || !bt->y1 || !bt->zmem || !bt->work || !bt->status)
    return set_err(HOPS_EINVAL, "batch has null buffers");
  if (bt->precision == HOPS_PREC_MIXED && !bt->phi_lo)
    return set_err(HOPS_EINVAL, "mixed-precision batch needs phi_lo");
  if (bt->precision != HOPS_PREC_C128 &&
      (!st->k_decay_f || !st->dn_coef_f || !st->mode_gw_f || !st->h_val_f || !st->l_val_f ||
       !st->lh_val_f))
    return set_err(HOPS_EINVAL, "complex64 batch needs the float coefficient tables");
  if ((long)st->n_hier * st->n_state * bt->n_traj >= (1L << 40))
    return set_err(HOPS_ENOTSUP, "batch too large");
  return HOPS_OK;
}

static int grid_for_warps(long warps) {
  long blocks = (warps * 32 + 255) / 256;
  const long cap = (long)sm_count() * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

// Stage-kernel shape: trajectories per chunk (32 * nb) and chunk-major order.
// 0 = choose automatically; set by hops_stage_tuning (the autotuner).
static int g_tune_nb = 0, g_tune_cm = -1;
// Step fusion: 0 = automatic (separate launches), 1 = separate scalar and
// stage launches, 2 = the persistent step kernel (batches of >= 32
// trajectories at 128 trajectories per task); set by hops_step_fusion.  The
// persistent kernel is exact (bit for bit the numbers of the separate
// launches) but slower on the 20-site ring at 128 trajectories: 4.1 against
// 2.0 ms per complex128 step, 2.5 against 1.7 mixed, 1.6 against 1.3
// complex64.  Its stage phases run 2.1x slower than k_wide's with the scalar
// phase's code in the same kernel (1.23x without it); the scalar phase,
// serial between two barriers, takes ~0.1 ms per stage against ~0.02 ms
// for k_scalars; the barriers themselves cost ~1 us.
static int g_fusion = 0;

extern "C" int hops_grid_barrier_test(uint32_t* bar, int32_t* out, int32_t n_ctas,
                                      int32_t n_sync, int32_t absent, int64_t limit_ns,
                                      void* stream) {
  if (!bar || !out || n_ctas < 1 || n_ctas > sm_count() || n_sync < 0 || limit_ns <= 0)
    return set_err(HOPS_EINVAL, "grid barrier test: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  CUDA_TRY(cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned), s));
  unsigned* b = bar;
  int32_t* o = out;
  int ns = n_sync, ab = absent;
  unsigned long long lim = (unsigned long long)limit_ns;
  void* args[] = {&b, &o, &ns, &ab, &lim};
  CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_barrier_test, dim3(n_ctas), dim3(128), args,
                                       0, s));
  return HOPS_OK;
}

extern "C" int hops_step_fusion(int32_t mode) {
  if (mode < 0 || mode > 2) return set_err(HOPS_EINVAL, "step fusion must be 0 (auto), 1 or 2");
  g_fusion = mode;
  return HOPS_OK;
}

extern "C" int hops_stage_tuning(int32_t nb, int32_t chunk_major) {
  if (nb != 0 && nb != 1 && nb != 2 && nb != 4 && nb != 8)
    return set_err(HOPS_EINVAL, "nb must be 0 (auto), 1, 2, 4 or 8");
  if (chunk_major < -1 || chunk_major > 3)
    return set_err(HOPS_EINVAL, "task order must be -1 (auto) or 0 .. 3");
  g_tune_nb = nb;
  g_tune_cm = chunk_major;
  return HOPS_OK;
}

template <typename R, typename ST, typename PT, bool SITE, int NB, bool LT>
static void launch_wide_lt(const hops_structure* st, int B, int stage, double h, const void* yin,
                           void* yout, void* phi, void* shadow, void* acc, const double* ws,
                           int chunk_major, cudaStream_t s) {
  const unsigned n_as = (unsigned)st->n_hier * st->n_state;
  const long nchunk = (B + 32 * NB - 1) / (32 * NB);
  // prefix of aux with up connections (order 3); 0 leaves order 3 = order 1
  const int n_pre = st->n_up_prefix > 0 && st->n_up_prefix <= st->n_hier ? st->n_up_prefix : 0;
  constexpr int threads = wide_threads(NB);
  constexpr size_t smem = wide_smem_bytes<ST, PT, NB>(threads / 32);
  // One wave: every CTA is resident from the start, so the warps in flight
  // work on one contiguous window of the task order (with more CTAs than fit,
  // the first wave's warps would stride over the whole task range and no task
  // order would keep a slice of Y in L2).  On the 20-site ring this alone
  // took 5 % off the complex128 stage against 8 waves of grid-stride CTAs.
  static int resident = 0;
  if (resident == 0) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_wide<R, ST, PT, SITE, NB, LT>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_wide<R, ST, PT, SITE, NB, LT>,
                                                      threads, smem) != cudaSuccess || nb < 1)
      nb = 1;
    resident = nb;
  }
  const long task_warps = chunk_major ? (long)n_as * nchunk : (long)n_as;
  long gl = (task_warps * 32 + threads - 1) / threads;
  if (gl > (long)sm_count() * resident) gl = (long)sm_count() * resident;
  const int grid = (int)(gl < 1 ? 1 : gl);
  if (smem > 48 * 1024) {
    // opt in to the large shared-memory carve-out once per device
    static int set_for = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (set_for != dev) {
      cudaFuncSetAttribute(k_wide<R, ST, PT, SITE, NB, LT>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      set_for = dev;
    }
  }
  launch_chain(k_wide<R, ST, PT, SITE, NB, LT>, dim3(grid), dim3(threads), smem, s,
      *st, B, stage, h, (const ST*)yin, (ST*)yout, (PT*)phi, (ST*)shadow, (ST*)acc, ws,
      FastDiv((unsigned)st->n_state), FastDiv(n_as), FastDiv((unsigned)st->n_hier),
      FastDiv(n_pre > 0 ? (unsigned)n_pre : 1u), (unsigned)n_pre * st->n_state, chunk_major);
}

// The low-temperature term is a separate instantiation: the check alone in the
// per-segment update measured 9 % on kernels without a correction.
template <typename R, typename ST, typename PT, bool SITE, int NB>
static void launch_wide(const hops_structure* st, int B, int stage, double h, const void* yin,
                        void* yout, void* phi, void* shadow, void* acc, const double* ws,
                        int chunk_major, cudaStream_t s) {
  if (st->lt_coef)
    launch_wide_lt<R, ST, PT, SITE, NB, true>(st, B, stage, h, yin, yout, phi, shadow, acc, ws,
                                              chunk_major, s);
  else
    launch_wide_lt<R, ST, PT, SITE, NB, false>(st, B, stage, h, yin, yout, phi, shadow, acc, ws,
                                               chunk_major, s);
}

// Persistent step kernel (k_persist) for the 128-trajectory task shape.
template <typename R, typename ST, typename PT, bool SITE, bool LT>
static int launch_persist_lt(const hops_structure* st, hops_batch* bt, int it0, int di,
                             int n_steps, double h, double* psi_out, int stage_rows,
                             size_t scal_smem, int chunk_major, cudaStream_t s) {
  constexpr int NB = 4;
  const int B = bt->n_traj;
  const unsigned n_as = (unsigned)st->n_hier * st->n_state;
  const long nchunk = (B + 32 * NB - 1) / (32 * NB);
  const int n_pre = st->n_up_prefix > 0 && st->n_up_prefix <= st->n_hier ? st->n_up_prefix : 0;
  constexpr int threads = wide_threads(NB);
  const size_t smem = std::max(wide_smem_bytes<ST, PT, NB>(threads / 32), scal_smem);
  auto kern = k_persist<R, ST, PT, SITE, NB, LT>;
  // occupancy at the largest shared memory any structure asks for (48 KB
  // scalars at most, wide_smem_bytes otherwise): one value per instantiation
  static int resident = 0;
  static int set_for = -1;
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  const size_t smem_max = std::max(wide_smem_bytes<ST, PT, NB>(threads / 32), (size_t)48 * 1024);
  if (set_for != dev) {
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
    set_for = dev;
  }
  if (resident == 0) {
    int nb = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, smem_max));
    resident = nb < 1 ? 1 : nb;
  }
  const long task_warps = chunk_major ? (long)n_as * nchunk : (long)n_as;
  long gl = (task_warps * 32 + threads - 1) / threads;
  if (gl > (long)sm_count() * resident) gl = (long)sm_count() * resident;
  int grid = (int)(gl < 1 ? 1 : gl);
  const BatchLayout bl(st->n_state, st->n_mode, st->n_lop, B);
  CUDA_TRY(cudaMemsetAsync(bt->work + bl.bar, 0, 4 * sizeof(unsigned), s));
  hops_structure stv = *st;
  hops_batch btv = *bt;
  FastDiv divS((unsigned)st->n_state), divAS(n_as), divH((unsigned)st->n_hier),
      divP(n_pre > 0 ? (unsigned)n_pre : 1u);
  unsigned n_pre_s = (unsigned)n_pre * st->n_state;
  void* args[] = {&stv, &btv, &it0, &di, &n_steps, &h, &psi_out, &stage_rows, &divS, &divAS,
                  &divH, &divP, &n_pre_s, &chunk_major};
  CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(threads), args, smem, s));
  return HOPS_OK;
}

template <typename R, typename ST, typename PT>
static int launch_persist(const hops_structure* st, hops_batch* bt, int it0, int di, int n_steps,
                          double h, double* psi_out, int stage_rows, size_t scal_smem,
                          int chunk_major, cudaStream_t s) {
  if (st->site_projector) {
    if (st->lt_coef)
      return launch_persist_lt<R, ST, PT, true, true>(st, bt, it0, di, n_steps, h, psi_out,
                                                      stage_rows, scal_smem, chunk_major, s);
    return launch_persist_lt<R, ST, PT, true, false>(st, bt, it0, di, n_steps, h, psi_out,
                                                     stage_rows, scal_smem, chunk_major, s);
  }
  if (st->lt_coef)
    return launch_persist_lt<R, ST, PT, false, true>(st, bt, it0, di, n_steps, h, psi_out,
                                                     stage_rows, scal_smem, chunk_major, s);
  return launch_persist_lt<R, ST, PT, false, false>(st, bt, it0, di, n_steps, h, psi_out,
                                                    stage_rows, scal_smem, chunk_major, s);
}

template <typename R, typename ST, typename PT, bool SITE>
static void launch_stage(const hops_structure* st, int B, int stage, double h, const void* yin,
                         void* yout, void* phi, void* shadow, void* acc, const double* ws,
                         int32_t* status, cudaStream_t s) {
  (void)status;
  if (B >= 32) {
    const int nbmax = (B + 31) / 32;
    // auto (measured on the 20-site ring, 128 trajectories, every precision):
    // 128 trajectories per warp task, the interior aux state by state
    // (order 3) when the structure names its up-connected prefix; the
    // autotuner overrides this per problem class
    int cm = g_tune_cm >= 0 ? g_tune_cm : (st->n_up_prefix > 0 ? 3 : 0);
    int nb = g_tune_nb;
    if (nb == 0) nb = 4;
    if (nb > nbmax) nb = nbmax >= 4 ? 4 : (nbmax >= 2 ? 2 : 1);
    if (nb > 8) nb = 8;
    if (nb == 1) launch_wide<R, ST, PT, SITE, 1>(st, B, stage, h, yin, yout, phi, shadow, acc, ws, cm, s);
    else if (nb == 2) launch_wide<R, ST, PT, SITE, 2>(st, B, stage, h, yin, yout, phi, shadow, acc, ws, cm, s);
    else if (nb == 4) launch_wide<R, ST, PT, SITE, 4>(st, B, stage, h, yin, yout, phi, shadow, acc, ws, cm, s);
    else launch_wide<R, ST, PT, SITE, 8>(st, B, stage, h, yin, yout, phi, shadow, acc, ws, cm, s);
  } else {
    const int grid = grid_for_warps(st->n_hier);
    if (st->n_state * B >= 64 && sizeof(ST) == 16)
      launch_chain(k_narrow<R, ST, PT, SITE, HOPS_NARROW_BIG_MINB>, dim3(grid), dim3(256), 0, s, *st, B, stage, h,
                   (const ST*)yin, (ST*)yout, (PT*)phi, (ST*)shadow, (ST*)acc, ws,
                   FastDiv((unsigned)B));
    else
      launch_chain(k_narrow<R, ST, PT, SITE, 4>, dim3(grid), dim3(256), 0, s, *st, B, stage, h,
                   (const ST*)yin, (ST*)yout, (PT*)phi, (ST*)shadow, (ST*)acc, ws,
                   FastDiv((unsigned)B));
  }
}

template <typename R, typename ST, typename PT>
static int run_stage(const hops_structure* st, int B, int stage, double h, const void* yin,
                     void* yout, void* phi, void* shadow, void* acc, const double* ws,
                     int32_t* status, cudaStream_t s) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (g_timing) {
    e0 = timing_event();
    e1 = timing_event();
    if (e0) cudaEventRecord(e0, s);
  }
  if (st->site_projector)
    launch_stage<R, ST, PT, true>(st, B, stage, h, yin, yout, phi, shadow, acc, ws, status, s);
  else
    launch_stage<R, ST, PT, false>(st, B, stage, h, yin, yout, phi, shadow, acc, ws, status, s);
  LAUNCH_CHECK();
  if (g_timing && e1) cudaEventRecord(e1, s);
  return HOPS_OK;
}

static size_t scalar_smem(const hops_structure* st) {
  return (size_t)(32 + 4 * st->n_lop + 2) * sizeof(double);
}

// Shared memory of k_scalars with the rows of psi_0 and the first-order aux
// staged (stage_rows = 1), or 0 when they do not fit in 48 KB.
static size_t scalar_smem_rows(const hops_structure* st) {
  const size_t b = scalar_smem(st) + (size_t)(1 + st->n_first) * st->n_state * 16;
  return b <= 48 * 1024 ? b : 0;
}

template <typename R, typename ST, typename PT>
static int propagate_impl(const hops_structure* st, hops_batch* bt, int32_t it0, int32_t di,
                          int32_t n_steps, double h, double* psi_out, cudaStream_t s) {
  const int B = bt->n_traj, S = st->n_state;
  const size_t smem_rows = scalar_smem_rows(st);
  const int stage_rows = smem_rows ? 1 : 0;
  const size_t smem = stage_rows ? smem_rows : scalar_smem(st);
  const bool normalized = bt->eom == HOPS_EOM_NORMALIZED_NONLINEAR;
  const size_t psi_stride = (size_t)B * S * 2;
  void* shadow = bt->precision == HOPS_PREC_MIXED ? bt->phi_lo : nullptr;
  // the persistent step kernel: 128 trajectories per task (or the automatic
  // shape) and fusion switched on
  const int cm = g_tune_cm >= 0 ? g_tune_cm : (st->n_up_prefix > 0 ? 3 : 0);
  const bool persist = g_fusion == 2 && B >= 32 && (g_tune_nb == 0 || g_tune_nb == 4);
  if (persist && n_steps > 0) {
    int rc = launch_persist<R, ST, PT>(st, bt, it0, di, n_steps, h, psi_out, stage_rows, smem,
                                       cm, s);
    if (rc) return rc;
  }
  for (int n = 0; n < (persist ? 0 : n_steps); ++n) {
    for (int i = 0; i < 4; ++i) {
      const int slot = i == 0 ? 0 : (i == 3 ? 2 : 1);
      const int it = it0 + 2 * n * di + slot * di;
      // stage 0 gathers from the state (or its complex64 copy in mixed mode)
      const void* yin = i == 0 ? (shadow ? shadow : bt->phi)
                               : (i == 1 ? bt->y0 : (i == 2 ? bt->y1 : bt->y0));
      void* yout = i == 0 ? bt->y0 : (i == 1 ? bt->y1 : (i == 2 ? bt->y0 : nullptr));
      const int recompute = (i == 0 && n > 0 && normalized) ? 1 : 0;
      double* psi_prev = (i == 0 && n > 0 && psi_out) ? psi_out + (size_t)(n - 1) * psi_stride : nullptr;
      launch_chain(k_scalars<R, ST, PT>, dim3(B), dim3(128), smem, s, *st, *bt, i, it, h, yin,
                   recompute, psi_prev, (const float*)nullptr, (const float*)nullptr,
                   (double*)nullptr, stage_rows);
      LAUNCH_CHECK();
      int rc = run_stage<R, ST, PT>(st, B, i, h, yin, yout, bt->phi, shadow, bt->acc, bt->work,
                                    bt->status, s);
      if (rc) return rc;
    }
  }
  if (n_steps > 0) {
    double* psi_last = psi_out ? psi_out + (size_t)(n_steps - 1) * psi_stride : nullptr;
    k_finalize<PT><<<B, 128, 0, s>>>(*st, *bt, psi_last, normalized ? 1 : 0);
    LAUNCH_CHECK();
    if (normalized && !bt->defer_scale) {
      const size_t E = (size_t)st->n_hier * B * S;
      long blocks = (long)((E + 255) / 256);
      if (blocks > (long)sm_count() * 8) blocks = (long)sm_count() * 8;
      const ScalarLayout lay(S, st->n_mode, st->n_lop);
      const BatchLayout bl(S, st->n_mode, st->n_lop, B);
      k_apply_scale<PT, ST><<<(int)blocks, 256, 0, s>>>((PT*)bt->phi, (ST*)shadow, B, E,
                                                         bt->work + bl.scaleB);
      LAUNCH_CHECK();
      k_reset<<<(B + 127) / 128, 128, 0, s>>>(bt->work, lay.stride, bl.scaleB, B, nullptr, 0);
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
  const BatchLayout bl(st->n_state, st->n_mode, st->n_lop, bt->n_traj);
  k_reset<<<(bt->n_traj + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
      bt->work, lay.stride, bl.scaleB, bt->n_traj, bt->status, 1);
  LAUNCH_CHECK();
  return HOPS_OK;
}

template <typename PT, typename ST>
static void settle_impl(const hops_structure* st, hops_batch* bt, cudaStream_t s) {
  const int B = bt->n_traj, S = st->n_state;
  const size_t E = (size_t)st->n_hier * B * S;
  long blocks = (long)((E + 255) / 256);
  if (blocks > (long)sm_count() * 8) blocks = (long)sm_count() * 8;
  const ScalarLayout lay(S, st->n_mode, st->n_lop);
  const BatchLayout bl(S, st->n_mode, st->n_lop, B);
  void* shadow = bt->precision == HOPS_PREC_MIXED ? bt->phi_lo : nullptr;
  k_apply_scale<PT, ST><<<(int)blocks, 256, 0, s>>>((PT*)bt->phi, (ST*)shadow, B, E,
                                                     bt->work + bl.scaleB);
  k_reset<<<(B + 127) / 128, 128, 0, s>>>(bt->work, lay.stride, bl.scaleB, B, nullptr, 0);
}

extern "C" int hops_batch_settle(const hops_structure* st, hops_batch* bt, void* stream) {
  int rc = check_structure(st);
  if (rc) return rc;
  if ((rc = check_batch(st, bt))) return rc;
  if (bt->eom != HOPS_EOM_NORMALIZED_NONLINEAR) return HOPS_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (bt->precision == HOPS_PREC_C128)
    settle_impl<double2, double2>(st, bt, s);
  else if (bt->precision == HOPS_PREC_MIXED)
    settle_impl<double2, float2>(st, bt, s);
  else
    settle_impl<float2, float2>(st, bt, s);
  LAUNCH_CHECK();
  return HOPS_OK;
}

// Every argument check of hops_rk4_propagate, done before anything is
// launched (also used by the no-allocation entry point).
int hops_check_propagate_args(const hops_structure* st, const hops_batch* bt, int32_t it0,
                              int32_t di, int32_t n_steps) {
  int rc = check_structure(st);
  if (rc) return rc;
  if ((rc = check_batch(st, bt))) return rc;
  if (n_steps < 0 || it0 < 0 || di < 0) return set_err(HOPS_EINVAL, "negative step/noise index");
  const long last = (long)it0 + 2L * n_steps * di;
  if (n_steps > 0 && bt->noise1 && last >= bt->n_t1)
    return set_err(HOPS_EINVAL, "noise 1 too short: needs index %ld, has %d samples", last, bt->n_t1);
  if (n_steps > 0 && bt->noise2 && last >= bt->n_t2)
    return set_err(HOPS_EINVAL, "noise 2 too short: needs index %ld, has %d samples", last, bt->n_t2);
  if (scalar_smem(st) > 48 * 1024) return set_err(HOPS_ENOTSUP, "too many L operators (%d)", st->n_lop);
  return HOPS_OK;
}

extern "C" int hops_rk4_propagate(const hops_structure* st, hops_batch* bt, int32_t it0,
                                  int32_t di, int32_t n_steps, double tau_over_hbar,
                                  double* psi_out_dev, void* stream) {
  int rc = hops_check_propagate_args(st, bt, it0, di, n_steps);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (bt->precision == HOPS_PREC_C128)
    return propagate_impl<double, double2, double2>(st, bt, it0, di, n_steps, tau_over_hbar, psi_out_dev, s);
  if (bt->precision == HOPS_PREC_MIXED)
    return propagate_impl<double, float2, double2>(st, bt, it0, di, n_steps, tau_over_hbar, psi_out_dev, s);
  return propagate_impl<float, float2, float2>(st, bt, it0, di, n_steps, tau_over_hbar, psi_out_dev, s);
}

template <typename R, typename ST, typename PT>
static int dsys_impl(const hops_structure* st, hops_batch* bt, const float* z1, const float* z2,
                     void* dphi, double* dz, cudaStream_t s) {
  const size_t smem_rows = scalar_smem_rows(st);
  k_scalars<R, ST, PT><<<bt->n_traj, 128, smem_rows ? smem_rows : scalar_smem(st), s>>>(
      *st, *bt, 4, 0, 0.0, bt->phi, 0, nullptr, z1, z2, dz, smem_rows ? 1 : 0);
  LAUNCH_CHECK();
  // stage 4 reads the state itself (mixed mode: its complex64 copy)
  const void* yin = bt->precision == HOPS_PREC_MIXED ? bt->phi_lo : bt->phi;
  return run_stage<R, ST, PT>(st, bt->n_traj, 4, 0.0, yin, dphi, bt->phi, nullptr, bt->acc,
                              bt->work, bt->status, s);
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
  if (bt->precision == HOPS_PREC_C128)
    return dsys_impl<double, double2, double2>(st, bt, z1_dev, z2_dev, dphi_dev, dzmem_dev, s);
  if (bt->precision == HOPS_PREC_MIXED)
    return dsys_impl<double, float2, double2>(st, bt, z1_dev, z2_dev, dphi_dev, dzmem_dev, s);
  return dsys_impl<float, float2, float2>(st, bt, z1_dev, z2_dev, dphi_dev, dzmem_dev, s);
}

static size_t resident_sc_doubles(int max_sc) { return (size_t)((max_sc + 1) & ~1); }

template <typename R, typename ST, typename PT>
static int resident_impl(hops_task* tasks, int n_tasks, int max_elems, int max_sc, int site,
                         cudaStream_t s) {
  using T = ST;
  int dev = 0, optin = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t scb = resident_sc_doubles(max_sc) * sizeof(double);
  const size_t budget = (size_t)optin - sizeof(hops_structure) - 32 * sizeof(double) - 64;
  const size_t full = scb + (size_t)max_elems * (sizeof(PT) + 3 * sizeof(T));
  const size_t half = scb + 2 * (size_t)max_elems * sizeof(T);
  int mode = 0;
  size_t smem = scb;
  if (full <= budget) {
    mode = 2;
    smem = full;
  } else if (half <= budget) {
    mode = 1;
    smem = half;
  } else if (scb > budget) {
    return set_err(HOPS_ENOTSUP, "resident scalar block of %zu bytes exceeds shared memory", scb);
  }
  int threads = ((max_elems + 31) / 32) * 32;
  if (threads < 64) threads = 64;
  if (threads > 512) threads = 512;
  const int scd = (int)resident_sc_doubles(max_sc);
  if (site) {
    CUDA_TRY(cudaFuncSetAttribute(k_resident<R, ST, PT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_resident<R, ST, PT, true><<<n_tasks, threads, smem, s>>>(tasks, mode, max_elems, scd);
  } else {
    CUDA_TRY(cudaFuncSetAttribute(k_resident<R, ST, PT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_resident<R, ST, PT, false><<<n_tasks, threads, smem, s>>>(tasks, mode, max_elems, scd);
  }
  LAUNCH_CHECK();
  return HOPS_OK;
}

extern "C" int hops_resident_propagate(hops_task* tasks_dev, int32_t n_tasks, int32_t max_elems,
                                       int32_t max_scalar_doubles, int32_t precision,
                                       int32_t all_site_projector, void* stream) {
  if (!tasks_dev || n_tasks <= 0 || max_elems <= 0 || max_scalar_doubles <= 0)
    return set_err(HOPS_EINVAL, "bad resident launch arguments");
  cudaStream_t s = (cudaStream_t)stream;
  if (precision == HOPS_PREC_C128)
    return resident_impl<double, double2, double2>(tasks_dev, n_tasks, max_elems,
                                                   max_scalar_doubles, all_site_projector, s);
  if (precision == HOPS_PREC_MIXED)
    return resident_impl<double, float2, double2>(tasks_dev, n_tasks, max_elems,
                                                  max_scalar_doubles, all_site_projector, s);
  if (precision == HOPS_PREC_C64)
    return resident_impl<float, float2, float2>(tasks_dev, n_tasks, max_elems,
                                                max_scalar_doubles, all_site_projector, s);
  return set_err(HOPS_EINVAL, "unknown precision %d", precision);
}

extern "C" int32_t hops_resident_scalar_doubles(int32_t n_state, int32_t n_mode, int32_t n_lop) {
  const ScalarLayout lay(n_state, n_mode, n_lop);
  return lay.stride + 2 * n_mode + 4 * n_lop + 2;
}

// ================================================== adaptive flux errors ====
// Error estimates of the adaptive basis update for a list of trajectories, one
// CTA each (basis/basis_functions_adaptive.py):
//   e_deriv[a*S+s] = |dPhi/dt / hbar + Phi / dt|^2           (error_deriv, :10-74)
//                    with Phi zeroed on aux whose mask entry is 0 (stable-aux
//                    variant used for the state basis) and e_deriv = 0 there
//   e_up[m*N+a]    = |w_m|^2 (1 + k_m(a))^2 sum_s |L_m[s,s]|^2 |Phi[s,a]|^2 / hbar^2
//                                                             (error_flux_up_hier_stable, :165-266)
//   e_down[m*N+a]  = |g_m/w_m|^2 sum_s |L_m[s,s] - <L_m>|^2 |Phi[s,a]|^2 / hbar^2
//                                                             (error_flux_down_hier_stable, :517-624)
// <L_m> is the expectation in the unmasked psi_0 (hops_basis.py:1105-1112);
// for modes whose L has no diagonal entry at s the diagonal is 0.  All FP64.
__global__ void __launch_bounds__(256) k_flux_errors(hops_flux_task* tasks, double hbar) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ hops_structure st;
  __shared__ double red[32];
  hops_flux_task* tk = tasks + blockIdx.x;
  if (threadIdx.x == 0) st = *tk->st;
  __syncthreads();
  const int S = st.n_state, M = st.n_mode, L = st.n_lop, N = st.n_hier;
  const int E = N * S;
  const ScalarLayout lay(S, M, L);
  double* ws = reinterpret_cast<double*>(smraw);
  double* sh = ws + lay.stride;                 // 4L + 2 doubles
  double* zdummy = sh + 4 * L + 2;              // 2M doubles (dz of the single derivative)
  const double2* phi = reinterpret_cast<const double2*>(tk->phi);
  const int32_t* mask = tk->aux_mask;
  // <L> of the unmasked psi_0 for e_down (hops_basis.py psi setter)
  double2* avg_full = reinterpret_cast<double2*>(zdummy + 2 * M);  // L doubles2
  {
    double p = 0.0;
    for (int s = threadIdx.x; s < S; s += blockDim.x) {
      const double2 v = phi[s];
      p += v.x * v.x + v.y * v.y;
    }
    const double n2 = block_sum(p, red);
    for (int j = threadIdx.x; j < L; j += blockDim.x) {
      double2 num = mk(0.0, 0.0);
      const int base = j * (S + 1);
      for (int r = 0; r < S; ++r) {
        const int q0 = st.l_ptr[base + r], q1 = st.l_ptr[base + r + 1];
        if (q0 == q1) continue;
        double2 row = mk(0.0, 0.0);
        for (int q = q0; q < q1; ++q) row = cfma(ld2(st.l_val, q), phi[st.l_col[q]], row);
        num = cadd(num, cconjmul(phi[r], row));
      }
      avg_full[j] = mk(num.x / n2, num.y / n2);
    }
  }
  StageIO io;
  io.zmem = tk->zmem;
  io.noise1 = tk->z1;
  io.noise2 = tk->z2;
  io.n_t1 = 1;
  io.n_t2 = 1;
  io.noise_c128 = 0;
  io.it = 0;
  io.stage = 4;
  io.eom = tk->eom;
  io.h = 0.0;
  io.ws = ws;
  io.zmem_out = zdummy;
  auto get = [&](int a, int s) -> double2 {
    return (mask && !mask[a]) ? mk(0.0, 0.0) : phi[a * S + s];
  };
  stage_scalars(st, io, get, red, sh);
  const CoefWS<double> cf{ws, lay};
  auto y = [&](int x, int sp) -> double2 { return (mask && !mask[x]) ? mk(0.0, 0.0) : phi[x * S + sp]; };
  const double inv_dt = 1.0 / tk->dt, inv_h = 1.0 / hbar;
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    const int a = e / S, s = e - a * S;
    double val = 0.0;
    if (!mask || mask[a]) {
      double2 k = st.site_projector ? deriv_elem<double, true>(st, a, s, y, cf)
                                    : deriv_elem<double, false>(st, a, s, y, cf);
      if (st.lt_coef && a == 0) k = cadd(k, cf.phys(s));  // LT term of psi_0
      const double2 ph = phi[e];
      const double re = k.x * inv_h + ph.x * inv_dt, im = k.y * inv_h + ph.y * inv_dt;
      val = re * re + im * im;
    }
    tk->e_deriv[e] = val;
  }
  if (tk->e_up) {
    const double ih2 = inv_h * inv_h;
    for (int i = threadIdx.x; i < M * N; i += blockDim.x) {
      const int m = i / N, a = i - m * N;
      const int j = st.mode_lop[m];
      const int base = j * (S + 1);
      const double2 w = ld2(st.mode_w, m), gw = ld2(st.mode_gw, m);
      const double w2 = w.x * w.x + w.y * w.y, gw2 = gw.x * gw.x + gw.y * gw.y;
      // k_m(a): depth of aux a in mode m (K2_aux_by_mode, hops_basis.py:1128-1140)
      const int km = tk->k_aux[i];
      const double2 al = avg_full[j];
      double sup = 0.0, sdn = 0.0;
      for (int s = 0; s < S; ++s) {
        double2 d = mk(0.0, 0.0);
        for (int q = st.l_ptr[base + s]; q < st.l_ptr[base + s + 1]; ++q)
          if (st.l_col[q] == s) d = ld2(st.l_val, q);
        const double2 v = phi[a * S + s];
        const double p2 = v.x * v.x + v.y * v.y;
        sup += (d.x * d.x + d.y * d.y) * p2;
        const double2 dd = csub(d, al);
        sdn += (dd.x * dd.x + dd.y * dd.y) * p2;
      }
      const double f = 1.0 + km;
      tk->e_up[i] = w2 * f * f * sup * ih2;
      tk->e_down[i] = gw2 * sdn * ih2;
    }
  }
}

extern "C" int32_t hops_flux_errors_smem_doubles(int32_t n_state, int32_t n_mode, int32_t n_lop) {
  const ScalarLayout lay(n_state, n_mode, n_lop);
  return lay.stride + 4 * n_lop + 2 + 2 * n_mode + 2 * n_lop + 2;
}

extern "C" int hops_flux_errors(hops_flux_task* tasks_dev, int32_t n_tasks, int32_t max_smem_doubles,
                                double hbar, void* stream) {
  if (!tasks_dev || n_tasks <= 0 || max_smem_doubles <= 0)
    return set_err(HOPS_EINVAL, "bad flux-error launch arguments");
  const size_t smem = (size_t)max_smem_doubles * sizeof(double);
  if (smem > 200 * 1024) return set_err(HOPS_ENOTSUP, "flux-error scalar block too large");
  CUDA_TRY(cudaFuncSetAttribute(k_flux_errors, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_flux_errors<<<n_tasks, 256, smem, (cudaStream_t)stream>>>(tasks_dev, hbar);
  LAUNCH_CHECK();
  return HOPS_OK;
}
