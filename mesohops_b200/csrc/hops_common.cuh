// Shared device helpers of the HOPS trajectory kernels (complex arithmetic and
// the per-stage FP64 scalars of the normalized nonlinear equation of motion).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/hops_b200.h"

// Host helpers shared by the library's translation units (not part of the C ABI).
// hops_set_error_text: replace the calling thread's last-error text.
// hops_check_propagate_args: every argument check of hops_rk4_propagate.
void hops_set_error_text(const char* msg);
int hops_check_propagate_args(const hops_structure* st, const hops_batch* bt, int32_t it0,
                              int32_t di, int32_t n_steps);

namespace hops {

// ---------------------------------------------------------------- complex ----
template <typename R> struct cplx;
template <> struct cplx<double> { using T = double2; };
template <> struct cplx<float> { using T = float2; };

__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 mkf(float x, float y) { return make_float2(x, y); }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return mk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return mkf(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return mk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return mkf(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return mk(a.x, -a.y); }
__device__ __forceinline__ float2 cconj(float2 a) { return mkf(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return mk(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return mkf(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return mkf(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * b + c
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(a.y, b.x, c.y);
  return c;
}
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
  c.x = fmaf(a.x, b.x, c.x);
  c.x = fmaf(-a.y, b.y, c.x);
  c.y = fmaf(a.x, b.y, c.y);
  c.y = fmaf(a.y, b.x, c.y);
  return c;
}
// conj(a) * b
__device__ __forceinline__ double2 cconjmul(double2 a, double2 b) {
  return mk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
template <typename T> __device__ __forceinline__ T czero();
template <> __device__ __forceinline__ double2 czero<double2>() { return mk(0.0, 0.0); }
template <> __device__ __forceinline__ float2 czero<float2>() { return mkf(0.f, 0.f); }
__device__ __forceinline__ double2 to_d(float2 a) { return mk((double)a.x, (double)a.y); }
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
template <typename T> __device__ __forceinline__ T from_d(double2 a);
template <> __device__ __forceinline__ double2 from_d<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 from_d<float2>(double2 a) {
  return mkf((float)a.x, (float)a.y);
}
__device__ __forceinline__ double2 ld2(const double* p, int i) {
  return reinterpret_cast<const double2*>(p)[i];
}
__device__ __forceinline__ float2 ld2f(const float* p, int i) {
  return reinterpret_cast<const float2*>(p)[i];
}
__device__ __forceinline__ bool finite2(double2 a) { return isfinite(a.x) && isfinite(a.y); }

// ------------------------------------------------------- scalar workspace ----
// Per-trajectory FP64 scalars of one RK stage (layout of hops_batch.work).
struct ScalarLayout {
  int S, M, L;
  int stride;  // doubles per trajectory
  __host__ __device__ ScalarLayout(int s, int m, int l) : S(s), M(m), L(l) {
    int n = 4 + 6 * L + 7 * M + 6 * S;
    stride = (n + 1) & ~1;
  }
  __host__ __device__ int scale() const { return 0; }
  __host__ __device__ int nc() const { return 1; }
  __host__ __device__ int n2() const { return 2; }
  __host__ __device__ int avgL() const { return 4; }
  __host__ __device__ int cz() const { return 4 + 2 * L; }
  __host__ __device__ int zst() const { return 4 + 4 * L; }
  __host__ __device__ int zacc() const { return 4 + 4 * L + 2 * M; }
  __host__ __device__ int upc() const { return 4 + 4 * L + 4 * M; }
  __host__ __device__ int diagD() const { return 4 + 4 * L + 6 * M; }
  // low-temperature correction: additive term of the physical wavefunction
  // (aux 0) per state, and <L_j^2>
  __host__ __device__ int phys() const { return 4 + 4 * L + 6 * M + 2 * S; }
  __host__ __device__ int avgL2() const { return 4 + 4 * L + 6 * M + 4 * S; }
  // float2 copies last: every complex-double field above starts at an even
  // offset (16-byte aligned), whatever the parity of M and S
  __host__ __device__ int upc_f() const { return 4 + 6 * L + 6 * M + 4 * S; }   // M float2
  __host__ __device__ int diagD_f() const { return 4 + 6 * L + 7 * M + 4 * S; } // S float2
  __host__ __device__ int phys_f() const { return 4 + 6 * L + 7 * M + 5 * S; }  // S float2
};

// Workspace of a batch: B per-trajectory ScalarLayout blocks followed by the
// stage coefficients in trajectory-fastest layout ([m][b], [s][b], [j][b]) so
// that the stage kernel reads them coalesced.
struct BatchLayout {
  // bar: 16 bytes (four uint32: arrivals, generation, error, spare) of the
  // grid barrier of the persistent step kernel
  size_t upcT, upcT_f, diagT, diagT_f, czT, czT_f, ncB, scaleB, physT, physT_f, bar, total;  // doubles
  __host__ __device__ static size_t even(size_t x) { return (x + 1) & ~(size_t)1; }
  __host__ __device__ BatchLayout(int S, int M, int L, int B) {
    const ScalarLayout lay(S, M, L);
    upcT = even((size_t)lay.stride * B);
    upcT_f = upcT + 2 * (size_t)M * B;
    diagT = even(upcT_f + (size_t)M * B);
    diagT_f = diagT + 2 * (size_t)S * B;
    czT = even(diagT_f + (size_t)S * B);
    czT_f = czT + 2 * (size_t)L * B;
    ncB = even(czT_f + (size_t)L * B);
    scaleB = ncB + B;
    physT = even(scaleB + B);            // LT term of aux 0, [s][b] complex
    physT_f = physT + 2 * (size_t)S * B;
    bar = even(physT_f + (size_t)S * B);
    total = bar + 2;
  }
};

// Stage constants of classic RK4 (integrator_rk.py:29-30).
__device__ __forceinline__ double rk_c(int i) { return i == 0 ? 0.0 : (i == 3 ? 1.0 : 0.5); }
__device__ __forceinline__ int rk_noise_slot(int i) { return i == 0 ? 0 : (i == 3 ? 2 : 1); }

// Block reduction of a double (all threads call; result valid in every thread).
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = (l < nw) ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (l == 0) red[0] = t;
  }
  __syncthreads();
  double r = red[0];
  __syncthreads();
  return r;
}

// Noise sample i of a row stored as complex64 or complex128.
__device__ __forceinline__ double2 noise_at(const void* p, size_t i, int c128) {
  if (c128) return reinterpret_cast<const double2*>(p)[i];
  const float2 v = reinterpret_cast<const float2*>(p)[i];
  return mk((double)v.x, (double)v.y);
}

struct StageIO {
  // inputs
  const double* zmem;   // [M] noise memory at the start of the step
  const void* noise1;   // [L][n_t1] of this trajectory (complex64, or complex128
  const void* noise2;   // if noise_c128); noise2 [L][n_t2] or null
  int n_t1, n_t2;
  int noise_c128;
  int it;               // noise time index of this stage
  int stage;            // 0..3, or 4 = single derivative (no RK bookkeeping)
  int eom;
  double h;             // tau / hbar
  // in/out (this trajectory's scalars)
  double* ws;           // ScalarLayout block of this trajectory
  double* zmem_out;     // final z_mem written at stage 3 (and dz at stage 4)
};

// Computes <L_j>, the noise coefficients cz_j = zhat_j - i z2_j, the norm
// correction, the z_mem RK4 bookkeeping and the derived per-state / per-mode
// coefficients for one trajectory.  Restates eom/eom_functions.py:11-213 and
// the z_mem half of integrator/integrator_rk.py:10-75.
//   get(a, s): stage-input element (aux a, state s) of this trajectory as double2.
//   getf(f, s): the same for the f-th first-order aux (st.first_aux[f]).
// All threads of the block must call it; red / sh are shared scratch
// (red >= 32 doubles, sh >= 4*L + 2 doubles).
template <class Get, class GetF>
__device__ void stage_scalars(const hops_structure& st, const StageIO& io, Get get, GetF getf,
                              double* red, double* sh) {
  const int S = st.n_state, M = st.n_mode, L = st.n_lop;
  ScalarLayout lay(S, M, L);
  double* ws = io.ws;
  const bool linear = io.eom == HOPS_EOM_LINEAR;
  const bool normalized = io.eom == HOPS_EOM_NORMALIZED_NONLINEAR;
  double2* avgL = reinterpret_cast<double2*>(sh);       // [L]
  double2* zhat = reinterpret_cast<double2*>(sh + 2 * L);  // [L]

  // |psi_0|^2
  double p = 0.0;
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double2 v = get(0, s);
    p += v.x * v.x + v.y * v.y;
  }
  const double n2 = block_sum(p, red);

  // <L_j> = psi0^H L_j psi0 / psi0^H psi0 (active L only), and zhat_j.
  for (int j = threadIdx.x; j < L; j += blockDim.x) {
    double2 num = mk(0.0, 0.0);
    const bool act = st.lop_active[j] != 0;
    if (!linear && act) {
      if (st.site_projector) {
        // L_j = v_j |s_j><s_j|: the one nonzero row, same operations as below
        const int sj = st.lop_site[j];
        if (sj >= 0) {
          const double2 row = cfma(ld2(st.lop_sval, j), get(0, sj), mk(0.0, 0.0));
          num = cadd(num, cconjmul(get(0, sj), row));
        }
      } else {
        const int base = j * (S + 1);
        for (int r = 0; r < S; ++r) {
          int q0 = st.l_ptr[base + r], q1 = st.l_ptr[base + r + 1];
          if (q0 == q1) continue;
          double2 row = mk(0.0, 0.0);
          for (int q = q0; q < q1; ++q) row = cfma(ld2(st.l_val, q), get(0, st.l_col[q]), row);
          num = cadd(num, cconjmul(get(0, r), row));
        }
      }
      num = mk(num.x / n2, num.y / n2);
    }
    avgL[j] = num;
    double2 ltc = mk(0.0, 0.0);  // conj(c_j) <L_j>: LT term of every aux (calc_LT_corr)
    if (st.lt_coef && !linear && act) {
      const int base = j * (S + 1);
      double2 num2 = mk(0.0, 0.0);
      for (int r = 0; r < S; ++r) {
        const int q0 = st.l2_ptr[base + r], q1 = st.l2_ptr[base + r + 1];
        if (q0 == q1) continue;
        double2 row = mk(0.0, 0.0);
        for (int q = q0; q < q1; ++q) row = cfma(ld2(st.l2_val, q), get(0, st.l2_col[q]), row);
        num2 = cadd(num2, cconjmul(get(0, r), row));
      }
      reinterpret_cast<double2*>(ws + lay.avgL2())[j] = mk(num2.x / n2, num2.y / n2);
      ltc = cmul(cconj(ld2(st.lt_coef, j)), num);
    }
    // compress_zmem: sum of z_mem over the modes of L_j, then + conj(z1).
    const double2 z1 = io.noise1 ? noise_at(io.noise1, (size_t)j * io.n_t1 + io.it, io.noise_c128)
                                 : mk(0.0, 0.0);
    double2 zs = mk(0.0, 0.0);
    if (!linear) {
      const double* zsrc = io.stage == 0 || io.stage == 4 ? io.zmem : ws + lay.zst();
      for (int m = 0; m < M; ++m)
        if (st.mode_lop[m] == j) zs = cadd(zs, ld2(zsrc, m));
    }
    double2 zh = cadd(mk(z1.x, -z1.y), zs);
    zhat[j] = zh;
    const double2 z2 = io.noise2 ? noise_at(io.noise2, (size_t)j * io.n_t2 + io.it, io.noise_c128)
                                 : mk(0.0, 0.0);
    double2 cz = (linear || act) ? mk(zh.x + z2.y, zh.y - z2.x) : mk(0.0, 0.0);
    cz = cadd(cz, ltc);
    // The LINEAR closure forms conj(z1) - 1j*z2 from complex64 samples without
    // any complex128 term, so the reference rounds it to complex64
    // (hops_eom.py:520,535); the float sum of two floats taken in double and
    // rounded once is the correctly rounded float sum.  Complex128 samples
    // (INTERPOLATE) are not rounded.
    if (linear && !io.noise_c128) cz = mk((double)(float)cz.x, (double)(float)cz.y);
    reinterpret_cast<double2*>(ws + lay.cz())[j] = cz;
    reinterpret_cast<double2*>(ws + lay.avgL())[j] = num;
  }
  __syncthreads();

  // Normalisation correction (eom_functions.py:163-213).
  double nc = 0.0;
  if (normalized) {
    double part_re = 0.0;
    if (threadIdx.x == 0) {
      double2 d = mk(0.0, 0.0);
      for (int j = 0; j < L; ++j)
        if (st.lop_active[j]) d = cfma(zhat[j], avgL[j], d);
      part_re = d.x;
      if (st.lt_coef) {
        // calc_LT_corr_to_norm_corr (eom_functions.py:254-281): real part of
        // sum_j Re(c_j) (2 <L_j>^2 - <L_j^2>)
        const double2* a2 = reinterpret_cast<const double2*>(ws + lay.avgL2());
        for (int j = 0; j < L; ++j) {
          if (!st.lop_active[j]) continue;
          const double2 l = avgL[j];
          part_re += ld2(st.lt_coef, j).x * (2.0 * (l.x * l.x - l.y * l.y) - a2[j].x);
        }
      }
    }
    for (int f = threadIdx.x; f < st.n_first; f += blockDim.x) {
      const int m = st.first_mode[f], j = st.mode_lop[m];
      if (!st.lop_active[j]) continue;
      const int base = j * (S + 1);
      double2 t1 = mk(0.0, 0.0), t2 = mk(0.0, 0.0);
      if (st.site_projector) {
        // one nonzero row of L_j: t1 has the single term of row s_j
        for (int r = 0; r < S; ++r) t2 = cadd(t2, cconjmul(get(0, r), getf(f, r)));
        const int sj = st.lop_site[j];
        if (sj >= 0) {
          const double2 row = cfma(ld2(st.lop_sval, j), getf(f, sj), mk(0.0, 0.0));
          t1 = cadd(t1, cconjmul(get(0, sj), row));
        }
      } else {
        for (int r = 0; r < S; ++r) {
          double2 p0 = get(0, r);
          t2 = cadd(t2, cconjmul(p0, getf(f, r)));
          int q0 = st.l_ptr[base + r], q1 = st.l_ptr[base + r + 1];
          if (q0 == q1) continue;
          double2 row = mk(0.0, 0.0);
          for (int q = q0; q < q1; ++q) row = cfma(ld2(st.l_val, q), getf(f, st.l_col[q]), row);
          t1 = cadd(t1, cconjmul(p0, row));
        }
      }
      double2 gw = ld2(st.mode_gw, m);
      // -(g/w) (t1 - <L> t2)
      double2 c = csub(t1, cmul(avgL[j], t2));
      part_re -= (gw.x * c.x - gw.y * c.y);
    }
    nc = block_sum(part_re, red);
  }

  // z_mem derivative, RK4 bookkeeping of z_mem, per-mode up coefficient.
  const double h = io.h;
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    const int j = st.mode_lop[m];
    double2* zst = reinterpret_cast<double2*>(ws + lay.zst());
    double2* zacc = reinterpret_cast<double2*>(ws + lay.zacc());
    double2 z0 = ld2(io.zmem, m);
    double2 zi = (io.stage == 0 || io.stage == 4) ? z0 : zst[m];
    double2 kz = mk(0.0, 0.0);
    double2 upc = mk(0.0, 0.0);
    if (!linear) {
      double2 g = ld2(st.mode_g, m), w = ld2(st.mode_w, m);
      double2 al = st.lop_active[j] ? avgL[j] : mk(0.0, 0.0);
      // calc_delta_zmem: conj(g) <L> - conj(w) z
      kz = csub(cmul(cconj(g), al), cmul(cconj(w), zi));
      upc = cmul(ld2(st.mode_gw, m), cconj(al));
    }
    reinterpret_cast<double2*>(ws + lay.upc())[m] = upc;
    reinterpret_cast<float2*>(ws + lay.upc_f())[m] = mkf((float)upc.x, (float)upc.y);
    if (io.stage == 4) {
      reinterpret_cast<double2*>(io.zmem_out)[m] = kz;
    } else if (io.stage == 0) {
      zacc[m] = kz;
      zst[m] = cadd(z0, cscale(cscale(kz, 0.5), h));
    } else if (io.stage < 3) {
      zacc[m] = cadd(zacc[m], cscale(kz, 2.0));
      zst[m] = cadd(z0, cscale(cscale(kz, rk_c(io.stage + 1)), h));
    } else {
      double2 sum = cadd(zacc[m], kz);
      reinterpret_cast<double2*>(io.zmem_out)[m] = cadd(z0, mk(h * sum.x / 6.0, h * sum.y / 6.0));
    }
  }

  // Per-state diagonal (site-projector form): -nc + sum_j cz_j v_j [s == s_j]
  // + (-iH)[s,s] (the H CSR of such a structure holds the couplings only).
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double2 d = mk(-nc, 0.0);
    if (st.site_projector) {
      const double2* cz = reinterpret_cast<const double2*>(ws + lay.cz());
      for (int j = 0; j < L; ++j)
        if (st.lop_site[j] == s) d = cfma(cz[j], ld2(st.lop_sval, j), d);
      if (st.h_diag) d = cadd(d, ld2(st.h_diag, s));
    }
    reinterpret_cast<double2*>(ws + lay.diagD())[s] = d;
    reinterpret_cast<float2*>(ws + lay.diagD_f())[s] = mkf((float)d.x, (float)d.y);
    if (st.lt_coef) {
      // LT term of the physical wavefunction: nonlinear
      // sum_j (c_j <L_j> L_j - c_j L_j^2) psi_0 (calc_LT_corr), LINEAR
      // -sum_j c_j L_j^2 psi_0 (calc_LT_corr_linear)
      double2 ph = mk(0.0, 0.0);
      for (int j = 0; j < L; ++j) {
        if (!linear && !st.lop_active[j]) continue;
        const double2 c = ld2(st.lt_coef, j);
        const int base = j * (S + 1);
        if (!linear) {
          double2 lp = mk(0.0, 0.0);
          for (int q = st.l_ptr[base + s]; q < st.l_ptr[base + s + 1]; ++q)
            lp = cfma(ld2(st.l_val, q), get(0, st.l_col[q]), lp);
          ph = cfma(cmul(c, avgL[j]), lp, ph);
        }
        double2 l2p = mk(0.0, 0.0);
        for (int q = st.l2_ptr[base + s]; q < st.l2_ptr[base + s + 1]; ++q)
          l2p = cfma(ld2(st.l2_val, q), get(0, st.l2_col[q]), l2p);
        ph = csub(ph, cmul(c, l2p));
      }
      reinterpret_cast<double2*>(ws + lay.phys())[s] = ph;
      reinterpret_cast<float2*>(ws + lay.phys_f())[s] = mkf((float)ph.x, (float)ph.y);
    }
  }
  if (threadIdx.x == 0) {
    ws[lay.nc()] = nc;
    ws[lay.n2()] = n2;
  }
  __syncthreads();
}

template <class Get>
__device__ void stage_scalars(const hops_structure& st, const StageIO& io, Get get, double* red,
                              double* sh) {
  stage_scalars(st, io, get, [&](int f, int s) { return get(st.first_aux[f], s); }, red, sh);
}

}  // namespace hops
